import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


def max_relative_error(a, b, small_cutoff):
    """maxRelativeError of the reference (core/NonRigidSolver/sanity_check.cpp:50-73):
    entries whose absolute difference is at most `small_cutoff` are ignored,
    the others are scored by |a - b| / max(|a|, |b|)."""
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    n = min(len(a), len(b))
    a, b = a[:n], b[:n]
    err = np.abs(a - b)
    sel = err > small_cutoff
    if not sel.any():
        return 0.0
    return float((err[sel] / np.maximum(np.abs(a[sel]), np.abs(b[sel]))).max())


def rel_norm_error(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


_SCENES = {}


def small_scene(kind):
    """Small seeded scenes that the CPU oracle handles in well under a second."""
    if kind not in _SCENES:
        from multiviewdynrecon_b200 import synth
        if kind == "sphere":
            s = synth.sphere_single_view(seed=11, num_nodes=384, width=160, height=120)
        elif kind == "sphere_rigid":
            s = synth.sphere_single_view(seed=12, num_nodes=256, width=128, height=96, rigid_offset=True)
        elif kind == "torso":
            s = synth.torso_multi_view(seed=13, num_nodes=512, num_views=3, width=160, height=120,
                                       features_per_view=60, cross_per_pair=80)
        elif kind == "torso_rigid":
            s = synth.torso_multi_view(seed=14, num_nodes=400, num_views=2, width=128, height=96,
                                       features_per_view=40, cross_per_pair=60, rigid_offset=True)
        elif kind == "body":
            s = synth.articulated_body(seed=15, num_nodes=600, num_views=3, width=192, height=108,
                                       cross_total=300)
        else:
            raise KeyError(kind)
        _SCENES[kind] = s
    return _SCENES[kind]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle
