"""B200-native non-rigid Gauss-Newton solver (MultiViewDynRecon NonRigidSolver stage).

The solver is a C++/CUDA shared library (libmvdr.so, built from csrc/ for
sm_100a) with the C ABI of include/mvdr.h. This package holds its Python
binding (`solver`), the ctypes mirror of the ABI (`abi`) and the synthetic
scene generator (`synth`).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmvdr.so")
CSRC = os.path.join(_HERE, "csrc")
_lib = None


class MvdrError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def build(verbose=False):
    """Compile libmvdr.so for sm_100a (nvcc cross-compiles without a GPU)."""
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-C", CSRC, "-j4"], check=True, stdout=out)
    return LIB_PATH


def _declare(L):
    vp, u32, i32 = C.c_void_p, C.c_uint32, C.c_int
    P = C.POINTER
    sigs = {
        "mvdr_config_default": (None, [P(abi.Config), u32, u32, u32, u32]),
        "mvdr_create": (i32, [P(abi.Config), P(vp)]),
        "mvdr_destroy": (i32, [vp]),
        "mvdr_set_inputs": (i32, [vp, P(abi.Inputs), vp]),
        "mvdr_set_inputs_host": (i32, [vp, P(abi.Inputs), vp]),
        "mvdr_set_inputs_textures": (i32, [vp, P(abi.Inputs), vp, vp]),
        "mvdr_node_se3_device": (i32, [vp, P(vp)]),
        "mvdr_save_input_bundle": (i32, [vp, C.c_char_p, vp]),
        "mvdr_load_input_bundle": (i32, [C.c_char_p, P(vp)]),
        "mvdr_input_bundle_config": (P(abi.Config), [vp]),
        "mvdr_input_bundle_inputs": (P(abi.Inputs), [vp]),
        "mvdr_free_input_bundle": (None, [vp]),
        "mvdr_build_index": (i32, [vp, vp]),
        "mvdr_gn_iteration": (i32, [vp, u32, vp]),
        "mvdr_solve": (i32, [vp, u32, u32, vp]),
        "mvdr_get_node_se3": (i32, [vp, vp, vp]),
        "mvdr_copy_node_se3_async": (i32, [vp, vp, vp]),
        "mvdr_batch_copy_node_se3_async": (i32, [vp, u32, vp, vp]),
        "mvdr_get_counts": (i32, [vp, P(abi.Counts), vp]),
        "mvdr_get_energy": (i32, [vp, P(C.c_double), vp]),
        "mvdr_get_array": (i32, [vp, i32, vp, C.c_size_t, P(C.c_size_t), vp]),
        "mvdr_apply_jtj": (i32, [vp, vp, vp, vp]),
        "mvdr_bsr6_spmv_dot_noalloc": (i32, [u32, u32, vp, vp, vp, vp, vp, vp, vp]),
        "mvdr_batch_create": (i32, [P(abi.Config), u32, P(vp)]),
        "mvdr_batch_destroy": (i32, [vp]),
        "mvdr_batch_set_inputs": (i32, [vp, u32, P(abi.Inputs), vp]),
        "mvdr_batch_set_inputs_host": (i32, [vp, u32, P(abi.Inputs), vp]),
        "mvdr_batch_solve": (i32, [vp, u32, u32, i32, vp]),
        "mvdr_batch_get_node_se3": (i32, [vp, u32, vp, vp]),
        "mvdr_batch_instance": (i32, [vp, u32, P(vp)]),
        "mvdr_batch_autotune": (i32, [vp, vp, P(C.c_double), u32, P(u32), P(u32), P(u32)]),
        "mvdr_batch_set_spmv_shape": (i32, [vp, u32]),
        "mvdr_batch_set_pcg_persistent": (i32, [vp, i32]),
        "mvdr_batch_set_wait_limit": (i32, [vp, C.c_uint64, u32]),
        "mvdr_batch_enqueue_stage": (i32, [vp, i32, vp]),
        "mvdr_render_solver_maps": (i32, [P(abi.SurfelGeometry), P(abi.SolverMapParams), P(abi.SolverMapView), u32,
                                          vp]),
        "mvdr_forward_warp": (i32, [vp, u32, P(abi.DeformSurfels), P(abi.DeformNodes), vp]),
        "mvdr_inverse_warp": (i32, [vp, u32, vp, P(abi.DeformSurfels), vp]),
        "mvdr_compute_node_error": (i32, [vp, P(abi.NodeError), vp]),
        "mvdr_correct_large_error_nodes": (i32, [vp, P(abi.Correction), vp]),
        "mvdr_last_error_string": (C.c_char_p, []),
        "mvdr_kernel_launch_count": (C.c_uint64, []),
        "mvdr_abi_layout": (i32, [C.c_char_p, P(C.c_size_t)]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def lib():
    """The loaded libmvdr.so. Raises if the library has not been built: there
    is no fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MvdrError(abi.MVDR_ESTATE, f"{LIB_PATH} is missing; run multiviewdynrecon_b200.build()")
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def check(status):
    if status != abi.MVDR_OK:
        raise MvdrError(status, lib().mvdr_last_error_string().decode(errors="replace"))
    return status


__all__ = ["abi", "build", "lib", "check", "MvdrError", "LIB_PATH"]
