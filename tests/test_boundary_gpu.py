"""The reference-facing boundary beyond device pointers (GPU).

* Texture objects: tests/native/texture_boundary.cpp, a C++ program compiled
  here against include/mvdr.h, solves an input bundle once with its maps as
  device arrays and once with the maps behind cudaTextureObject_t (cudaArrays
  and pitched memory, as Renderer::SolverMaps and CameraObservation hold
  them); the warp fields must be bit-identical.
* The warp field's device view (mvdr_node_se3_device, the counterpart of
  SolvedNodeSE3()) holds the checked copy's values (in the native test) and
  keeps its address.
* Input bundles: a solve replayed from a saved bundle gives the original
  solve's warp field bit for bit.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

from conftest import ROOT, small_scene
from multiviewdynrecon_b200 import LIB_PATH, abi, check, lib
from multiviewdynrecon_b200.solver import NonRigidSolver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib()


def _config(scene):
    return abi.make_config(scene, use_density=True)  # every map of the view in use


def _solved(scene, cfg, gn, pcg):
    s = NonRigidSolver(cfg)
    s.set_solver_input(scene)
    s.solve_non_rigid_alignment(gn, pcg)
    return s


def test_native_texture_boundary(tmp_path):
    scene = small_scene("torso")  # 3 views: two through cudaArrays, one through pitched memory
    cfg = _config(scene)
    s = NonRigidSolver(cfg)
    s.set_solver_input(scene)
    bundle = tmp_path / "torso.mvdrib"
    s.save_input_bundle(bundle)
    exe = tmp_path / "texture_boundary"
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cxx = shutil.which("g++") or shutil.which("c++")
    assert cxx, "a C++ compiler is needed to build the native test"
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(cuda, "include"), os.path.join(ROOT, "tests", "native", "texture_boundary.cpp"),
                    "-L", os.path.dirname(LIB_PATH), "-lmvdr", "-L", os.path.join(cuda, "lib64"), "-lcudart",
                    f"-Wl,-rpath,{os.path.dirname(LIB_PATH)}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(bundle), str(scene.gn_iterations), str(scene.pcg_iterations)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bit-identical" in r.stdout


def test_node_se3_device_view_is_the_solver_field():
    """The device view stays at one address across solves and rebinds (the
    native test compares its contents with mvdr_get_node_se3)."""
    scene = small_scene("torso")
    s = _solved(scene, _config(scene), 2, 10)
    p0 = s.node_se3_device()
    assert p0
    s.set_solver_input(scene)
    s.solve_non_rigid_alignment(1, 5)
    assert s.node_se3_device() == p0


def test_input_bundle_replays_the_solve(tmp_path):
    scene = small_scene("torso")
    cfg = _config(scene)
    a = _solved(scene, cfg, scene.gn_iterations, scene.pcg_iterations)
    fa = a.solved_node_se3().cpu().numpy()
    path = tmp_path / "b.mvdrib"
    s = NonRigidSolver(cfg)
    s.set_solver_input(scene)
    s.save_input_bundle(path)
    h = C.c_void_p()
    check(lib().mvdr_load_input_bundle(str(path).encode(), C.byref(h)))
    try:
        bcfg = lib().mvdr_input_bundle_config(h).contents
        bin_ = lib().mvdr_input_bundle_inputs(h).contents
        assert bytes(bcfg) == bytes(cfg)
        assert bin_.num_nodes == scene.num_nodes and bin_.num_views == scene.num_views
        b = NonRigidSolver(bcfg)
        check(lib().mvdr_set_inputs_host(b.h, C.byref(bin_), None))
        b.num_nodes = scene.num_nodes
        b.solve_non_rigid_alignment(scene.gn_iterations, scene.pcg_iterations)
        assert np.array_equal(b.solved_node_se3().cpu().numpy().view(np.uint32), fa.view(np.uint32))
        b.close()
    finally:
        lib().mvdr_free_input_bundle(h)
    # a file that is not a bundle is refused
    junk = tmp_path / "junk"
    junk.write_bytes(b"not a bundle at all")
    h2 = C.c_void_p()
    assert lib().mvdr_load_input_bundle(str(junk).encode(), C.byref(h2)) == abi.MVDR_EINVAL
