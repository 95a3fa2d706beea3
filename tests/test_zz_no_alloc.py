"""mvdr_bsr6_spmv_dot_noalloc: the block SpMV with its fused dot product for
callers that cannot allocate device memory (their GPU memory belongs to another
allocator, or their loop forbids cudaMalloc after start-up).

The entry point keeps its scratch in a static device array, so it is checked
here twice in a row: the second call must not see anything the first one left
behind. Its output is compared with mvdr_apply_jtj, the solver entry point that
applies the same materialised JtJ, at the operator tolerance of the parity
tests (relative 2-norm 1e-5). This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_norm_error, small_scene
from multiviewdynrecon_b200 import abi, lib
from multiviewdynrecon_b200.solver import NonRigidSolver

MAX_BLOCK_ROWS = 262144  # MVDR_NOALLOC_MAX_BLOCK_ROWS in include/mvdr.h


def _block_csr(solver, n):
    """The solver's damped JtJ as row-major 6x6 block CSR (diagonal block
    first in every block row, then the off-diagonal blocks in key order)."""
    diag = solver.get_array(abi.ARRAY_DIAG_BLOCKS).reshape(n, 6, 6)
    keys = solver.get_array(abi.ARRAY_NODEPAIR_KEY).astype(np.int64)
    off = solver.get_array(abi.ARRAY_OFFDIAG_BLOCKS).reshape(-1, 6, 6)
    off = np.transpose(off, (0, 2, 1))  # exported as blk[6k + r] = A(r, k)
    enc = 4096 if n <= 4096 else 1 << (n - 1).bit_length()
    rows, cols = keys // enc, keys % enc
    rowptr = np.zeros(n + 1, np.int32)
    colidx, blocks = [], []
    for i in range(n):
        sel = np.nonzero(rows == i)[0]
        colidx += [i] + cols[sel].tolist()
        blocks += [diag[i]] + [off[s] for s in sel]
        rowptr[i + 1] = len(colidx)
    return rowptr, np.asarray(colidx, np.int32), np.ascontiguousarray(np.stack(blocks), np.float32)


def _noalloc(rowptr, colidx, blocks, x, n):
    y = torch.empty_like(x)
    dot = torch.empty(1, dtype=torch.float64, device="cuda")
    st = lib().mvdr_bsr6_spmv_dot_noalloc(
        n, colidx.numel(), C.c_void_p(rowptr.data_ptr()), C.c_void_p(colidx.data_ptr()),
        C.c_void_p(blocks.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
        C.c_void_p(dot.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.MVDR_OK, lib().mvdr_last_error_string()
    return y, dot


@pytest.mark.gpu
def test_noalloc_spmv_matches_apply_jtj():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    scene = small_scene("torso")
    n = scene.num_nodes
    cfg = abi.make_config(scene, precision=abi.PRECISION_FP32, mode=abi.MODE_MATERIALIZED)
    g = NonRigidSolver(cfg)
    g.set_solver_input(scene)
    g.build_index()
    g.gn_iteration(scene.pcg_iterations)
    torch.cuda.synchronize()
    rowptr, colidx, blocks = (torch.from_numpy(a).cuda() for a in _block_csr(g, n))
    gen = torch.Generator(device="cpu").manual_seed(5)
    for call in range(2):
        x = torch.randn(6 * n, generator=gen).cuda()
        y_ref = g.apply_jtj(x)
        y, dot = _noalloc(rowptr, colidx, blocks, x, n)
        torch.cuda.synchronize()
        y_ref64 = y_ref.cpu().numpy().astype(np.float64)
        assert rel_norm_error(y.cpu().numpy(), y_ref64) < 1e-5, call
        dot_ref = float(np.dot(x.cpu().numpy().astype(np.float64), y_ref64))
        assert abs(dot.item() - dot_ref) <= 1e-5 * abs(dot_ref), (call, dot.item(), dot_ref)


def test_noalloc_rejects_sizes_above_the_maximum():
    # the size check comes before any CUDA call, so these pointers are never used
    p = C.c_void_p(256)
    st = lib().mvdr_bsr6_spmv_dot_noalloc(MAX_BLOCK_ROWS + 1, 1, p, p, p, p, p, p, None)
    assert st == abi.MVDR_ECAPACITY
    assert b"exceed the maximum" in lib().mvdr_last_error_string()
