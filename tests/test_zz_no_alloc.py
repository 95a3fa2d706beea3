"""mvdr_bsr6_spmv_dot_noalloc: the block SpMV with its fused dot product for
callers that cannot allocate device memory (their GPU memory belongs to another
allocator, or their loop forbids cudaMalloc after start-up).

The entry point keeps its scratch in a static device array, so it is checked
here twice in a row: the second call must not see anything the first one left
behind. Its output is compared with mvdr_apply_jtj, the solver entry point that
applies the same materialised JtJ, and with a float64 numpy product of the
same block-CSR matrix, at the operator tolerance of the parity tests (relative
2-norm 1e-5). A column index outside the matrix skips its block and makes the
dot NaN; the call after it must be clean again. This file is collected last
on purpose.
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


def _numpy_product(rowptr, colidx, blocks, x):
    """y = A x in float64 over the same float blocks, skipping blocks whose
    column is outside the matrix."""
    n = len(rowptr) - 1
    x = np.asarray(x, np.float64).reshape(n, 6)
    y = np.zeros((n, 6))
    for i in range(n):
        for s in range(rowptr[i], rowptr[i + 1]):
            c = colidx[s]
            if 0 <= c < n:
                y[i] += blocks[s].astype(np.float64) @ x[c]
    return y.reshape(-1)


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
    rp_h, ci_h, bl_h = _block_csr(g, n)
    rowptr, colidx, blocks = (torch.from_numpy(a).cuda() for a in (rp_h, ci_h, bl_h))
    gen = torch.Generator(device="cpu").manual_seed(5)
    for call in range(2):
        x = torch.randn(6 * n, generator=gen).cuda()
        y_ref = g.apply_jtj(x)
        y, dot = _noalloc(rowptr, colidx, blocks, x, n)
        torch.cuda.synchronize()
        y_ref64 = y_ref.cpu().numpy().astype(np.float64)
        assert rel_norm_error(y.cpu().numpy(), y_ref64) < 1e-5, call
        y_np = _numpy_product(rp_h, ci_h, bl_h, x.cpu().numpy())
        assert rel_norm_error(y.cpu().numpy(), y_np) < 1e-6, call
        dot_ref = float(np.dot(x.cpu().numpy().astype(np.float64), y_np))
        assert abs(dot.item() - dot_ref) <= 1e-5 * abs(dot_ref), (call, dot.item(), dot_ref)


@pytest.mark.gpu
def test_noalloc_bad_column_then_clean_call():
    """A column index equal to the row count is skipped (the kernel checks it
    before any access) and makes the dot NaN; the shared error flag is cleared
    before the next call, whose result is clean again. Zero block rows give a
    zero dot."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(9)
    n = 300
    rowptr = np.zeros(n + 1, np.int32)
    cols = []
    for i in range(n):
        row = sorted({i, *rng.integers(0, n, 4).tolist()})
        cols += row
        rowptr[i + 1] = len(cols)
    colidx = np.asarray(cols, np.int32)
    blocks = rng.normal(size=(len(colidx), 6, 6)).astype(np.float32)
    x_h = rng.normal(size=6 * n).astype(np.float32)
    bad = colidx.copy()
    bad[7] = n  # one column past the matrix
    x = torch.from_numpy(x_h).cuda()
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    y, dot = _noalloc(dev(rowptr), dev(bad), dev(blocks), x, n)
    torch.cuda.synchronize()
    assert np.isnan(dot.item())
    assert rel_norm_error(y.cpu().numpy(), _numpy_product(rowptr, bad, blocks, x_h)) < 1e-6
    for _ in range(2):
        y, dot = _noalloc(dev(rowptr), dev(colidx), dev(blocks), x, n)
        torch.cuda.synchronize()
        y_np = _numpy_product(rowptr, colidx, blocks, x_h)
        assert rel_norm_error(y.cpu().numpy(), y_np) < 1e-6
        dot_ref = float(np.dot(x_h.astype(np.float64), y_np))
        assert abs(dot.item() - dot_ref) <= 1e-5 * abs(dot_ref)
    zero = torch.zeros(1, dtype=torch.int32, device="cuda")
    dot0 = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    st = lib().mvdr_bsr6_spmv_dot_noalloc(
        0, 0, C.c_void_p(zero.data_ptr()), None, None, C.c_void_p(zero.data_ptr()), C.c_void_p(zero.data_ptr()),
        C.c_void_p(dot0.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert st == abi.MVDR_OK
    assert dot0.item() == 0.0


def test_noalloc_rejects_sizes_above_the_maximum():
    # the size check comes before any CUDA call, so these pointers are never used
    p = C.c_void_p(256)
    st = lib().mvdr_bsr6_spmv_dot_noalloc(MAX_BLOCK_ROWS + 1, 1, p, p, p, p, p, p, None)
    assert st == abi.MVDR_ECAPACITY
    assert b"exceed the maximum" in lib().mvdr_last_error_string()
