"""Known-answer tests that pin the CPU oracle (no GPU).

The reference cannot be built or run here and ships no golden vectors, so the
oracle's restatement is checked against mathematics instead:
* dual-quaternion / SE(3) conversions and the twist update against closed forms;
* the 6x6 inverses against numpy;
* the term and node-pair indices against their definitions;
* the assembled JtJ blocks and Jt r against a sparse Jacobian built
  independently in numpy;
* the bin-block SpMV against the dense operator, PCG against a direct solve;
* smooth-term Jacobians against central finite differences;
* the committed golden fixtures (tests/golden) as a regression pin.
"""
import math
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import max_relative_error, rel_norm_error, small_scene
from multiviewdynrecon_b200 import abi, synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rand_rot(rng, scale=1.0):
    return synth.rodrigues(rng.normal(0, scale, 3))


def test_dq_roundtrip(oracle_mod):
    rng = np.random.default_rng(0)
    for _ in range(50):
        R = rand_rot(rng)
        t = rng.normal(0, 0.5, 3)
        dq = synth.se3_to_dq(R[None], t[None])[0]
        m = oracle_mod.dq_to_mat34(dq)
        Rb = m[:9].reshape(3, 3).T
        assert np.allclose(Rb, R, atol=2e-6)
        assert np.allclose(m[9:], t, atol=2e-6)
        back = oracle_mod.mat34_to_dq(m)
        # q and -q are the same rotation
        s = 1.0 if np.dot(back[:4], dq[:4]) > 0 else -1.0
        assert np.allclose(s * back, dq, atol=2e-6)


def test_twist_update_closed_form(oracle_mod):
    rng = np.random.default_rng(1)
    for k in range(30):
        R0, t0 = rand_rot(rng), rng.normal(0, 0.3, 3)
        dq0 = synth.se3_to_dq(R0[None], t0[None])[0].astype(np.float64)
        w = rng.normal(0, 0.05, 3) if k % 5 else np.array([1e-5, -2e-5, 1e-5])
        tw = np.concatenate([w, rng.normal(0, 0.01, 3)])
        out = oracle_mod.apply_twist(dq0, tw)
        m = oracle_mod.dq_to_mat34(out.astype(np.float32))
        # T_new = [exp(w) | t] T_old, identity rotation when sum|w| < 1e-4
        Rw = np.eye(3) if np.abs(w).sum() < 1e-4 else synth.rodrigues(w)
        assert np.allclose(m[:9].reshape(3, 3).T, Rw @ R0, atol=5e-6)
        assert np.allclose(m[9:], Rw @ t0 + tw[3:], atol=5e-6)


def test_block_inverses(oracle_mod):
    rng = np.random.default_rng(2)
    for _ in range(20):
        G = rng.normal(size=(6, 6))
        A = G @ G.T + 0.5 * np.eye(6)
        ref = np.linalg.inv(A)
        assert np.allclose(oracle_mod.cholesky_inverse(A), ref, rtol=1e-10, atol=1e-12)
        assert max_relative_error(oracle_mod.gauss_jordan_inverse(A), ref, 1e-6 * np.abs(ref).max()) < 1e-4


def _run_oracle(oracle_mod, scene, fp64=False, gn=0, pcg=10):
    cfg = abi.make_config(scene)
    o = oracle_mod.Oracle(scene, cfg, fp64=fp64)
    o.build_index()
    for _ in range(gn):
        o.gn_iteration(pcg)
    o.eval_terms()
    o.assemble()
    return o


def _term_node_lists(scene, o):
    """(terms, nodes-of-term) in the reference's term order."""
    c = o.counts()
    knn_d = o.get(abi.ARRAY_DENSE_KNN)
    lists = [tuple(int(x) for x in k) for k in knn_d]
    lists += [tuple(int(x) for x in e) for e in scene.node_graph]
    fg = o.get(abi.ARRAY_FOREGROUND_PIXELS)
    assert len(fg) == c.foreground_terms
    return lists, c


@pytest.mark.parametrize("kind", ["sphere", "torso"])
def test_index_definitions(oracle_mod, kind):
    scene = small_scene(kind)
    o = _run_oracle(oracle_mod, scene)
    c = o.counts()
    # dense pixels: every valid index-map pixel, in scan order, view by view
    pix = o.get(abi.ARRAY_DENSE_PIXELS)
    exp = []
    for v, view in enumerate(scene.views):
        ys, xs = np.nonzero(view.index_map != 0xFFFFFFFF)
        exp.append(np.stack([xs, ys, np.full_like(xs, v), np.zeros_like(xs)], 1))
    exp = np.concatenate(exp, 0)
    assert np.array_equal(pix.astype(np.int64), exp)
    # term -> nodes in reference order (dense, smooth, foreground, feature, cross)
    knn = [o.get(abi.ARRAY_DENSE_KNN)]
    terms = [tuple(int(x) for x in k) for k in knn[0]]
    terms += [tuple(int(x) for x in e) for e in scene.node_graph]
    cfg = abi.make_config(scene)
    fg_pix = o.get(abi.ARRAY_FOREGROUND_PIXELS)
    for (x, y, v, _) in fg_pix:
        s = scene.views[v].index_map[y, x]
        terms.append(tuple(int(a) for a in scene.surfel_knn[s]))
    if cfg.use_feature:
        terms += [tuple(int(a) for a in k) for k in scene.feature.knn]
    if cfg.use_cross_view:
        terms += [tuple(int(a) for a in k) for k in scene.cross_view.knn]
    T = c.dense_terms + c.smooth_terms + c.foreground_terms + c.feature_terms + c.cross_terms
    assert len(terms) == T
    # node -> term: each node lists exactly the terms that contain it, ascending
    off = o.get(abi.ARRAY_NODE2TERM_OFFSET)
    idx = o.get(abi.ARRAY_NODE2TERM_INDEX)
    per_node = [[] for _ in range(scene.num_nodes)]
    for t, nodes in enumerate(terms):
        for n in nodes:
            per_node[n].append(t)
    for n in range(scene.num_nodes):
        assert list(idx[off[n]:off[n + 1]]) == per_node[n]
    # node pair -> term: unique pairs i < j in key order, each with the
    # ascending terms that contain both nodes
    enc = 4096
    pairs = {}
    for t, nodes in enumerate(terms):
        ns = nodes if len(nodes) == 4 else nodes[:2]
        for a in ns:
            for b in ns:
                if a < b:
                    pairs.setdefault(a * enc + b, []).append(t)
    keys = sorted(pairs)
    hk = o.get(abi.ARRAY_HALF_NODEPAIR_KEY)
    assert list(hk) == keys
    npi = o.get(abi.ARRAY_NODEPAIR_TERM_INDEX)
    assert list(npi) == [t for k in keys for t in pairs[k]]
    sym = o.get(abi.ARRAY_NODEPAIR_KEY)
    rng_ = o.get(abi.ARRAY_NODEPAIR_TERM_RANGE)
    sym_exp = sorted(keys + [(k % enc) * enc + k // enc for k in keys])
    assert list(sym) == sym_exp
    for s, key in enumerate(sym):
        i, j = key // enc, key % enc
        h = min(i, j) * enc + max(i, j)
        assert list(npi[rng_[s, 0]:rng_[s, 1]]) == pairs[h]
    blk = o.get(abi.ARRAY_BLKROW_OFFSET)
    rows = sym // enc
    assert np.array_equal(blk, np.searchsorted(rows, np.arange(scene.num_nodes + 1)))


def _sparse_jacobian(scene, o, cfg=None, lam=None, density=0.0):
    """Independent assembly: sparse J (scalar rows x 6N), lambda^2 per row, r.
    `lam` = (smooth, foreground, feature, cross) weights (the global phase by
    default); `density` > 0 adds each dense pixel's density row with that
    weight."""
    c = o.counts()
    cfg = cfg or abi.make_config(scene)
    if lam is None:
        lam = (5.0, 2e-3 if cfg.use_foreground else 0.0, 1.0, 1.0 if cfg.use_cross_view else 0.0)
    jr = o.get(abi.ARRAY_TERM_JACOBIAN)
    sm = o.get(abi.ARRAY_SMOOTH_TERMS)
    wv = o.get(abi.ARRAY_WARPED_CORRESPONDENCE)
    knn_d = o.get(abi.ARRAY_DENSE_KNN)
    w_d = o.get(abi.ARRAY_DENSE_KNN_WEIGHT)
    fg_pix = o.get(abi.ARRAY_FOREGROUND_PIXELS)
    rows, cols, vals, lam2, res = [], [], [], [], []
    row = 0

    def add_row(entries, l2, r):
        nonlocal row
        for (node, jv) in entries:
            for q in range(6):
                rows.append(row)
                cols.append(6 * node + q)
                vals.append(jv[q])
        lam2.append(l2)
        res.append(r)
        row += 1

    Td = c.dense_terms
    for t in range(Td):
        J = jr[t, :6].astype(np.float64)
        add_row([(int(knn_d[t, k]), w_d[t, k] * J) for k in range(4)], 1.0, float(jr[t, 6]))
    if density:
        dj = o.get(abi.ARRAY_DENSITY_JACOBIAN)
        for t in range(Td):
            J = dj[t, :6].astype(np.float64)
            add_row([(int(knn_d[t, k]), w_d[t, k] * J) for k in range(4)], density ** 2, float(dj[t, 6]))

    def skew_rows(p):
        return np.array([[0, p[2], -p[1]], [-p[2], 0, p[0]], [p[1], -p[0], 0]], np.float64)

    for k, (i, j) in enumerate(scene.node_graph):
        s = sm[k].astype(np.float64)
        if s[6] == 0:
            continue
        a, b = s[:3], s[3:6]
        Si, Sj = skew_rows(a), skew_rows(b)
        for ch in range(3):
            Ji = np.concatenate([Si[ch], np.eye(3)[ch]])
            Jj = -np.concatenate([Sj[ch], np.eye(3)[ch]])
            add_row([(int(i), Ji), (int(j), Jj)], lam[0] ** 2, s[8 + ch])
    for f in range(c.foreground_terms):
        x, y, v, _ = fg_pix[f]
        s_id = scene.views[v].index_map[y, x]
        J = jr[Td + f, :6].astype(np.float64)
        add_row([(int(scene.surfel_knn[s_id, k]), scene.surfel_knn_weight[s_id, k] * J) for k in range(4)],
                lam[1] ** 2, float(jr[Td + f, 6]))
    for base, corr, l in ((0, scene.feature if cfg.use_feature else None, lam[2]),
                          (c.feature_terms, scene.cross_view if cfg.use_cross_view else None, lam[3])):
        if corr is None:
            continue
        for k in range(corr.count):
            p = wv[base + k, :3].astype(np.float32)
            raw = wv[base + k, 4:7].astype(np.float32)
            hw = np.where(np.abs(raw) < np.float32(7.5e-2), np.float32(1.0),
                          np.float32(7.5e-2) / np.abs(raw)).astype(np.float32).astype(np.float64)
            S = skew_rows(p.astype(np.float64))
            for ch in range(3):
                Jc = hw[ch] * np.concatenate([S[ch], np.eye(3)[ch]])
                add_row([(int(corr.knn[k, q]), corr.knn_weight[k, q] * Jc) for q in range(4)], l ** 2,
                        hw[ch] * raw[ch])
    n = 6 * scene.num_nodes
    J = sp.csr_matrix((vals, (rows, cols)), shape=(row, n))
    L = sp.diags(np.asarray(lam2))
    A = (J.T @ L @ J).tocsr() + 1e-2 * sp.eye(n, format="csr")
    b = -(J.T @ (np.asarray(lam2) * np.asarray(res)))
    return A, b


@pytest.mark.parametrize("kind", ["sphere", "torso", "torso_rigid"])
def test_assembly_matches_sparse_jacobian(oracle_mod, kind):
    scene = small_scene(kind)
    o = _run_oracle(oracle_mod, scene, fp64=True)
    A, b = _sparse_jacobian(scene, o)
    N = scene.num_nodes
    D = o.get(abi.ARRAY_DIAG_BLOCKS, as_double=True).reshape(N, 6, 6)
    Ad = A.toarray() if N <= 600 else None
    for n in range(N):
        ref = Ad[6 * n:6 * n + 6, 6 * n:6 * n + 6]
        assert max_relative_error(D[n], ref, 1e-9 * max(1.0, np.abs(ref).max())) < 1e-9
    bo = o.get(abi.ARRAY_JTR, as_double=True).reshape(-1)
    assert max_relative_error(bo, b, 1e-9 * np.abs(b).max()) < 1e-8
    sym = o.get(abi.ARRAY_NODEPAIR_KEY)
    off = o.get(abi.ARRAY_OFFDIAG_BLOCKS, as_double=True)
    for s, key in enumerate(sym):
        i, j = key // 4096, key % 4096
        ref = Ad[6 * i:6 * i + 6, 6 * j:6 * j + 6]
        blk = off[s].reshape(6, 6).T  # blk[6k + r] = A(r, k)
        assert max_relative_error(blk, ref, 1e-9 * max(1.0, np.abs(ref).max())) < 1e-8
    # every non-zero block of A is one of the indexed blocks
    nz_blocks = {(r // 6, c // 6) for r, c in zip(*A.nonzero())}
    idx_blocks = {(k // 4096, k % 4096) for k in sym} | {(n, n) for n in range(N)}
    assert nz_blocks <= idx_blocks


@pytest.mark.parametrize("compat", [False, True])
def test_density_terms_match_the_reference_formula(oracle_mod, compat):
    """The oracle's density terms (one per dense pixel) against an independent
    restatement of computeDensityMapJacobian / computeImageDensityJacobainAndResidual."""
    from image_terms import density_terms
    scene = small_scene("torso")
    flags = abi.COMPAT_REF_FOREGROUND_FRAME if compat else 0
    o = oracle_mod.Oracle(scene, abi.make_config(scene, compat_flags=flags, use_density=True), fp64=True)
    o.build_index()
    o.eval_terms()
    dj = o.get(abi.ARRAY_DENSITY_JACOBIAN)
    assert len(dj) == o.counts().dense_terms
    want = density_terms(scene, o.get(abi.ARRAY_DENSE_PIXELS), frame0=not compat)
    pix = np.ascontiguousarray(dj[:, 7]).view(np.uint32).astype(np.int64)
    pix = np.where(pix == abi.MVDR_INVALID_INDEX, -1, pix)
    same = pix == want[:, 7].astype(np.int64)
    assert same.mean() > 0.999
    got = dj.astype(np.float64)
    assert max_relative_error(got[same, :7], want[same, :7], 1e-6 * np.abs(want[:, :7]).max()) < 1e-5
    assert np.abs(want[:, 6]).max() > 0.01  # the term is not trivially zero


def test_density_assembly_matches_sparse_jacobian(oracle_mod):
    """With the density term in the local phase (lambda_density = 1e-2 from
    the first iteration; foreground and feature weights 0), the assembled
    blocks and Jt r equal the independent sparse Jacobian's."""
    scene = small_scene("torso")
    cfg = abi.make_config(scene, use_density=True, num_global_iterations=0)
    o = oracle_mod.Oracle(scene, cfg, fp64=True)
    o.build_index()
    o.eval_terms()
    o.assemble()
    A, b = _sparse_jacobian(scene, o, cfg=cfg, lam=(5.0, 0.0, 0.0, 1.0), density=1e-2)
    N = scene.num_nodes
    Ad = A.toarray()
    D = o.get(abi.ARRAY_DIAG_BLOCKS, as_double=True).reshape(N, 6, 6)
    for n in range(N):
        ref = Ad[6 * n:6 * n + 6, 6 * n:6 * n + 6]
        assert max_relative_error(D[n], ref, 1e-9 * max(1.0, np.abs(ref).max())) < 1e-9
    bo = o.get(abi.ARRAY_JTR, as_double=True).reshape(-1)
    assert max_relative_error(bo, b, 1e-9 * np.abs(b).max()) < 1e-8
    sym = o.get(abi.ARRAY_NODEPAIR_KEY)
    off = o.get(abi.ARRAY_OFFDIAG_BLOCKS, as_double=True)
    for s_, key in enumerate(sym):
        i, j = key // 4096, key % 4096
        ref = Ad[6 * i:6 * i + 6, 6 * j:6 * j + 6]
        assert max_relative_error(off[s_].reshape(6, 6).T, ref, 1e-9 * max(1.0, np.abs(ref).max())) < 1e-8
    # the density rows changed the system
    A0, b0 = _sparse_jacobian(scene, o, cfg=cfg, lam=(5.0, 0.0, 0.0, 1.0), density=0.0)
    assert np.abs(b - b0).max() > 1e-6 * np.abs(b).max()
    # and the energy counts them: sum (lambda_d r_d)^2 on top of the others
    dj = o.get(abi.ARRAY_DENSITY_JACOBIAN).astype(np.float64)
    o2 = oracle_mod.Oracle(scene, abi.make_config(scene, use_density=False, num_global_iterations=0), fp64=True)
    o2.build_index()
    o2.eval_terms()
    o2.assemble()
    # (the kernels and the oracle weight the residual in float: ~1e-7 relative)
    assert math.isclose(o.energy() - o2.energy(), float(((1e-2 * dj[:, 6]) ** 2).sum()), rel_tol=1e-6)


@pytest.mark.parametrize("kind", ["sphere", "torso"])
def test_binblock_spmv_and_pcg(oracle_mod, kind):
    scene = small_scene(kind)
    o = _run_oracle(oracle_mod, scene, fp64=True)
    A, b = _sparse_jacobian(scene, o)
    rng = np.random.default_rng(3)
    x = rng.normal(size=A.shape[0])
    y = o.apply_jtj(x)
    assert rel_norm_error(y, A @ x) < 1e-10
    # PCG converges to the direct solution
    o.pcg(400)
    xs = o.get(abi.ARRAY_INCREMENT, as_double=True).reshape(-1)
    direct = sp.linalg.spsolve(A.tocsc(), b)
    assert rel_norm_error(xs, direct) < 1e-6


def test_smooth_jacobian_finite_difference(oracle_mod):
    """The smooth term's twist Jacobian equals the central difference of its
    residual Ti xj - Tj xj under T <- exp(h e_c) T (exact, no skinning)."""
    scene = small_scene("sphere")
    rng = np.random.default_rng(4)
    cfg = abi.make_config(scene)
    o = oracle_mod.Oracle(scene, cfg, fp64=True)
    o.build_index()
    o.eval_terms()
    sm0 = o.get(abi.ARRAY_SMOOTH_TERMS)
    edges = rng.choice(len(scene.node_graph), 12, replace=False)
    h = 2e-4
    for e in edges:
        i, j = (int(a) for a in scene.node_graph[e])
        a = sm0[e, :3].astype(np.float64)
        Si = np.array([[0, a[2], -a[1]], [-a[2], 0, a[0]], [a[1], -a[0], 0]])
        for c in range(6):
            tw = np.zeros(6)
            tw[c] = h
            res = []
            for sgn in (1, -1):
                dq_i = scene.node_se3[i].astype(np.float64)
                n = oracle_mod.apply_twist(dq_i, sgn * tw).astype(np.float32)
                dq = scene.node_se3.copy()
                dq[i] = n
                s2 = synth.perturb_warp_field(scene, 0)
                s2.node_se3 = dq
                o2 = oracle_mod.Oracle(s2, cfg, fp64=True)
                o2.build_index()
                o2.eval_terms()
                sm = o2.get(abi.ARRAY_SMOOTH_TERMS)[e].astype(np.float64)
                res.append(sm[:3] - sm[3:6])
            fd = (res[0] - res[1]) / (2 * h)
            analytic = np.array([Si[ch, c] if c < 3 else float(ch == c - 3) for ch in range(3)])
            assert np.allclose(fd, analytic, atol=2e-3), (e, c, fd, analytic)


def test_gauss_newton_reduces_energy(oracle_mod):
    scene = small_scene("torso")
    cfg = abi.make_config(scene)
    o = oracle_mod.Oracle(scene, cfg, fp64=False)
    o.build_index()
    energies = []
    for _ in range(4):
        o.eval_terms()
        o.assemble()
        energies.append(o.energy())
        o.pcg(15)
        o.update()
    assert energies[-1] < 0.2 * energies[0]
    assert all(e1 < e0 for e0, e1 in zip(energies, energies[1:]))


def test_compat_view_lookup_only_changes_multiview(oracle_mod):
    scene = small_scene("sphere")
    cfg = abi.make_config(scene, compat_flags=abi.COMPAT_REF_VIEW_LOOKUP)
    a = _run_oracle(oracle_mod, scene)
    o = oracle_mod.Oracle(scene, cfg)
    o.build_index()
    o.eval_terms()
    assert np.array_equal(a.get(abi.ARRAY_TERM_JACOBIAN).view(np.uint32),
                          o.get(abi.ARRAY_TERM_JACOBIAN).view(np.uint32))


@pytest.mark.parametrize("compat", [False, True])
def test_foreground_terms_match_the_reference_formula(oracle_mod, compat):
    """The oracle's foreground terms against an independent restatement of
    computeImageDensityJacobainAndResidual (density_map_jacobian.cuh:12-79):
    by default with the reference vertex moved to frame 0 first, and under
    MVDR_COMPAT_REF_FOREGROUND_FRAME warped in its own camera's frame as the
    reference does. Views 1 and 2 of the torso have InitialCameraSE3 != I,
    so the two forms differ there and agree on view 0."""
    from image_terms import foreground_terms
    scene = small_scene("torso")
    flags = abi.COMPAT_REF_FOREGROUND_FRAME if compat else 0
    o = oracle_mod.Oracle(scene, abi.make_config(scene, compat_flags=flags), fp64=True)
    o.build_index()
    o.eval_terms()
    Td = o.counts().dense_terms
    pix = o.get(abi.ARRAY_FOREGROUND_PIXELS)
    jr = o.get(abi.ARRAY_TERM_JACOBIAN)[Td:]
    got = jr.astype(np.float64)
    want = foreground_terms(scene, pix, frame0=not compat)
    got_pix = np.ascontiguousarray(jr[:, 7]).view(np.uint32).astype(np.int64)
    got_pix = np.where(got_pix == abi.MVDR_INVALID_INDEX, -1, got_pix)
    same = got_pix == want[:, 7].astype(np.int64)
    assert same.mean() > 0.999
    assert max_relative_error(got[same, :7], want[same, :7], 1e-6 * np.abs(want[:, :7]).max()) < 1e-5
    # the other form really differs on the views with a camera offset
    other = foreground_terms(scene, pix, frame0=compat)
    on_v0 = pix[:, 2] == 0
    assert np.allclose(other[on_v0, :7], want[on_v0, :7], rtol=1e-9, atol=1e-12)
    assert np.abs(other[~on_v0, :7] - want[~on_v0, :7]).max() > 1e-3 * np.abs(want[:, :7]).max()


def test_compat_foreground_frame_changes_only_foreground_terms(oracle_mod):
    scene = small_scene("torso")
    a = _run_oracle(oracle_mod, scene)
    o = oracle_mod.Oracle(scene, abi.make_config(scene, compat_flags=abi.COMPAT_REF_FOREGROUND_FRAME))
    o.build_index()
    o.eval_terms()
    Td = a.counts().dense_terms
    ja, jb = a.get(abi.ARRAY_TERM_JACOBIAN), o.get(abi.ARRAY_TERM_JACOBIAN)
    assert np.array_equal(ja[:Td].view(np.uint32), jb[:Td].view(np.uint32))
    assert not np.array_equal(ja[Td:].view(np.uint32), jb[Td:].view(np.uint32))
    for which in (abi.ARRAY_FOREGROUND_PIXELS, abi.ARRAY_NODE2TERM_INDEX, abi.ARRAY_NODEPAIR_KEY):
        assert np.array_equal(a.get(which), o.get(which))


@pytest.mark.parametrize("name", ["sphere_small", "torso_small"])
def test_golden_fixtures(oracle_mod, name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    g = np.load(path)
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    scene = mg.SCENES[name]()
    cfg = abi.make_config(scene)
    o = oracle_mod.Oracle(scene, cfg)
    o.build_index()
    for key in mg.INDEX_ARRAYS:
        assert np.array_equal(o.get(getattr(abi, key)), g[key]), key
    o.eval_terms()
    o.assemble()
    for key in ("ARRAY_DIAG_BLOCKS", "ARRAY_JTR"):
        assert max_relative_error(o.get(getattr(abi, key)), g[key], 1e-6) < 1e-5, key
    o.pcg(scene.pcg_iterations)
    o.update()
    assert max_relative_error(o.get(abi.ARRAY_NODE_SE3), g["ARRAY_NODE_SE3"], 1e-7) < 1e-5
    assert math.isclose(o.energy(), float(g["energy"]), rel_tol=1e-6)


@pytest.mark.parametrize("kind,uniform,tol", [("torso", True, 1e-5), ("body", True, 1e-5),
                                              ("torso", False, 1e-3)])
def test_adjoint_products_match_finite_differences(oracle_mod, kind, uniform, tol):
    """The oracle's own J^T r and J^T J p (FP64) equal central finite
    differences of its weighted residuals on 64 random twist coordinates: to
    rounding on a uniform warp field, where the skinning Jacobian model is
    exact, and to its first-order accuracy on a per-node perturbed field."""
    from fd_adjoint import DAMPING, fd_adjoint_reference, fd_config, random_coords, uniform_field
    scene = small_scene(kind)
    if uniform:
        scene = uniform_field(scene)
    cfg = fd_config(scene)
    rng = np.random.default_rng(21)
    coords = random_coords(rng, scene.num_nodes)
    p = rng.normal(size=len(coords))
    b_fd, jtjp_fd, o = fd_adjoint_reference(oracle_mod, scene, cfg, coords, p)
    o.assemble()
    b = o.get(abi.ARRAY_JTR, as_double=True).reshape(-1, 6)
    b_or = np.array([b[n, c] for n, c in coords])
    assert rel_norm_error(b_or, b_fd) < tol
    x = np.zeros(6 * scene.num_nodes)
    for (n, c), v in zip(coords, p):
        x[6 * n + c] += v
    y = o.apply_jtj(x)
    y_or = np.array([y[6 * n + c] - DAMPING * x[6 * n + c] for n, c in coords])
    assert rel_norm_error(y_or, jtjp_fd) < tol
