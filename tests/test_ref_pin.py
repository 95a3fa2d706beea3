"""Pins the CPU oracle to the reference's own code (no GPU).

oracle/_ref/libref_pin.so is the reference's header-only solver math compiled
from the reference tree (oracle/Makefile, target `ref`; oracle/ref_pin.cu
calls it): the dual-quaternion blend and conversions, the 6x6 Gauss-Jordan
inverse, the Huber weight, the point-to-point and smooth-term Jacobians and
their Jt r, the node-pair encoding and the term-type offsets. Each test feeds
the same seeded inputs to the reference's function and to the oracle's
restatement. Where both run the same float operations in the same order the
bar is bit equality; elsewhere it is stated beside the check.

tests/golden/ref_vectors.npz holds the reference's outputs for these inputs
(written by tests/golden/make_ref_vectors.py from the harness), so the oracle
stays pinned where the reference tree, and with it the harness, is absent.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import small_scene
from multiviewdynrecon_b200 import abi, synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_vectors.npz")


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def ref_or_skip(oracle_mod):
    L = oracle_mod.ref_lib()
    if L is None:
        pytest.skip("reference harness not built (oracle/_ref/libref_pin.so)")
    return L


def inputs(seed=7, n=300):
    """Seeded inputs shared with make_ref_vectors.py."""
    rng = np.random.default_rng(seed)
    nodes = 64
    R = synth.rodrigues_batch(rng.normal(0, 0.4, (nodes, 3)))
    t = rng.normal(0, 0.5, (nodes, 3))
    field = synth.se3_to_dq(R, t)
    knn = rng.integers(0, nodes, (n, 4)).astype(np.uint16)
    w = rng.random((n, 4)).astype(np.float32) + 0.05
    w = (w / w.sum(1, keepdims=True)).astype(np.float32)
    G = rng.normal(size=(n, 6, 6))
    spd = (np.einsum("nij,nkj->nik", G, G) + 0.3 * np.eye(6)).astype(np.float32)
    pts = rng.normal(0, 1.0, (n, 3)).astype(np.float32)
    raw = np.concatenate([rng.normal(0, 0.02, (n // 2, 3)), rng.normal(0, 0.3, (n - n // 2, 3))]).astype(np.float32)
    pts2 = (pts + rng.normal(0, 0.01, (n, 3))).astype(np.float32)
    mats = np.stack([synth.mat34_pack(synth.rodrigues(rng.normal(0, 1.0, 3)), rng.normal(0, 0.5, 3))
                     for _ in range(n)]).astype(np.float32)
    return dict(field=field, knn=knn, w=w, spd=spd, pts=pts, raw=raw, pts2=pts2, mats=mats)


def reference_outputs(L, d):
    """The reference harness's outputs for the inputs d."""
    n = len(d["knn"])
    out = {k: [] for k in ("blend", "dq2m", "m2dq", "gj", "huber", "p2p_j", "p2p_jtr", "sm_j_i", "sm_j_j",
                           "sm_jtr_i", "sm_jtr_j")}
    field = np.ascontiguousarray(d["field"], np.float32)
    for k in range(n):
        m = np.zeros(12, np.float32)
        L.ref_blend_se3(_p(field), _p(np.ascontiguousarray(d["knn"][k])), _p(np.ascontiguousarray(d["w"][k])), _p(m))
        out["blend"].append(m)
        m2 = np.zeros(12, np.float32)
        L.ref_dq_to_mat34(_p(np.ascontiguousarray(field[k % len(field)])), _p(m2))
        out["dq2m"].append(m2)
        q = np.zeros(8, np.float32)
        L.ref_mat34_to_dq(_p(np.ascontiguousarray(d["mats"][k])), _p(q))
        out["m2dq"].append(q)
        inv = np.zeros(36, np.float32)
        L.ref_gauss_jordan6(_p(np.ascontiguousarray(d["spd"][k].T.reshape(-1))), _p(inv))
        out["gj"].append(inv)
        tgt = np.concatenate([d["pts"][k] - d["raw"][k], [1.0]]).astype(np.float32)
        wv = np.concatenate([d["pts"][k], [1.0]]).astype(np.float32)
        out["huber"].append(np.float32(L.ref_huber(float(d["raw"][k, 0]))))
        j = np.zeros(18, np.float32)
        L.ref_p2p_jacobian(_p(tgt), _p(wv), _p(j))
        out["p2p_j"].append(j)
        jr = np.zeros(6, np.float32)
        L.ref_p2p_jt_residual(_p(tgt), _p(wv), _p(jr))
        out["p2p_jtr"].append(jr)
        a, b = d["pts"][k].copy(), d["pts2"][k].copy()
        for is_i, key in ((1, "i"), (0, "j")):
            js = np.zeros(18, np.float32)
            L.ref_smooth_jacobian(_p(a), _p(b), is_i, _p(js))
            out["sm_j_" + key].append(js)
            jsr = np.zeros(6, np.float32)
            L.ref_smooth_jt_residual(_p(a), _p(b), is_i, _p(jsr))
            out["sm_jtr_" + key].append(jsr)
    return {k: np.array(v) for k, v in out.items()}


def oracle_outputs(O, d):
    n = len(d["knn"])
    L = O.lib()
    out = {k: [] for k in ("blend", "dq2m", "m2dq", "gj", "huber", "p2p_j", "p2p_jtr", "sm_j_i", "sm_j_j",
                           "sm_jtr_i", "sm_jtr_j")}
    field = np.ascontiguousarray(d["field"], np.float32)
    for k in range(n):
        m = np.zeros(12, np.float32)
        L.orc_blend_se3(_p(field), _p(np.ascontiguousarray(d["knn"][k])), _p(np.ascontiguousarray(d["w"][k])), _p(m))
        out["blend"].append(m)
        m2 = O.dq_to_mat34(field[k % len(field)])
        out["dq2m"].append(m2)
        out["m2dq"].append(O.mat34_to_dq(d["mats"][k]))
        # the oracle rounds to float first; its output has the reference's
        # layout (column reloc[j] at 6 reloc[j] + i)
        inv = O.gauss_jordan_inverse(d["spd"][k].astype(np.float64))
        out["gj"].append(inv.astype(np.float32).reshape(-1))
        out["huber"].append(np.float32(L.orc_huber(float(d["raw"][k, 0]))))
        rec = np.zeros(8, np.float32)
        tgt = (d["pts"][k] - d["raw"][k]).astype(np.float32)
        # the record's raw residual: warped - target in float, as the kernel
        # (and the reference's Jacobian) forms it
        rec[:3], rec[3], rec[4:7] = d["pts"][k], 1.0, (d["pts"][k] - tgt).astype(np.float32)
        J, r = np.zeros(18), np.zeros(3)
        L.orc_p2p_rows(_p(rec), _p(J), _p(r))
        out["p2p_j"].append(J.astype(np.float32))
        out["p2p_jtr"].append((J.reshape(3, 6) * r[:, None]).sum(0))
        a, b = d["pts"][k], d["pts2"][k]
        s12 = np.zeros(12, np.float32)
        s12[:3], s12[3:6], s12[6], s12[8:11] = a, b, 1.0, (a - b).astype(np.float32)
        for is_i, key in ((1, "i"), (0, "j")):
            J, r = np.zeros(18), np.zeros(3)
            L.orc_smooth_rows(_p(s12), is_i, _p(J), _p(r))
            out["sm_j_" + key].append(J.astype(np.float32))
            out["sm_jtr_" + key].append((J.reshape(3, 6) * r[:, None]).sum(0))
    return {k: np.array(v) for k, v in out.items()}


def _check(ref, orc):
    # bit-equal: the blend and se3 matrix, the DQ <-> mat34 conversions, the
    # Gauss-Jordan inverse with partial pivoting, the Huber weight and the
    # Jacobian rows run the same float operations in the same order
    for key in ("blend", "dq2m", "m2dq", "gj", "huber", "p2p_j", "sm_j_i", "sm_j_j"):
        assert np.array_equal(np.asarray(ref[key], np.float32), np.asarray(orc[key], np.float32)), key
    # Jt r: the reference accumulates w^2 r per channel in float; the oracle
    # forms (w J)(w r) in double
    for key in ("p2p_jtr", "sm_jtr_i", "sm_jtr_j"):
        a, b = np.asarray(ref[key], np.float64), np.asarray(orc[key], np.float64)
        assert np.abs(a - b).max() <= 1e-6 * max(1.0, np.abs(a).max()), key


def test_oracle_matches_reference_header_math(oracle_mod):
    L = ref_or_skip(oracle_mod)
    d = inputs()
    _check(reference_outputs(L, d), oracle_outputs(oracle_mod, d))


def test_oracle_matches_committed_reference_vectors(oracle_mod):
    """The same check against the reference outputs committed as fixtures."""
    g = np.load(GOLDEN)
    d = {k[3:]: g[k] for k in g.files if k.startswith("in_")}
    ref = {k[4:]: g[k] for k in g.files if k.startswith("ref_")}
    _check(ref, oracle_outputs(oracle_mod, d))


def test_committed_vectors_are_the_harness_outputs(oracle_mod):
    L = ref_or_skip(oracle_mod)
    g = np.load(GOLDEN)
    d = {k[3:]: g[k] for k in g.files if k.startswith("in_")}
    ref = reference_outputs(L, d)
    for k, v in ref.items():
        assert np.array_equal(v, g["ref_" + k]), k


@pytest.mark.parametrize("kind", ["torso", "body"])
def test_index_keys_and_term_offsets_match_reference(oracle_mod, kind):
    """Node-pair keys are the reference's encode_nodepair of the pair's nodes;
    the term offsets and every term's (type, typed index) are those of
    size2offset / query_typed_index."""
    L = ref_or_skip(oracle_mod)
    scene = small_scene(kind)
    o = oracle_mod.Oracle(scene, abi.make_config(scene))
    o.build_index()
    keys = o.get(abi.ARRAY_HALF_NODEPAIR_KEY)
    i, j = keys // 4096, keys % 4096
    assert all(L.ref_encode_nodepair(int(a), int(b)) == int(k) for a, b, k in zip(i, j, keys))
    c = o.counts()
    sizes = np.array([c.dense_terms, c.smooth_terms, c.foreground_terms, c.feature_terms, c.cross_terms], np.uint32)
    total = int(sizes.sum())
    offs = np.zeros(5, np.uint32)
    types = np.zeros(total, np.uint32)
    typed = np.zeros(total, np.uint32)
    L.ref_term_offsets(_p(sizes), _p(offs), _p(types), _p(typed))
    assert np.array_equal(offs, np.cumsum(sizes))
    # the term order of the oracle's index: node -> term entries refer to
    # term ids whose types follow the same offsets
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    want_type = np.repeat(np.arange(5), sizes)
    want_typed = np.arange(total) - starts[want_type]
    assert np.array_equal(types, want_type) and np.array_equal(typed, want_typed)
