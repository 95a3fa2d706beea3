"""Central finite differences of the FP64 oracle's weighted residual vector,
for checking the adjoint products J^T r and J^T J p (the configuration that
compares them on 64 random nodes with a step of ~1e-4 per twist coordinate).

The residual vector stacks every scalar term with its weight lambda (and, for
the feature and cross-view terms, its Huber weight frozen at the base point,
as the Gauss-Newton step treats it). With the projected pixels and validity
frozen too, it is a smooth function of the warp field, so
    J e_k  ~  (R(x + h e_k) - R(x - h e_k)) / 2h
where x + h e_k applies the twist h e_k to one node (T <- exp(h e_k) T).
"""
import numpy as np

from multiviewdynrecon_b200 import abi

# global-iteration penalties (PenaltyConstants.cpp:25-37) used by make_config's
# elastic schedule
GLOBAL_LAMBDA = dict(smooth=5.0, foreground=2e-3, feature=1.0, cross=1.0)
DAMPING = 1e-2  # added to the diagonal of every diagonal block
# the twist update leaves the rotation unchanged when sum |omega| < 1e-4
# (SolverIterationData.cu:9-57), so the rotational step must be larger
STEP = 2e-4


def huber_weight(r):
    a = np.abs(r).astype(np.float32)
    return np.where(a < np.float32(7.5e-2), np.float32(1.0), np.float32(7.5e-2) / np.maximum(a, np.float32(1e-30)))


def weighted_residuals(o, cfg, hw0=None):
    """The lambda-weighted scalar residuals of the oracle's current
    evaluation, and the Huber weights used for the point-to-point terms."""
    c = o.counts()
    td, tf, tp, tc = c.dense_terms, c.foreground_terms, c.feature_terms, c.cross_terms
    jr = o.get(abi.ARRAY_TERM_JACOBIAN).reshape(-1, 8)[:td + tf]
    valid = jr[:, 7].view(np.uint32) != 0xFFFFFFFF
    r_pix = np.where(valid, jr[:, 6].astype(np.float64), 0.0)
    r_pix[td:] *= GLOBAL_LAMBDA["foreground"] if cfg.use_foreground else 0.0
    sm = o.get(abi.ARRAY_SMOOTH_TERMS).reshape(-1, 12)
    r_sm = np.where(sm[:, 6:7] != 0, sm[:, 8:11].astype(np.float64), 0.0) * GLOBAL_LAMBDA["smooth"]
    wv = o.get(abi.ARRAY_WARPED_CORRESPONDENCE).reshape(-1, 8)[:tp + tc]
    raw = wv[:, 4:7].astype(np.float64)
    if hw0 is None:
        hw0 = huber_weight(raw).astype(np.float64)
    lam = np.r_[np.full(tp, GLOBAL_LAMBDA["feature"] if cfg.use_feature else 0.0),
                np.full(tc, GLOBAL_LAMBDA["cross"] if cfg.use_cross_view else 0.0)][:, None]
    return np.concatenate([r_pix, r_sm.ravel(), (raw * hw0 * lam).ravel()]), hw0


def fd_columns(oracle_mod, o, cfg, base_dq, coords, hw0, h=STEP):
    """J e_k for each (node, twist coordinate) in `coords`, as rows."""
    cols = []
    for n, c in coords:
        res = []
        for sgn in (1.0, -1.0):
            dq = base_dq.copy()
            tw = np.zeros(6)
            tw[c] = sgn * h
            dq[n] = oracle_mod.apply_twist(base_dq[n], tw)
            o.set_node_se3(dq)
            o.eval_terms()
            res.append(weighted_residuals(o, cfg, hw0)[0])
        cols.append((res[0] - res[1]) / (2.0 * h))
    o.set_node_se3(base_dq)
    o.eval_terms()
    return np.array(cols)


def fd_config(scene, **kw):
    """The scene's configuration without the foreground term: its residual
    samples a mask at a (frozen) pixel, so a finite difference sees no
    change, while its Jacobian is the reference's image-gradient model
    (DensityForegroundJacobianResidual.cu:41-142), not a derivative of the
    sampled value. Every other term is a smooth function of the warp field."""
    cfg = abi.make_config(scene, **kw)
    cfg.use_foreground = 0
    return cfg


def uniform_field(scene, seed=0, rot_deg=1.0, trans=0.005):
    """A copy of `scene` whose nodes all carry the same rigid transform. The
    Jacobian of a skinned term with respect to node i's twist is modelled as
    w_i times the twist Jacobian of the blended transform; that is exact when
    the term's nodes share one transform and first-order accurate otherwise
    (a few 1e-4 relative on the per-node perturbed fields of the synthetic
    scenes). On this copy finite differences can check it to rounding."""
    import copy
    from multiviewdynrecon_b200 import synth
    rng = np.random.default_rng(seed)
    R = synth.rodrigues(rng.normal(0, np.radians(rot_deg), 3))
    t = rng.normal(0, trans, 3)
    n = scene.num_nodes
    s = copy.copy(scene)
    s.node_se3 = synth.se3_to_dq(np.repeat(R[None], n, 0), np.repeat(t[None], n, 0))
    return s


def random_coords(rng, num_nodes, count=64):
    nodes = rng.choice(num_nodes, count, replace=False)
    return [(int(n), int(rng.integers(6))) for n in nodes]


def fd_adjoint_reference(oracle_mod, scene, cfg, coords, p_coeffs, term_jr=None, smooth=None):
    """Finite-difference J^T r (negated, i.e. the right-hand side b) at the
    coordinates, and (J^T J p) restricted to them for p = sum_k p_k e_k,
    from the FP64 oracle at the scene's warp field. Pixel and validity
    decisions are frozen from (term_jr, smooth), by default the oracle's own
    at the base point."""
    o = oracle_mod.Oracle(scene, cfg, fp64=True)
    o.build_index()
    base_dq = scene.node_se3.astype(np.float64)
    o.set_node_se3(base_dq)
    if term_jr is None:
        o.eval_terms()
        term_jr, smooth = o.get(abi.ARRAY_TERM_JACOBIAN), o.get(abi.ARRAY_SMOOTH_TERMS)
    o.freeze(term_jr, smooth)
    o.eval_terms()
    r0, hw0 = weighted_residuals(o, cfg)
    cols = fd_columns(oracle_mod, o, cfg, base_dq, coords, hw0)
    b_fd = -cols @ r0
    jp = p_coeffs @ cols
    jtjp_fd = cols @ jp
    return b_fd, jtjp_fd, o
