"""Writes the golden fixtures tests/golden/*.npz from the CPU oracle.

The reference ships no golden vectors and cannot run here, so these fixtures
are a regression pin of the oracle itself: index arrays (exact), the first
iteration's diagonal blocks and Jt r, the warp field after one Gauss-Newton
iteration and the energy. Regenerate with

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from multiviewdynrecon_b200 import abi, synth  # noqa: E402

SCENES = {
    "sphere_small": lambda: synth.sphere_single_view(seed=101, num_nodes=96, width=64, height=48),
    "torso_small": lambda: synth.torso_multi_view(seed=102, num_nodes=128, num_views=3, width=64, height=48,
                                                  features_per_view=20, cross_per_pair=20),
}

INDEX_ARRAYS = ["ARRAY_DENSE_PIXELS", "ARRAY_NODE2TERM_OFFSET", "ARRAY_NODE2TERM_INDEX", "ARRAY_HALF_NODEPAIR_KEY",
                "ARRAY_NODEPAIR_TERM_INDEX", "ARRAY_NODEPAIR_KEY", "ARRAY_NODEPAIR_TERM_RANGE",
                "ARRAY_BLKROW_OFFSET", "ARRAY_BINBLOCK_ROWPTR", "ARRAY_BINBLOCK_COLPTR"]


def main():
    import oracle
    for name, make in SCENES.items():
        scene = make()
        cfg = abi.make_config(scene)
        o = oracle.Oracle(scene, cfg)
        o.build_index()
        out = {k: o.get(getattr(abi, k)) for k in INDEX_ARRAYS}
        o.eval_terms()
        o.assemble()
        out["ARRAY_DIAG_BLOCKS"] = o.get(abi.ARRAY_DIAG_BLOCKS)
        out["ARRAY_JTR"] = o.get(abi.ARRAY_JTR)
        out["energy"] = np.array(o.energy())
        o.pcg(scene.pcg_iterations)
        o.update()
        out["ARRAY_NODE_SE3"] = o.get(abi.ARRAY_NODE_SE3)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
