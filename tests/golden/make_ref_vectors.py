"""Writes tests/golden/ref_vectors.npz: the reference's own outputs for the
seeded inputs of tests/test_ref_pin.py, computed by the reference's header
math compiled into oracle/_ref/libref_pin.so (oracle/Makefile, target `ref`,
which needs the reference tree). The fixture keeps the oracle pinned to the
reference where that tree is absent. Regenerate with

    make -C oracle ref && python tests/golden/make_ref_vectors.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)


def main():
    import oracle
    from test_ref_pin import inputs, reference_outputs
    L = oracle.ref_lib()
    if L is None:
        raise SystemExit("build the harness first: make -C oracle ref")
    d = inputs()
    ref = reference_outputs(L, d)
    out = {f"in_{k}": v for k, v in d.items()}
    out.update({f"ref_{k}": v for k, v in ref.items()})
    np.savez_compressed(os.path.join(HERE, "ref_vectors.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
