"""Generate the committed golden I(q) vectors from the C oracle.

    python tests/golden/make_golden.py

Inputs are regenerated from the seeded generators in thistle_b200.inputs;
outputs are the oracle's restatement of the reference integrators
(bessel_mode 0: the reference's own 100-term dphrec start) for types 1, 2,
7 and 8, the resolved CMS (type 9) on the seeded 1-RDM pair of
``inputs.cms_onerdms``, and the elastic aligned intensity of type 4 on the
CASE(4) grid.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from thistle_b200 import inputs as I  # noqa: E402


def main():
    for cfg in (1, 2):
        p = I.CONFIGS[cfg]()
        out = {"q": p.q}
        for t in (1, 2, 7, 8):
            out[f"type{t}"] = O.scattering(p, t, nthreads=8)
        d1, d2 = I.cms_onerdms(p)
        pc = I.Problem(**{**p.__dict__, "onerdm": d1})
        out["type9"] = O.scattering(pc, 9, onerdm2=d2, nthreads=8)
        # type 4 on the reference's CASE(4) grid of nq vectors: |F(q)|^2
        out["type4"] = O.elastic_aligned(p, nq=p.nq)[2]
        np.savez(os.path.join(HERE, f"golden_cfg{cfg}.npz"), **out)
        print(cfg, {k: v[:2] for k, v in out.items()})


if __name__ == "__main__":
    main()
