"""Algorithmic FLOPs of stage 1 (the q-independent Hermite part of every
quartet) for the AB6 bench workload, counted by the oracle.

    python -m oracle.stage1_flops

Per quartet, tot_integral_k_ijkr (src/Integrals.f90:5155-5219) updates the
Bessel-order coefficients h_saved once for every six-deep Hermite product
that passes both cutoffs; with T_E such updates and LLmax = L, its work is
F_E = 2 (L + 1) T_E FLOP (one multiply-add per order 0..L).  Quartets on the
P = Q branch (loop 5, |H| < cutoffcentre) sum their tot_integral_ijkr_pzero
terms into q-polynomial coefficients instead: 2 T_E.  The counts depend only
on the inputs and the cutoffs, so they are computed once and written to
profiles/stage1_ab6_flops.json, which bench.py reads for its stage-1
roofline.  Test infrastructure: the product never runs this.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


def main():
    from oracle import oracle as O
    from thistle_b200 import inputs as I
    t0 = time.time()
    p = I.config3_ab6()
    rho = O.pair_density(p)
    qs = O.enum_quartets(p.ng)
    te, p0 = O.count_te(p, qs, rho=rho, nthreads=os.cpu_count() or 1)
    heads = np.searchsorted(p.group, np.arange(1, p.ng + 1))
    gl = (p.l + p.m + p.n)[heads]
    L = gl[qs[:, 0]] + gl[qs[:, 1]] + gl[qs[:, 2]] + gl[qs[:, 3]]
    fe = np.where(p0, 2 * te, 2 * (L + 1) * te)
    per_class = {}
    for LL in np.unique(L):
        sel = L == LL
        per_class[int(LL)] = {"quartets": int(sel.sum()), "p0_quartets": int(p0[sel].sum()),
                              "T_E": int(te[sel].sum()), "flops": int(fe[sel].sum())}
    out = {
        "workload": f"ab6_total_j0: {len(p.atoms)} atoms, {p.ngto} primitives ({p.ng} shells), {p.nmo} MOs, "
                    f"{p.mat.shape[0]}-row 2-RDM, cutoffz {p.cutoffz}, cutoffmd {p.cutoffmd}, "
                    f"cutoffcentre {p.cutoffcentre}",
        "formula": "F_E = 2 (LLmax + 1) T_E per Bessel-branch quartet, 2 T_E per P = Q quartet; T_E = Hermite "
                   "products passing |ztot| >= cutoffz and |prod6| > cutoffmd",
        "quartets": int(qs.shape[0]),
        "T_E": int(te.sum()),
        "flops_per_step": int(fe.sum()),
        "per_llmax": per_class,
        "command": "python -m oracle.stage1_flops",
        "seconds": round(time.time() - t0, 1),
    }
    path = os.path.join(ROOT, "profiles", "stage1_ab6_flops.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path, out["flops_per_step"], out["T_E"])


if __name__ == "__main__":
    main()
