"""Generate the committed full-size golden fixtures from the C oracle.

    python tests/golden/make_golden_large.py [section ...]

Sections (default: all): ab6, ab6_sample, cfg5, cfg5_adjoint, cfg5_aligned,
cfg4, refrdm, co.  Inputs are regenerated from the seeded generators in
thistle_b200.inputs (the tests regenerate the same inputs); only the
oracle's outputs, the sample selections and small derived inputs are stored.

The oracle evaluates every group quartet of the reference's five loops with
the reference's kernels; the contraction of the 2-RDM rows is read from the
summed pair density (``oracle.pair_density``, checked against the
reference-order contraction by tests/test_oracle_fast_modes.py).  Bessel
functions: bessel_mode 1 (accurate start of dphrec) for the full grids,
plus bessel_mode 0 (the reference's own 100-term start) where stated.

The refrdm section reads the reference's own 2-RDM files
(src/HF_NonZero2RM_MO_Coeffs, src/NonZero2RDM_MO_Coeffs, src/twordm.dat) and
the co section its CO molden file (src/UCCSD_CO_4Bohr_Molden_631star.txt,
through thistle_b200.molden) from a reference checkout (THISTLE_REFERENCE,
default /root/reference), and store the parsed arrays, so that the GPU tests
need no checkout.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from thistle_b200 import inputs as I  # noqa: E402

NT = os.cpu_count() or 8
REF = os.environ.get("THISTLE_REFERENCE", "/root/reference")


def _save(name, **arrs):
    np.savez_compressed(os.path.join(HERE, name), **arrs)
    print(f"wrote {name}: " + ", ".join(f"{k}{np.shape(v)}" for k, v in arrs.items()), flush=True)


def shell_L(p):
    """Angular momentum of each group (shell), 0-based group order."""
    heads = np.searchsorted(p.group, np.arange(1, p.ng + 1))
    return (p.l + p.m + p.n)[heads]


def strata(p, qs):
    """Stratum of every quartet of a five-loop list: the shell types
    (Li, Lj, Lk, Lr), which fix LLmax and the (LK, side) sub-range of the
    GPU's stage 1 (LK = the smaller of the bra's and the ket's angular
    momentum, side = whether the bra's is the smaller)."""
    gl = shell_L(p).astype(np.int64)
    return ((gl[qs[:, 0]] * 5 + gl[qs[:, 1]]) * 5 + gl[qs[:, 2]]) * 5 + gl[qs[:, 3]]


def stratified_sample(p, qs, frac, minimum, seed):
    """Indices (sorted) of a sample with ``frac`` of every stratum, at least
    ``minimum`` quartets (or the whole stratum)."""
    st = strata(p, qs)
    rng = np.random.default_rng(seed)
    pick = []
    for s in np.unique(st):
        idx = np.flatnonzero(st == s)
        k = min(idx.size, max(minimum, int(np.ceil(frac * idx.size))))
        pick.append(rng.choice(idx, size=k, replace=False))
    return np.sort(np.concatenate(pick)).astype(np.int64)


def hmax_of(p):
    a = np.asarray(p.atoms)
    return float(np.max(np.linalg.norm(a[:, None, :] - a[None, :, :], axis=-1)))


def sec_ab6():
    p = I.config3_ab6()
    t = time.time()
    rho = O.pair_density(p)
    out = {"q": p.q}
    for ty in (1, 7):
        out[f"type{ty}"] = O.scattering(p, ty, rho=rho, bessel_mode=1, nthreads=NT)
        print(f"ab6 type {ty}: {time.time() - t:.0f} s", flush=True)
    out["type2"] = O.scattering(p, 2, bessel_mode=1, nthreads=NT)
    # the reference's own Bessel start, on the points where it has converged
    ok = p.q * hmax_of(p) <= 70.0
    out["ref_mask"] = ok
    out["type1_ref"] = O.scattering(p, 1, rho=rho, bessel_mode=0, nthreads=NT, q=p.q[ok])
    print(f"ab6 done: {time.time() - t:.0f} s", flush=True)
    _save("golden_ab6.npz", **out)


def sec_ab6_sample():
    p = I.config3_ab6()
    qs = O.enum_quartets(p.ng)
    idx = stratified_sample(p, qs, 0.01, 40, 20261204)
    rho = O.pair_density(p)
    sub = qs[idx]
    out = {"q": p.q, "index": idx.astype(np.int32)}
    for ty in (1, 7):
        out[f"type{ty}"] = O.scattering(p, ty, quartets=sub, rho=rho, bessel_mode=1, nthreads=NT)
    out["type2"] = O.scattering(p, 2, quartets=sub, bessel_mode=1, nthreads=NT)
    _save("golden_ab6_sample.npz", **out)


def sec_cfg5():
    p = I.config5_fit()
    rho = O.pair_density(p)
    out = {"q": p.q}
    for ty in (1, 7):
        out[f"type{ty}"] = O.scattering(p, ty, rho=rho, bessel_mode=1, nthreads=NT)
    out["type2"] = O.scattering(p, 2, bessel_mode=1, nthreads=NT)
    ok = p.q * hmax_of(p) <= 70.0
    out["ref_mask"] = ok
    out["type1_ref"] = O.scattering(p, 1, rho=rho, bessel_mode=0, nthreads=NT, q=p.q[ok])
    _save("golden_cfg5.npz", **out)


# coordinates (atom, axis) differentiated per displaced geometry
ADJ_COORDS = np.array([[0, 0], [1, 1], [2, 2], [3, 0], [4, 2], [5, 1]], dtype=np.int32)
ADJ_H = 1.0e-4


def sec_cfg5_adjoint():
    """sum_q v(q) dI(q)/dR by central differences of the oracle (h = 1e-4
    bohr) at six nuclear coordinates of two displaced ring geometries."""
    base = I.config5_fit()
    geoms = I.config5_geometries(base, 3)[1:]
    rho = O.pair_density(base)  # the density does not depend on the geometry
    v = np.random.default_rng(20261205).standard_normal((2, base.nq))
    fd = np.zeros((2, len(ADJ_COORDS)))
    t = time.time()
    for g in range(2):
        for c, (a, ax) in enumerate(ADJ_COORDS):
            val = []
            for sgn in (1.0, -1.0):
                R = geoms[g].copy()
                R[a, ax] += sgn * ADJ_H
                val.append(O.scattering(base.with_geometry(R), 1, rho=rho, bessel_mode=1, nthreads=NT))
            fd[g, c] = np.dot(v[g], val[0] - val[1]) / (2.0 * ADJ_H)
            print(f"adjoint fd geometry {g} coordinate {c}: {time.time() - t:.0f} s", flush=True)
    _save("golden_cfg5_adjoint.npz", geoms=geoms, v=v, coords=ADJ_COORDS, h=np.array(ADJ_H), fd=fd)


ALIGNED_STRIDE = 131  # 64^3 / 131 -> 2002 vectors


def sec_cfg5_aligned():
    p = I.config5_fit()
    grid = I.config5_aligned_grid()
    idx = np.arange(0, grid.shape[0], ALIGNED_STRIDE)
    rho = O.pair_density(p)
    t = time.time()
    re = O.aligned_list(p, grid[idx], rho=rho, nthreads=NT)
    print(f"aligned slice: {time.time() - t:.0f} s", flush=True)
    _save("golden_cfg5_aligned.npz", stride=np.array(ALIGNED_STRIDE), index=idx.astype(np.int32), re=re)


CFG4_MOLECULES = 8  # the first molecules of the seeded 1024-molecule batch; #4 has 12 atoms


def sec_cfg4():
    mols = I.config4_batch(CFG4_MOLECULES)
    out = {"q": mols[0].q, "natoms": np.array([len(p.atoms) for p in mols])}
    t = time.time()
    for ty in (1, 2, 7):
        rows = []
        for p in mols:
            rho = O.pair_density(p) if ty != 2 else None
            rows.append(O.scattering(p, ty, rho=rho, bessel_mode=1, nthreads=NT))
        out[f"type{ty}"] = np.stack(rows)
        print(f"cfg4 type {ty}: {time.time() - t:.0f} s", flush=True)
    _save("golden_cfg4.npz", **out)


# the reference's 2-RDM files and the basis each is evaluated on
REF_RDMS = [
    # (key, file, reader, nelec, basis: 'h2' (configuration 1) or 'diatomic' (configuration 2))
    ("hf", "src/HF_NonZero2RM_MO_Coeffs", "rows", 14, "diatomic"),
    ("ci", "src/NonZero2RDM_MO_Coeffs", "rows", 10, "diatomic"),
    ("h2", "src/twordm.dat", "listing", 2, "h2"),
]


def refrdm_problem(key, mat, total, nelec, basis):
    """A seeded problem carrying one of the reference's 2-RDMs: the basis and
    grid of configuration 1 or 2, as many Loewdin-orthonormal MOs as the
    2-RDM's largest index."""
    base = I.config1_h2() if basis == "h2" else I.config2_diatomic()
    nmo = int(np.max(mat))
    rng = np.random.default_rng(I.SEED0 + 100 + nmo)
    C = I.lowdin_mos(rng, nmo, base.ga, base.l, base.m, base.n, base.xx, base.yy, base.zz)
    p = base.with_geometry(base.atoms)
    p.mmod = C
    p.mat = np.asarray(mat, dtype=np.int32)
    p.total = np.asarray(total, dtype=np.float64)
    p.nelec = nelec
    p.name = f"ref_{key}"
    return p


def sec_refrdm():
    from thistle_b200 import main_calculation as MC
    out = {}
    for key, rel, reader, nelec, basis in REF_RDMS:
        path = os.path.join(REF, rel)
        mat, total = (MC.read_twordm if reader == "rows" else MC.read_twordm_listing)(path)
        p = refrdm_problem(key, mat, total, nelec, basis)
        out[f"{key}_mat"] = mat
        out[f"{key}_total"] = total
        for ty in (1, 7):
            out[f"{key}_type{ty}"] = O.scattering(p, ty, bessel_mode=1, nthreads=NT)
    _save("golden_refrdm.npz", **out)


CO_MOLDEN = "src/UCCSD_CO_4Bohr_Molden_631star.txt"


def co_problem(g, rdm):
    """The CO basis of the reference's molden fixture (parsed arrays in g)
    carrying the reference's HF 2-RDM file and its 1-RDM, 60 q on 0..8
    (q[0] = 1e-10)."""
    q = np.linspace(0.0, 8.0, 60)
    q[0] = 1e-10
    atoms = np.array(g["atoms"]).reshape(-1, 3)
    mat, total = rdm["hf_mat"], rdm["hf_total"]
    p = I.Problem(name="co", atoms=atoms, ga=g["ga"], l=g["l"], m=g["m"], n=g["n"], xx=g["x"], yy=g["y"],
                  zz=g["z"], group=g["group"], atom_of=g["atom_of"], mmod=g["mmod"], mat=mat, total=total,
                  onerdm=np.zeros((1, 1)), q=q, nelec=14)
    nmo = int(mat.max())
    G = np.zeros((nmo,) * 4)
    G[tuple((mat - 1).T)] = total
    p.onerdm = I.onerdm_from_2rdm(G, 14)
    return p


def sec_co():
    """The reference's CO molden file through the molden reader (decontracted,
    the reference's unit handling), with the HF 2-RDM file."""
    from thistle_b200 import molden
    gt, at = molden.read_orbitals(os.path.join(REF, CO_MOLDEN), N=100, decontract=True)
    atom_of = np.array([int(np.argmin(np.sum((at.xyz - np.array([x, y, z])) ** 2, axis=1)))
                        for x, y, z in zip(gt.x, gt.y, gt.z)], dtype=np.int32)
    g = dict(ga=gt.ga, l=gt.l, m=gt.m, n=gt.n, x=gt.x, y=gt.y, z=gt.z, group=gt.group, mmod=gt.mo.T.copy(),
             atoms=at.xyz, numbers=at.numbers, atom_of=atom_of)
    p = co_problem(g, np.load(os.path.join(HERE, "golden_refrdm.npz")))
    for ty in (1, 2, 7):
        g[f"type{ty}"] = O.scattering(p, ty, bessel_mode=1, nthreads=NT)
    g["q"] = p.q
    _save("golden_co.npz", **g)


SECTIONS = {"co": sec_co, "ab6": sec_ab6, "ab6_sample": sec_ab6_sample, "cfg5": sec_cfg5, "cfg5_adjoint": sec_cfg5_adjoint,
            "cfg5_aligned": sec_cfg5_aligned, "cfg4": sec_cfg4, "refrdm": sec_refrdm}


def main(argv):
    for name in (argv or list(SECTIONS)):
        t = time.time()
        SECTIONS[name]()
        print(f"section {name}: {time.time() - t:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
