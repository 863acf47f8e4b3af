"""ctypes wrapper of the C oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle_thistle.so`` (built from ``thistle_oracle.c`` by
``oracle/build.py``).  Only tests, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline and reference legs import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle_thistle.so")
        if not os.path.exists(path):
            from . import build as _b  # type: ignore
            _b.build()
        _LIB = C.CDLL(path)
        _LIB.orc_count_quartets.restype = C.c_long
        _LIB.orc_enum_quartets.restype = C.c_long
    return _LIB


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int))


def count_quartets(ng: int) -> int:
    return int(lib().orc_count_quartets(C.c_int(ng)))


def enum_quartets(ng: int) -> np.ndarray:
    n = count_quartets(ng)
    out = np.zeros((n, 5), dtype=np.int32)
    lib().orc_enum_quartets(C.c_int(ng), out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def pair_density(prob) -> np.ndarray:
    """The per-quartet contraction ztot of the 2-RDM rows, for every pair of
    function pairs at once: rho[P(x,y), P(u,v)] = 1/8 sum_t [z11(t,x,y)
    z22(t,u,v) + z22(t,x,y) z11(t,u,v)] with z11, z22 of variables_total
    (src/Variables.f90:1045-1065) and P(x,y) = max(x,y)(max+1)/2 + min(x,y).

    The rows enter through their eight index placements summed into a dense
    MO-space array G[a,b,c,d] (each row adds total/8 at (m1,m2,m3,m4),
    (m2,m1,m3,m4), (m1,m2,m4,m3), (m2,m1,m4,m3) and the four with the pairs
    exchanged), then four contractions with the MO coefficients.  This is the
    same quantity as the reference's per-quartet dgemm pair
    (src/Integrals.f90:109-127) in another summation order; tests compare the
    two modes of the oracle on configurations 1-3.  Returns (np, np)."""
    n, ngto = prob.mmod.shape
    C = np.asarray(prob.mmod, dtype=np.float64)
    m = np.asarray(prob.mat, dtype=np.int64) - 1
    v = np.asarray(prob.total, dtype=np.float64) / 8.0
    m1, m2, m3, m4 = m[:, 0], m[:, 1], m[:, 2], m[:, 3]
    G = np.zeros((n, n, n, n))
    for (a, b, c, d) in ((m1, m2, m3, m4), (m2, m1, m3, m4), (m1, m2, m4, m3), (m2, m1, m4, m3),
                         (m3, m4, m1, m2), (m4, m3, m1, m2), (m3, m4, m2, m1), (m4, m3, m2, m1)):
        np.add.at(G, (a, b, c, d), v)
    # x: first function of the bra pair, y second, u, v the ket pair
    T = np.tensordot(C, G, axes=([0], [0]))            # (x, b, c, d)
    T = np.tensordot(T, C, axes=([1], [0]))            # (x, c, d, y)
    T = np.ascontiguousarray(T.transpose(0, 3, 1, 2))  # (x, y, c, d)
    r, c_ = np.tril_indices(ngto)
    V = T[r, c_]                                       # (np, c, d), P(x,y) with x >= y
    del T
    npair = r.size
    out = np.empty((npair, npair))
    blk = max(1, int(2.0e8 // max(1, ngto * ngto)))
    for s0 in range(0, npair, blk):
        W = np.tensordot(V[s0:s0 + blk], C, axes=([1], [0]))   # (blk, d, u)
        W = np.tensordot(W, C, axes=([1], [0]))                # (blk, u, v)
        out[s0:s0 + blk] = W[:, r, c_]
    return out


def scattering(prob, type_: int = 1, *, bessel_mode: int = 0, nthreads: int = 0,
               quartets=None, weights=None, q=None, rho=None, onerdm2=None) -> np.ndarray:
    """Reference restatement of total_scattering_calculation_2 (types 1, 2,
    7, 8 and 9).

    rho: optional ``pair_density(prob)`` for types 1 and 7; the per-quartet
    contraction of the 2-RDM rows is then read from it (the rest of the
    evaluation is unchanged).  onerdm2: type 9 (resolved CMS) only, the ket's
    1-RDM (zj); the bra's (zi) is ``prob.onerdm``."""
    keep = []

    def d(x):
        a, p = _d(x)
        keep.append(a)
        return p

    def i(x):
        a, p = _i(x)
        keep.append(a)
        return p

    qv = prob.q if q is None else np.asarray(q, dtype=np.float64)
    nq = qv.size
    out = np.zeros(nq)
    mat_cm = np.asfortranarray(prob.mat.astype(np.int32)).ravel(order="F")
    mmod_cm = np.asfortranarray(prob.mmod).ravel(order="F")
    one_cm = np.asfortranarray(prob.onerdm).ravel(order="F")
    if type_ == 9:
        if onerdm2 is None or np.shape(onerdm2) != prob.onerdm.shape:
            raise ValueError("type 9 needs onerdm2 with the shape of prob.onerdm")
        one_cm = np.concatenate([one_cm, np.asfortranarray(onerdm2, dtype=np.float64).ravel(order="F")])
    if quartets is not None:
        qt = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 5)
        qptr, nqt = i(qt), qt.shape[0]
    else:
        qptr, nqt = None, 0
    wptr = d(weights) if weights is not None else None
    rptr = None
    if rho is not None and type_ != 2:
        npair = prob.ngto * (prob.ngto + 1) // 2
        if rho.shape != (npair, npair):
            raise ValueError("rho must be pair_density(prob)")
        rptr = d(rho)
    rc = lib().orc_scattering_ex(
        C.c_int(type_), C.c_int(prob.ngto), d(prob.ga), i(prob.l), i(prob.m), i(prob.n),
        d(prob.xx), d(prob.yy), d(prob.zz), i(prob.group), d(mmod_cm), C.c_int(prob.nmo),
        i(mat_cm), d(prob.total), C.c_int(prob.mat.shape[0]), d(one_cm), C.c_int(prob.onerdm.shape[0]),
        d(qv), C.c_int(nq), C.c_double(prob.cutoffz), C.c_double(prob.cutoffmd),
        C.c_double(prob.cutoffcentre), C.c_int(bessel_mode), C.c_int(nthreads),
        qptr, C.c_long(nqt), wptr, rptr, out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle orc_scattering failed with code {rc}")
    return out


def aligned(prob, qal: np.ndarray, *, nthreads: int = 0):
    keep = []

    def d(x):
        a, p = _d(x)
        keep.append(a)
        return p

    def i(x):
        a, p = _i(x)
        keep.append(a)
        return p

    qal = np.ascontiguousarray(qal, dtype=np.float64).reshape(-1, 3)
    nq = qal.shape[0]
    re, im = np.zeros(nq), np.zeros(nq)
    mat_cm = np.asfortranarray(prob.mat.astype(np.int32)).ravel(order="F")
    mmod_cm = np.asfortranarray(prob.mmod).ravel(order="F")
    rc = lib().orc_aligned(
        C.c_int(prob.ngto), d(prob.ga), i(prob.l), i(prob.m), i(prob.n), d(prob.xx), d(prob.yy),
        d(prob.zz), i(prob.group), d(mmod_cm), C.c_int(prob.nmo), i(mat_cm), d(prob.total),
        C.c_int(prob.mat.shape[0]), d(qal), C.c_int(nq), C.c_double(prob.cutoffz),
        C.c_double(prob.cutoffmd), C.c_int(nthreads), re.ctypes.data_as(C.POINTER(C.c_double)),
        im.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle orc_aligned failed with code {rc}")
    return re, im


def aligned_list(prob, qal: np.ndarray, *, quartets=None, rho=None, nthreads: int = 0) -> np.ndarray:
    """Real part of the aligned intensity as the weighted sum over the five
    loops' quartet list (default: all of them) instead of all ng^4 ordered
    quartets; see orc_aligned_list.  rho as in ``scattering``."""
    keep = []

    def d(x):
        a, p = _d(x)
        keep.append(a)
        return p

    def i(x):
        a, p = _i(x)
        keep.append(a)
        return p

    qal = np.ascontiguousarray(qal, dtype=np.float64).reshape(-1, 3)
    nq = qal.shape[0]
    qs = enum_quartets(prob.ng) if quartets is None else np.ascontiguousarray(quartets, dtype=np.int32)
    re = np.zeros(nq)
    mat_cm = np.asfortranarray(prob.mat.astype(np.int32)).ravel(order="F")
    mmod_cm = np.asfortranarray(prob.mmod).ravel(order="F")
    rc = lib().orc_aligned_list(
        C.c_int(prob.ngto), d(prob.ga), i(prob.l), i(prob.m), i(prob.n), d(prob.xx), d(prob.yy),
        d(prob.zz), i(prob.group), d(mmod_cm), C.c_int(prob.nmo), i(mat_cm), d(prob.total),
        C.c_int(prob.mat.shape[0]), d(rho) if rho is not None else None, d(qal), C.c_int(nq), i(qs),
        C.c_long(qs.shape[0]), C.c_double(prob.cutoffz), C.c_double(prob.cutoffmd), C.c_int(nthreads),
        re.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle orc_aligned_list failed with code {rc}")
    return re


def qcoord3(k0: float = 10.583544175):
    qx, qy, qz = np.zeros(3131), np.zeros(3131), np.zeros(3131)
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    lib().orc_qcoord3(C.c_double(k0), p(qx), p(qy), p(qz))
    return np.stack([qx, qy, qz], axis=1)


def kernel_quartet(kind, pzero, mu, l, m, n, group_start, group_count, hx, hy, hz, h,
                   dx1, dy1, dz1, dx2, dy2, dz2, gi, gj, gk, gr, zcontr, zcontr2,
                   cutoff1=1e-14, cutoff2=1e-14, bessel_mode=0):
    """One per-quartet kernel with Fortran argument meaning and layouts."""
    keep = []

    def d(x):
        a = np.asfortranarray(np.asarray(x, dtype=np.float64)).ravel(order="F")
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_double))

    def i(x):
        a = np.ascontiguousarray(np.asarray(x, dtype=np.int32).ravel())
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_int))

    mu = np.asarray(mu, dtype=np.float64)
    dx1 = np.asarray(dx1, dtype=np.float64)
    dt, dl = dx1.shape[0], dx1.shape[1]
    f = np.zeros(mu.size)
    rc = lib().orc_kernel_quartet(
        C.c_int(kind), C.c_int(pzero), d(mu), C.c_int(mu.size), C.c_int(len(l)), i(l), i(m), i(n),
        C.c_int(len(group_start)), i(group_start), i(group_count), C.c_double(hx), C.c_double(hy),
        C.c_double(hz), C.c_double(h), d(dx1), d(dy1), d(dz1), d(dx2), d(dy2), d(dz2), C.c_int(dt),
        C.c_int(dl), C.c_int(gi), C.c_int(gj), C.c_int(gk), C.c_int(gr), d(zcontr), d(zcontr2),
        C.c_double(cutoff1), C.c_double(cutoff2), C.c_int(bessel_mode),
        f.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle kernel failed with code {rc}")
    return f


def dphrec(x, lmax1: int, leps1: int = 100) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros((x.size, lmax1))
    lib().orc_dphrec(x.ctypes.data_as(C.POINTER(C.c_double)), C.c_int(x.size), C.c_int(leps1),
                     C.c_int(lmax1), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def md_chain(l1, l2, PA, PB, a) -> np.ndarray:
    out = np.zeros(l1 + l2 + 1)
    lib().orc_md_chain(C.c_int(l1), C.c_int(l2), C.c_double(PA), C.c_double(PB), C.c_double(a),
                       out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def nuclear(prob, Zn, *, bessel_mode: int = 1, q=None) -> np.ndarray:
    """Nuclear-electron term Ine(q) of electron scattering (nuclei_electron_integration)
    with the AO density of the problem's 1-RDM; atoms at prob.atoms with charges Zn."""
    keep = []

    def d(x):
        a, p = _d(x)
        keep.append(a)
        return p

    def i(x):
        a, p = _i(x)
        keep.append(a)
        return p

    qv = prob.q if q is None else np.asarray(q, dtype=np.float64)
    out = np.zeros(qv.size)
    geom = np.asfortranarray(np.asarray(prob.atoms, dtype=np.float64)).ravel(order="F")
    rc = lib().orc_nuclear(
        C.c_int(prob.ngto), d(prob.ga), i(prob.l), i(prob.m), i(prob.n), d(prob.xx), d(prob.yy), d(prob.zz),
        i(prob.group), d(np.asfortranarray(prob.mmod).ravel(order="F")), C.c_int(prob.nmo),
        d(np.asfortranarray(prob.onerdm).ravel(order="F")), C.c_int(prob.onerdm.shape[0]), d(qv),
        C.c_int(qv.size), C.c_double(prob.cutoffz), C.c_double(prob.cutoffmd), C.c_double(prob.cutoffcentre),
        d(np.asarray(Zn, dtype=np.float64)), d(geom), C.c_int(len(prob.atoms)), C.c_int(bessel_mode),
        out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle orc_nuclear failed with code {rc}")
    return out


def nuclear_nuclear(prob, Zn, q=None) -> np.ndarray:
    """Inn(q) = sum_ij Zn_i Zn_j sinc(q R_ij) (src/main_calculation.f90:302-311; sinc(0) = 1)."""
    qv = prob.q if q is None else np.asarray(q, dtype=np.float64)
    R = np.asarray(prob.atoms, dtype=np.float64)
    Zn = np.asarray(Zn, dtype=np.float64)
    out = np.zeros(qv.size)
    for a in range(len(R)):
        for b in range(len(R)):
            x = qv * np.sqrt(np.sum((R[a] - R[b]) ** 2))
            s = np.where(np.abs(x) < 1e-10, 1.0, np.sin(x) / np.where(np.abs(x) < 1e-10, 1.0, x))
            out += Zn[a] * Zn[b] * s
    return out


def electron(prob, type_: int, Zn, *, bessel_mode: int = 1, nthreads: int = 0) -> np.ndarray:
    """Electron scattering, types 5 (total) and 6 (elastic) of main_calculation
    (src/main_calculation.f90:277-329, 330-...): I_e - 2 Ine + Inn with I_e the
    total (type 5) or elastic (type 6) j0 intensity."""
    Ie = scattering(prob, 1 if type_ == 5 else 2, bessel_mode=bessel_mode, nthreads=nthreads)
    return Ie - 2.0 * nuclear(prob, Zn, bessel_mode=bessel_mode) + nuclear_nuclear(prob, Zn)


def count_te(prob, quartets=None, *, rho=None, nthreads: int = 0):
    """Per listed quartet (default: the five loops' list) the number T_E of
    innermost Hermite-product updates of tot_integral_k_ijkr that pass both
    cutoffs, and whether the quartet takes the P = Q branch (whose
    tot_integral_ijkr_pzero terms are counted instead).  Returns (te, is_p0)."""
    keep = []

    def d(x):
        a, p = _d(x)
        keep.append(a)
        return p

    def i(x):
        a, p = _i(x)
        keep.append(a)
        return p

    qs = enum_quartets(prob.ng) if quartets is None else np.ascontiguousarray(quartets, dtype=np.int32)
    te = np.zeros(qs.shape[0], dtype=np.int64)
    p0 = np.zeros(qs.shape[0], dtype=np.int32)
    mat_cm = np.asfortranarray(prob.mat.astype(np.int32)).ravel(order="F")
    mmod_cm = np.asfortranarray(prob.mmod).ravel(order="F")
    rc = lib().orc_count_te(
        C.c_int(prob.ngto), d(prob.ga), i(prob.l), i(prob.m), i(prob.n), d(prob.xx), d(prob.yy), d(prob.zz),
        i(prob.group), d(mmod_cm), C.c_int(prob.nmo), i(mat_cm), d(prob.total), C.c_int(prob.mat.shape[0]),
        d(rho) if rho is not None else None, C.c_double(prob.cutoffz), C.c_double(prob.cutoffmd),
        C.c_double(prob.cutoffcentre), i(qs), C.c_long(qs.shape[0]), C.c_int(nthreads),
        te.ctypes.data_as(C.POINTER(C.c_long)), p0.ctypes.data_as(C.POINTER(C.c_int)))
    if rc != 0:
        raise RuntimeError(f"oracle orc_count_te failed with code {rc}")
    return te, p0.astype(bool)


def elastic_aligned_grid(nq: int) -> np.ndarray:
    """The q vectors of CASE(4) (src/main_calculation.f90:227-241), shape (nq, 3)."""
    out = np.zeros((nq, 3))
    lib().orc_elastic_aligned_grid(C.c_int(nq), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def elastic_aligned(prob, qal=None, nq: int = 100):
    """Elastic aligned intensity |F(q)|^2 of CASE(4) (elastic_integration_alig,
    src/Integrals.f90:2366-2490); q vectors default to the CASE(4) grid.
    Returns (F_re, F_im, |F|^2)."""
    keep = []

    def d(x):
        a, p = _d(x)
        keep.append(a)
        return p

    def i(x):
        a, p = _i(x)
        keep.append(a)
        return p

    qal = elastic_aligned_grid(nq) if qal is None else np.ascontiguousarray(qal, dtype=np.float64).reshape(-1, 3)
    n = qal.shape[0]
    fr, fi, res = np.zeros(n), np.zeros(n), np.zeros(n)
    rc = lib().orc_elastic_aligned(
        C.c_int(prob.ngto), d(prob.ga), i(prob.l), i(prob.m), i(prob.n), d(prob.xx), d(prob.yy), d(prob.zz),
        i(prob.group), d(np.asfortranarray(prob.mmod).ravel(order="F")), C.c_int(prob.nmo),
        d(np.asfortranarray(prob.onerdm).ravel(order="F")), C.c_int(prob.onerdm.shape[0]), d(qal), C.c_int(n),
        fr.ctypes.data_as(C.POINTER(C.c_double)), fi.ctypes.data_as(C.POINTER(C.c_double)),
        res.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle orc_elastic_aligned failed with code {rc}")
    return fr, fi, res
