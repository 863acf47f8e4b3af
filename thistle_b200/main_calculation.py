"""Host-side mirror of THISTLE's calculation dispatcher, on the B200 path.

``total_scattering_calculation`` keeps the argument meaning and order of the
f2py call the reference's Python driver makes
(``main_calculation.total_scattering_calculation``, src/main_calculation.f90:13-15,
called at src/scattering_main_routine.py:240-247) and returns ``(q_abs, result)``
like it.  The CI vectors of that call (``confs, civecs``) are replaced by the
RDMs they produce, which is the ``readrdm`` form of
``total_scattering_calculation_2`` (src/main_calculation.f90:501-849);
``total_scattering_calculation_2`` itself reads the same RDM files as the
reference (read_twordm / read_onerdm, src/one_rdm.f90:2072-2147).

Every call runs on the current CUDA device through libthistle_b200.so; errors
come back as :class:`ThistleError` with the library's status code.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import ThistleError, check, colmajor_f64, colmajor_i32, dptr, iptr

TOTAL_J0 = 1
ELASTIC_J0 = 2
TOTAL_ALIGNED = 3
ELASTIC_ALIGNED = 4
TOTAL_J2 = 7
ELASTIC_J2 = 8
TOTAL_ELECTRON = 5
ELASTIC_ELECTRON = 6
RESOLVED_CMS = 9
TOTAL_J1 = 10  # refused: the reference's tot_integration_j1 stops before integrating


def read_twordm(filename):
    """Rows ``p q r s value`` of a 2-RDM file (src/one_rdm.f90:2112-2147)."""
    rows = np.loadtxt(filename, ndmin=2)
    mat = rows[:, :4].astype(np.int32)
    total = rows[:, 4].astype(np.float64)
    return mat, total


def read_twordm_listing(filename):
    """2-RDM rows as the reference's Python builder writes them
    (src/twordm.py:300-316): ``[p s q r] value`` per line, the index list
    printed by numpy with 0-based MO indices in the (m1, m2, m3, m4) order of
    the Fortran rows.  Returns read_twordm's 1-based ``(mat, total)``."""
    mat, total = [], []
    with open(filename) as f:
        for line in f:
            line = line.strip()
            if not line:
                continue
            head, _, val = line.rpartition("]")
            idx = [int(t) for t in head.lstrip("[").split()]
            if len(idx) != 4:
                raise ValueError(f"{filename}: expected 4 indices in {line!r}")
            mat.append([i + 1 for i in idx])
            total.append(float(val))
    return np.asarray(mat, dtype=np.int32).reshape(-1, 4), np.asarray(total, dtype=np.float64)


def read_onerdm(filename):
    """Rows ``i j value``; the matrix size is the last row's i (src/one_rdm.f90:2072-2108)."""
    rows = np.loadtxt(filename, ndmin=2)
    maxnmo = int(rows[-1, 0])
    D = np.zeros((maxnmo, maxnmo))
    for i, j, v in rows:
        D[int(i) - 1, int(j) - 1] = v
    return D


def _onerdms(onerdm, onerdm2):
    """Column-major 1-RDM argument of the C-ABI: one matrix, or for the
    resolved CMS the bra's and the ket's back to back."""
    if onerdm is None:
        return None, 0
    one = colmajor_f64(onerdm)
    nmo1 = int(np.asarray(onerdm).shape[0])
    if onerdm2 is not None:
        if np.shape(onerdm2) != np.shape(onerdm):
            raise ValueError("the two 1-RDMs of the resolved CMS must have one shape")
        one = np.concatenate([one, colmajor_f64(onerdm2)])
    return one, nmo1


def total_scattering_calculation(type, Zn, geom, state1, state2, maxl, ngto, ng, ga, l, m, n, xx, yy, zz,
                                 mmod, q, nq, group, cutoffz, cutoffmd, cutoffcentre, mat=None, total=None,
                                 onerdm=None, onerdm2=None):
    """I(q) for calculation ``type`` (1 total j0, 2 elastic j0, 3 total aligned, 4 elastic aligned,
    5 total electron, 6 elastic electron, 7 total j2, 8 elastic j2, 9 resolved CMS).

    Type 9 (CASE(9), src/main_calculation.f90:438-471) takes two 1-RDMs:
    ``onerdm`` for the bra's density zi and ``onerdm2`` for the ket's zj (the
    reference's transition 1-RDMs of states 1-3 and 2-3).  Type 10 raises
    :class:`ThistleError`: the reference's tot_integration_j1 stops before it
    integrates (src/Integrals.f90:526-527).

    Types 5 and 6 return I_e - 2 Ine + Inn (I_e the total or elastic j0
    intensity, Ine the nuclear-electron term, Inn the nuclear-nuclear sinc
    sum) and need ``Zn`` (natoms,), ``geom`` (natoms, 3) and ``onerdm``; type
    5 also the 2-RDM rows.

    Type 3 runs on the reference's QCOORD3 grid (``nq`` must be 3131; ``q``
    is not read): ``q_abs`` is |q| of the grid vectors and ``result`` the real
    part of the aligned intensity.  Type 4 runs on the reference's CASE(4) grid
    of ``nq`` vectors (``elastic_aligned_grid``; ``q`` is not read) and
    returns |q| and the elastic aligned intensity |F(q)|^2.

    ``mmod`` is (norbs, ngto) as the reference passes it; ``mat``/``total``
    are the 2-RDM rows (types 1 and 7), ``onerdm`` the 1-RDM (types 2 and 8).
    ``state1``/``state2`` select CI states in the reference and are unused
    here, where the RDMs are inputs.  Returns ``(q_abs, result)``.
    """
    del state1, state2
    ga = _abi.as_f64(ga)
    l, m, n, group = (_abi.as_i32(a) for a in (l, m, n, group))
    xx, yy, zz, q = (_abi.as_f64(a) for a in (xx, yy, zz, q))
    mmod = np.asarray(mmod, dtype=np.float64)
    norbs = mmod.shape[0]
    mcm = colmajor_f64(mmod)
    matcm = colmajor_i32(mat) if mat is not None else None
    tot = _abi.as_f64(total) if total is not None else None
    nmat = 0 if mat is None else int(np.asarray(mat).shape[0])
    if type == RESOLVED_CMS and (onerdm is None or onerdm2 is None):
        raise ValueError("type 9 needs onerdm and onerdm2")
    one, nmo1 = _onerdms(onerdm, onerdm2 if type == RESOLVED_CMS else None)
    Zn = _abi.as_f64(Zn) if Zn is not None else None
    natoms = 0
    if geom is not None:
        geom = np.asarray(geom, dtype=np.float64).reshape(-1, 3)
        natoms = int(geom.shape[0])
        if Zn is not None and Zn.size != natoms:
            raise ValueError(f"{Zn.size} nuclear charges for {natoms} atoms")
        geom = colmajor_f64(geom)
    q_abs = np.zeros(int(nq))
    result = np.zeros(int(nq))
    rc = _abi.lib().thistle_total_scattering(
        int(type), dptr(Zn), dptr(geom), natoms, int(maxl), int(ngto), int(ng), dptr(ga), iptr(l), iptr(m),
        iptr(n), dptr(xx), dptr(yy), dptr(zz), dptr(mcm), norbs, dptr(q), int(nq), iptr(group),
        float(cutoffz), float(cutoffmd), float(cutoffcentre), iptr(matcm), dptr(tot), nmat, dptr(one), nmo1,
        dptr(q_abs), dptr(result))
    check(rc)
    return q_abs, result


def total_scattering_calculation_2(type, Zn, geom, state1, state2, maxl, ngto, ng, ga, l, m, n, xx, yy, zz,
                                   mmod, q, nq, group, cutoffz, cutoffmd, cutoffcentre, fileJ, fileJ_2,
                                   readrdm=True):
    """The ``readrdm`` branch of total_scattering_calculation_2: type 1 and 7
    read the 2-RDM from ``fileJ_2``, types 2 and 8 the 1-RDM from ``fileJ``;
    type 9 reads its two 1-RDMs (bra, then ket) from ``fileJ`` and
    ``fileJ_2`` (the reference builds them from CI files there,
    src/main_calculation.f90:820-846, which is upstream of this path)."""
    if not readrdm:
        raise ThistleError(-7, "only the readrdm path is provided; CI-vector RDM construction is upstream")
    mat = total = onerdm = onerdm2 = None
    if type in (TOTAL_J0, TOTAL_J2):
        mat, total = read_twordm(fileJ_2)
    elif type in (ELASTIC_J0, ELASTIC_J2):
        onerdm = read_onerdm(fileJ)
    elif type == RESOLVED_CMS:
        onerdm, onerdm2 = read_onerdm(fileJ), read_onerdm(fileJ_2)
    return total_scattering_calculation(type, Zn, geom, state1, state2, maxl, ngto, ng, ga, l, m, n, xx, yy,
                                        zz, mmod, q, nq, group, cutoffz, cutoffmd, cutoffcentre, mat=mat,
                                        total=total, onerdm=onerdm, onerdm2=onerdm2)


class ScatteringPlan:
    """One basis + density + q grid on the device, executed per geometry."""

    def __init__(self, type, ga, l, m, n, xx, yy, zz, group, mmod, q, cutoffz, cutoffmd, cutoffcentre,
                 mat=None, total=None, onerdm=None, onerdm2=None):
        self._p = C.c_void_p()
        self.type = int(type)
        self._keep = [_abi.as_f64(ga), _abi.as_i32(l), _abi.as_i32(m), _abi.as_i32(n), _abi.as_f64(xx),
                      _abi.as_f64(yy), _abi.as_f64(zz), _abi.as_i32(group)]
        ga, l, m, n, xx, yy, zz, group = self._keep
        mmod = np.asarray(mmod, dtype=np.float64)
        self.ngto = int(ga.size)
        self.ng = int(group.max())
        # first function of each group (its centre is the group's)
        self.group_first = np.array([int(np.argmax(group == k + 1)) for k in range(self.ng)])
        self.ngeom = 1
        if self.type == TOTAL_ALIGNED:
            # nq vectors; the C side takes them (3, nq) column-major = rows of (qx, qy, qz)
            self.q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).reshape(-1, 3))
            self.nq = int(self.q.shape[0])
        else:
            self.q = _abi.as_f64(q)
            self.nq = int(self.q.size)
        mcm = colmajor_f64(mmod)
        matcm = colmajor_i32(mat) if mat is not None else None
        tot = _abi.as_f64(total) if total is not None else None
        one, nmo1 = _onerdms(onerdm, onerdm2 if self.type == RESOLVED_CMS else None)
        rc = _abi.lib().thistle_plan_create(
            C.byref(self._p), self.type, self.ngto, dptr(ga), iptr(l), iptr(m), iptr(n), dptr(xx), dptr(yy),
            dptr(zz), iptr(group), dptr(mcm), int(mmod.shape[0]), iptr(matcm), dptr(tot),
            0 if mat is None else int(np.asarray(mat).shape[0]), dptr(one),
            nmo1, dptr(self.q), self.nq, float(cutoffz),
            float(cutoffmd), float(cutoffcentre))
        check(rc)

    @classmethod
    def from_problem(cls, prob, type=TOTAL_J0, q=None, onerdm2=None):
        """Plan of a Problem; type 9 takes ``prob.onerdm`` for the bra and
        ``onerdm2`` for the ket."""
        one = type in (ELASTIC_J0, ELASTIC_J2, RESOLVED_CMS)
        return cls(type, prob.ga, prob.l, prob.m, prob.n, prob.xx, prob.yy, prob.zz, prob.group, prob.mmod,
                   prob.q if q is None else q, prob.cutoffz, prob.cutoffmd, prob.cutoffcentre,
                   mat=prob.mat if not one else None, total=prob.total if not one else None,
                   onerdm=prob.onerdm if one else None, onerdm2=onerdm2)

    def set_centres(self, xx, yy, zz):
        xx, yy, zz = (_abi.as_f64(a) for a in (xx, yy, zz))
        check(_abi.lib().thistle_plan_set_centres(self._p, dptr(xx), dptr(yy), dptr(zz)))

    def execute(self, out=None):
        out = np.zeros(self.nq) if out is None else out
        check(_abi.lib().thistle_plan_execute(self._p, dptr(out)))
        return out

    def execute_aligned(self):
        """Aligned plans: (Re, Im) of I(q) per q vector (Im is identically zero)."""
        re, im = np.zeros(self.nq), np.zeros(self.nq)
        check(_abi.lib().thistle_plan_execute_aligned(self._p, dptr(re), dptr(im)))
        return re, im

    def vjp(self, v):
        """Total j0: sum_q v(q) dI(q)/dA_g for every group centre A_g, shape (ng, 3)."""
        v = _abi.as_f64(v)
        if v.size != self.nq:
            raise ValueError(f"cotangent has {v.size} entries, the plan {self.nq} q points")
        g = np.zeros((self.ng, 3))
        check(_abi.lib().thistle_plan_vjp(self._p, dptr(v), dptr(g)))
        return g

    def form_factor(self, qvec):
        """Elastic plans: F(q) of the electron density on q vectors (nq, 3)
        and the elastic aligned intensity |F|^2 (type 4): (re, im, abs2)."""
        qv = np.ascontiguousarray(np.asarray(qvec, dtype=np.float64).reshape(-1, 3))
        n = qv.shape[0]
        re, im, a2 = np.zeros(n), np.zeros(n), np.zeros(n)
        check(_abi.lib().thistle_plan_form_factor(self._p, dptr(qv), n, dptr(re), dptr(im), dptr(a2)))
        return re, im, a2

    def nuclear(self, Zn, geom):
        """Elastic plans: the nuclear-electron term Ine(q) for nuclei at geom
        (natoms, 3) with charges Zn, at the plan's current centres."""
        Zn = _abi.as_f64(Zn)
        g3 = np.asarray(geom, dtype=np.float64).reshape(-1, 3)
        if g3.shape[0] != Zn.size:
            raise ValueError(f"geom has {g3.shape[0]} atoms, Zn {Zn.size}")
        g = colmajor_f64(g3)
        out = np.zeros(self.nq)
        check(_abi.lib().thistle_plan_nuclear(self._p, dptr(Zn), dptr(g), int(Zn.size), dptr(out)))
        return out

    def vjp_device(self, v_ptr: int, grad_ptr: int):
        """Device pointers (nq and 3 ng doubles), on the plan's stream."""
        check(_abi.lib().thistle_plan_vjp_device(self._p, C.c_void_p(v_ptr), C.c_void_p(grad_ptr)))

    # --- geometry batches -------------------------------------------------
    def set_batch(self, ngeom: int):
        """Hold ngeom geometries (all at geometry 0's centres until set_centres_batch)."""
        check(_abi.lib().thistle_plan_set_batch(self._p, int(ngeom)))
        self.ngeom = int(ngeom)

    def set_centres_batch(self, xyz):
        """Centres of every geometry: array (ngeom, ngto, 3)."""
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(self.ngeom, self.ngto, 3))
        check(_abi.lib().thistle_plan_set_centres_batch(self._p, dptr(xyz)))

    def execute_batch(self):
        out = np.zeros((self.ngeom, self.nq))
        check(_abi.lib().thistle_plan_execute_batch(self._p, dptr(out)))
        return out

    def vjp_batch(self, v):
        v = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(self.ngeom, self.nq))
        g = np.zeros((self.ngeom, self.ng, 3))
        check(_abi.lib().thistle_plan_vjp_batch(self._p, dptr(v), dptr(g)))
        return g

    def use_graph(self, enable: bool = True):
        check(_abi.lib().thistle_plan_use_graph(self._p, int(bool(enable))))

    def autotune_batch(self, gmax: int):
        """Pick the batch size, the stage-2 q tile and the stage-2 pair tile by
        timing forward + adjoint; returns (ngeom, qtile, geoms/s) and leaves
        the pair tile in the plan (``stage2_tile``)."""
        g, qt, gps = C.c_int32(0), C.c_int32(0), C.c_double(0.0)
        check(_abi.lib().thistle_plan_autotune_batch(self._p, int(gmax), C.byref(g), C.byref(qt), C.byref(gps)))
        self.ngeom = g.value
        return g.value, qt.value, gps.value

    def set_stage2_tile(self, quartets_per_lane: int, warps_per_block: int):
        """Stage-2 pair tile: quartets per lane (1, 2) and warps per block (4, 8)."""
        check(_abi.lib().thistle_plan_set_stage2_tile(self._p, int(quartets_per_lane), int(warps_per_block)))

    def set_pipeline(self, enable: bool = True):
        """Overlap each class's stage 2 with the later classes' stage 1 (the
        default); the result is the same either way."""
        check(_abi.lib().thistle_plan_set_pipeline(self._p, int(bool(enable))))

    def stage2_tile(self):
        k, nw = C.c_int32(0), C.c_int32(0)
        check(_abi.lib().thistle_plan_stage2_tile(self._p, C.byref(k), C.byref(nw)))
        return k.value, nw.value

    def set_centres_batch_device(self, ptr: int):
        """Centres of every geometry from device memory ((ngeom, ngto, 3)
        doubles at ``ptr``), stream-ordered on the plan's stream."""
        check(_abi.lib().thistle_plan_set_centres_batch_device(self._p, C.c_void_p(ptr)))

    def execute_batch_device(self, ptr: int):
        """I(q) of every geometry, (ngeom, nq) doubles to the device address ``ptr``."""
        check(_abi.lib().thistle_plan_execute_batch_device(self._p, C.c_void_p(ptr)))

    def vjp_batch_device(self, v_ptr: int, grad_ptr: int):
        """Device cotangents (ngeom, nq) -> group-centre gradients (ngeom, ng, 3)."""
        check(_abi.lib().thistle_plan_vjp_batch_device(self._p, C.c_void_p(v_ptr), C.c_void_p(grad_ptr)))

    def execute_device(self, ptr: int):
        """Integrator only, I(q) to the device address ``ptr`` (stream-ordered)."""
        check(_abi.lib().thistle_plan_execute_device(self._p, C.c_void_p(ptr)))

    def recompute_device(self, ptr: int):
        """Density transform + quartet enumeration + integrator from the
        device-resident inputs, I(q) to the device address ``ptr``."""
        check(_abi.lib().thistle_plan_recompute_device(self._p, C.c_void_p(ptr)))

    def set_stream(self, stream_handle: int):
        """Use a caller-owned CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        check(_abi.lib().thistle_plan_set_stream(self._p, C.c_void_p(stream_handle)))

    def class_counts(self):
        a = np.zeros(51, dtype=np.int64)
        check(_abi.lib().thistle_plan_class_counts(self._p, a.ctypes.data_as(_abi.I64)))
        a = a.reshape(17, 3)
        return {int(L): (int(n), int(p0)) for L, n, p0 in a if n}

    def execute_quartets(self, quartets):
        qt = np.ascontiguousarray(np.asarray(quartets, dtype=np.int32).reshape(-1, 4))
        out = np.zeros(self.nq)
        check(_abi.lib().thistle_plan_execute_quartets(self._p, iptr(qt), qt.shape[0], dptr(out)))
        return out

    def density(self):
        """The transformed density: the pair density (np, np) of total / j2 /
        aligned plans, the AO density (ngto, ngto) of elastic plans, and the
        two (zi, zj) of a resolved CMS plan as (2, ngto, ngto)."""
        need = C.c_int64(0)
        check(_abi.lib().thistle_plan_density(self._p, None, 0, C.byref(need)))
        out = np.zeros(need.value)
        check(_abi.lib().thistle_plan_density(self._p, dptr(out), need.value, C.byref(need)))
        if self.type == RESOLVED_CMS:
            return np.stack([z.reshape(self.ngto, self.ngto, order="F") for z in out.reshape(2, -1)])
        k = int(round(np.sqrt(need.value)))
        return out.reshape(k, k) if self.type not in (ELASTIC_J0, ELASTIC_J2) else out.reshape(k, k, order="F")

    def info(self):
        a = np.zeros(6, dtype=np.int64)
        check(_abi.lib().thistle_plan_info(self._p, a.ctypes.data_as(_abi.I64)))
        return dict(nquart=int(a[0]), nclasses=int(a[1]), ng=int(a[2]), ngto=int(a[3]), nq=int(a[4]),
                    launches=int(a[5]))

    def timings(self):
        a = np.zeros(6)
        check(_abi.lib().thistle_plan_timings(self._p, dptr(a)))
        return dict(pair_tables=a[0], stage1=a[1], stage2=a[2], reduce=a[3], transform=a[4], quartets=a[5])

    def records(self):
        """Device address of the last execution's stage-1 records, the class
        table (begin, end, record offset, stride per LLmax class) and the
        device address of the q grid."""
        rec, qd = C.c_void_p(), C.c_void_p()
        n = np.zeros(1, dtype=np.int32)
        b, e, o = (np.zeros(20, dtype=np.int64) for _ in range(3))
        rs = np.zeros(20, dtype=np.int32)
        check(_abi.lib().thistle_plan_records(self._p, C.byref(rec), iptr(n), b.ctypes.data_as(_abi.I64),
                                              e.ctypes.data_as(_abi.I64), o.ctypes.data_as(_abi.I64),
                                              iptr(rs), C.byref(qd)))
        k = int(n[0])
        return dict(rec=rec.value, q=qd.value, ncls=k, begin=b[:k].copy(), end=e[:k].copy(),
                    recoff=o[:k].copy(), rs=rs[:k].copy())

    def stage_totals(self):
        """Summed device ms per stage over the executions since the last call."""
        a = np.zeros(4)
        n = np.zeros(1, dtype=np.int64)
        check(_abi.lib().thistle_plan_stage_totals(self._p, dptr(a), n.ctypes.data_as(_abi.I64)))
        return dict(pair_tables=a[0], stage1=a[1], stage2=a[2], reduce=a[3], executions=int(n[0]))

    def close(self):
        if self._p:
            _abi.lib().thistle_plan_destroy(self._p)
            self._p = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MoleculeBatch:
    """Several plans (different molecules and bases, one geometry each, the
    same calculation type, at most 1024 q points each) executed together:
    stage 2 is one persistent launch over every (plan, class, block) item,
    the other stages one launch per kernel shape.  The plans must
    stay open while the batch is used; ``execute`` returns one I(q) array per
    plan, for each plan's current centres."""

    def __init__(self, plans):
        self.plans = list(plans)
        self._b = C.c_void_p()
        arr = (C.c_void_p * len(self.plans))(*[p._p.value for p in self.plans])
        check(_abi.lib().thistle_batch_create(C.byref(self._b), arr, len(self.plans)))
        self._split = np.cumsum([p.nq for p in self.plans])[:-1]
        self._nq = int(sum(p.nq for p in self.plans))

    def use_graph(self, enable: bool = True):
        check(_abi.lib().thistle_batch_use_graph(self._b, int(bool(enable))))

    def execute(self):
        out = np.zeros(self._nq)
        check(_abi.lib().thistle_batch_execute(self._b, dptr(out)))
        return np.split(out, self._split)

    def execute_device(self, ptr: int):
        """All plans' I(q), one after the other, to the device address ``ptr``
        (stream-ordered on the first plan's stream)."""
        check(_abi.lib().thistle_batch_execute_device(self._b, C.c_void_p(ptr)))

    def set_stage2_tile(self, quartets_per_lane: int, warps_per_block: int):
        """Stage-2 pair tile of the persistent launch: quartets per lane (1, 2)
        and warps per block (4, 8)."""
        check(_abi.lib().thistle_batch_set_stage2_tile(self._b, int(quartets_per_lane), int(warps_per_block)))

    def stage2_tile(self):
        k, nw = C.c_int32(0), C.c_int32(0)
        check(_abi.lib().thistle_batch_stage2_tile(self._b, C.byref(k), C.byref(nw)))
        return k.value, nw.value

    def autotune(self):
        """Time the batch at the four stage-2 pair tiles and keep the fastest;
        returns (quartets per lane, warps per block, molecules/s)."""
        k, nw, mps = C.c_int32(0), C.c_int32(0), C.c_double(0.0)
        check(_abi.lib().thistle_batch_autotune(self._b, C.byref(k), C.byref(nw), C.byref(mps)))
        return k.value, nw.value, mps.value

    def info(self):
        a = np.zeros(3, dtype=np.int64)
        check(_abi.lib().thistle_batch_info(self._b, a.ctypes.data_as(_abi.I64)))
        return dict(plans=int(a[0]), nq=int(a[1]), launches=int(a[2]))

    def close(self):
        if self._b:
            _abi.lib().thistle_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def atom_gradient(prob, group_grad):
    """Sum per-group centre gradients (ng, 3) onto the atoms carrying them."""
    g0 = np.array([np.argmax(prob.group == k + 1) for k in range(prob.ng)])
    out = np.zeros((prob.atoms.shape[0], 3))
    np.add.at(out, prob.atom_of[g0], np.asarray(group_grad))
    return out


def elastic_aligned_grid(nq: int) -> np.ndarray:
    """The reference's q vectors of the elastic aligned intensity (CASE(4),
    src/main_calculation.f90:227-241), shape (nq, 3)."""
    out = np.zeros((int(nq), 3))
    check(_abi.lib().thistle_elastic_aligned_grid(int(nq), dptr(out)))
    return out


def qcoord3(k0: float = 10.583544175) -> np.ndarray:
    """The reference's 3131 aligned q vectors (QCOORD3), shape (3131, 3)."""
    out = np.zeros((3131, 3))
    check(_abi.lib().thistle_qcoord3(float(k0), dptr(out)))
    return out


def aligned(prob, qvec=None):
    """Aligned total intensity (Re, Im) of a Problem on q vectors (default: the QCOORD3 grid)."""
    qv = qcoord3() if qvec is None else np.asarray(qvec, dtype=np.float64).reshape(-1, 3)
    with ScatteringPlan.from_problem(prob, TOTAL_ALIGNED, q=qv) as pl:
        return pl.execute_aligned()


def scattering(prob, type=TOTAL_J0, q=None, Zn=None, onerdm2=None):
    """I(q) of an :class:`thistle_b200.inputs.Problem` through Entry 1
    (types 5 and 6: nuclei at ``prob.atoms`` with charges ``Zn``; type 9:
    ``prob.onerdm`` on the bra, ``onerdm2`` on the ket)."""
    qv = prob.q if q is None else np.asarray(q, dtype=np.float64)
    two = type in (TOTAL_J0, TOTAL_J2, TOTAL_ELECTRON)
    one = type in (ELASTIC_J0, ELASTIC_J2, ELASTIC_ALIGNED, TOTAL_ELECTRON, ELASTIC_ELECTRON, RESOLVED_CMS)
    _, res = total_scattering_calculation(
        type, Zn, prob.atoms, 0, 0, int(max(prob.l.max(), prob.m.max(), prob.n.max())), prob.ngto, prob.ng,
        prob.ga, prob.l, prob.m, prob.n, prob.xx, prob.yy, prob.zz, prob.mmod, qv, qv.size, prob.group,
        prob.cutoffz, prob.cutoffmd, prob.cutoffcentre,
        mat=prob.mat if two else None, total=prob.total if two else None,
        onerdm=prob.onerdm if one else None, onerdm2=onerdm2)
    return res
