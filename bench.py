"""Benchmark of the B200 scattering-intensity path.

Workload (one step): the total j0 intensity of the AB6 octahedral molecule of
the benchmark configurations -- 7 atoms, 203 primitives in 98 shells, 40 MOs,
a 5 % sparse PSD 2-RDM (134 401 rows), 500 q points on 0..15 bohr^-1 --
computed from inputs already resident in HBM: density transform, quartet
enumeration, pair tables, stage 1 (Hermite densities and expansion
coefficients) and stage 2 (the quartet x q Bessel sum), i.e. everything the
reference's tot_integration does for the 11 920 622 group quartets of its five
loops.  The metric is reference-defined quartet.q evaluations per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl thistle|reference]

N > 1 (under torchrun) runs N independent replicas, one per GPU ("replicas
only": the path needs no collective); value = all ranks' quartet.q / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 quartet.q evals/s (total j0, AB6 octahedral, 500 q)"
UNIT = "quartet.q/s"


def fb_flops(L: int) -> int:
    """Algorithmic FLOPs of one Bessel-branch quartet.q: per order 2 (j_b by
    recurrence) + 1 ((q/H)^b update) + 2 (FMA into the sum); fixed 10: qH, 1/x,
    sincos (2), Gaussian exponent (2), exp (1), x K K' w (2), accumulate (1)."""
    return 5 * (L + 1) + 10


def p0_flops(L: int) -> int:
    """P = Q branch: Horner over L/2+1 even powers (2 each) + exp, scale, add."""
    return 2 * (L // 2 + 1) + 3


WORKLOAD = "ab6"


def workload():
    from thistle_b200 import inputs as I
    if WORKLOAD == "ab6_4atom":
        return I.config3_ab6(natoms=4)
    return I.config3_ab6()


def max_over_ranks(ms: float, device: str) -> float:
    """The slowest rank's time (every rank calls this, in the same order)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world: int, units_per_step: int, steps: int, ms: float) -> float:
    """Replicas: every rank processes units_per_step per step; the job's rate
    is all ranks' units over the slowest rank's time."""
    return world * units_per_step * steps / (ms * 1e-3)


def workload_config(p, nquart):
    return {
        "workload": f"ab6_total_j0: {len(p.atoms)} atoms, {p.ngto} primitives ({p.ng} shells), {p.nmo} MOs, "
                    f"{p.mat.shape[0]}-row 5% sparse 2-RDM, {p.nq} q on 0..15 bohr^-1",
        "quartets_per_step": int(nquart),
        "quartet_q_per_step": int(nquart) * p.nq,
        "l2": "inputs larger than L2 (pair density %.1f GB, quartet records > 0.5 GB); no flush"
              % (8 * (p.ngto * (p.ngto + 1) / 2) ** 2 / 1e9),
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smmax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smmax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smmax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def llmax_of_quartets(p, qs):
    heads = np.searchsorted(p.group, np.arange(1, p.ng + 1))
    gl = (p.l + p.m + p.n)[heads]
    return gl[qs[:, 0]] + gl[qs[:, 1]] + gl[qs[:, 2]] + gl[qs[:, 3]]


def stratified_indices(L, frac, rng):
    """A proportional sample stratified by LLmax class: round(frac x class
    size) quartets of every class (at least one), so the sample's mix of
    classes is the workload's and its rate estimates the whole run's."""
    pick = []
    for LL in np.unique(L):
        idx = np.flatnonzero(L == LL)
        k = max(1, int(round(frac * idx.size)))
        pick.append(rng.choice(idx, size=min(k, idx.size), replace=False))
    return np.sort(np.concatenate(pick))


def cpu_baseline(p, target_s: float = 15.0, seed: int = 11):
    """The oracle (C restatement of the reference's five loops with its
    per-quartet dgemm contraction of the 2-RDM rows, dphrec Bessel functions)
    on a sample of the workload's quartets stratified by LLmax class, all host
    threads; the rate is extrapolated to the whole workload."""
    from oracle import oracle as O
    ncores = os.cpu_count() or 1
    qs = O.enum_quartets(p.ng)
    L = llmax_of_quartets(p, qs)
    rng = np.random.default_rng(seed)
    frac = 2e-5
    while True:
        idx = stratified_indices(L, frac, rng)
        t0 = time.perf_counter()
        O.scattering(p, 1, quartets=qs[idx], nthreads=ncores)
        dt = time.perf_counter() - t0
        if dt >= 0.5 * target_s or frac >= 1.0:
            break
        frac = min(1.0, frac * max(2.0, 1.05 * target_s / max(dt, 1e-3)))
    n = idx.size
    value = n * p.nq / dt
    return {"value": value, "unit": UNIT, "cores": ncores, "cpu_model": cpu_model(), "kind": "port",
            "extrapolated": True,
            "sample": f"{n} of {len(qs)} group quartets ({100 * n / len(qs):.3f} %), stratified by LLmax class "
                      f"in proportion to the class sizes (seed {seed}), all {p.nq} q; {dt:.1f} s on {ncores} host "
                      f"threads ({cpu_model()}); oracle/thistle_oracle.c restating tot_integration with the "
                      f"per-quartet dgemm of the 2-RDM rows (the reference's transform) inside every quartet; "
                      f"rate extrapolated to all quartets"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle import oracle as O
    p = workload()
    ncores = os.cpu_count() or 1
    qs = O.enum_quartets(p.ng)
    L = llmax_of_quartets(p, qs)
    rng = np.random.default_rng(17)
    # each step a sample stratified by LLmax class (in proportion to the class
    # sizes) of 0.25-2 s of work on all host threads (about a minute for the
    # whole run), sized from a first untimed call
    frac = 2e-5
    idx = stratified_indices(L, frac, rng)
    t0 = time.perf_counter()
    O.scattering(p, 1, quartets=qs[idx], nthreads=ncores)
    step_s = min(2.0, max(0.25, 60.0 / max(1, args.warmup + args.steps)))
    frac = min(1.0, frac * step_s / max(time.perf_counter() - t0, 1e-3))
    times, counts = [], []
    for s in range(args.warmup + args.steps):
        idx = stratified_indices(L, frac, rng)
        t0 = time.perf_counter()
        O.scattering(p, 1, quartets=qs[idx], nthreads=ncores)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
            counts.append(idx.size)
    tot = sum(times)
    per_step = int(np.mean(counts))
    value = sum(counts) * p.nq / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; BASELINE configuration 3 shapes)",
        "config": {"workload": workload_config(p, len(qs))["workload"],
                   "sample_per_step": f"about {per_step} group quartets x {p.nq} q, stratified by LLmax "
                                      f"class in proportion to the class sizes"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "cpu_model": cpu_model(), "kind": "port",
                         "extrapolated": True,
                         "sample": f"about {per_step} group quartets per step stratified by LLmax class, {ncores} "
                                   f"host threads ({cpu_model()}); the C restatement of tot_integration with its "
                                   f"per-quartet dgemm (no Fortran compiler on this image)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def h2d_bytes(p):
    ng = p.ng
    npair = ng * (ng + 1) // 2
    return int(8 * p.ngto + 24 * p.ngto + 4 * p.ngto + 8 * ng + 8 * p.nq + 8 * p.nmo * p.ngto
               + 16 * p.mat.shape[0] + 8 * p.mat.shape[0] + 8 * (npair + 1) + 4 * ng)


def e2e_entry1(p, steps, warmup):
    """Entry 1 (thistle_total_scattering) from pinned host buffers: set-up,
    H2D, transform, enumeration, integrator, D2H -- per step."""
    import torch
    from thistle_b200 import main_calculation as MC

    def pinned(a):
        t = torch.empty(a.shape, dtype={np.float64: torch.float64, np.int32: torch.int32}[a.dtype.type],
                        pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    args = dict(ga=pinned(p.ga), l=pinned(p.l), m=pinned(p.m), n=pinned(p.n), xx=pinned(p.xx), yy=pinned(p.yy),
                zz=pinned(p.zz), group=pinned(p.group), mmod=pinned(np.ascontiguousarray(p.mmod)),
                q=pinned(p.q), mat=pinned(np.ascontiguousarray(p.mat)), total=pinned(p.total))

    def call():
        return MC.total_scattering_calculation(
            1, None, None, 0, 0, 2, p.ngto, p.ng, args["ga"], args["l"], args["m"], args["n"], args["xx"],
            args["yy"], args["zz"], args["mmod"], args["q"], p.nq, args["group"], p.cutoffz, p.cutoffmd,
            p.cutoffcentre, mat=args["mat"], total=args["total"])[1]

    for _ in range(warmup):
        call()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        res = call()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    return dt, res


def run_fit(args):
    print(json.dumps(fit6_section(args.fit_geometries, args.fit_plain, args.fit_gmax)), flush=True)
    return 0


def fit6_section(ngeom_total, nplain_max, gmax):
    """Configuration 5: a 6-atom ring (configuration-2 basis per atom, 30 MOs,
    dense 2-RDM, 400 q) at 512 geometries; per geometry the forward I(q) and
    the adjoint dLoss/dR for Loss = sum_q (I(q; R) - I_ref(q))^2.  The plain
    path runs one geometry per call (set_centres, execute, vjp); the batched
    path holds an autotuned number of geometries per plan, replays CUDA graphs
    and runs every stage once per batch.  Both from the same plan set-up."""
    import torch
    from thistle_b200 import inputs as I
    from thistle_b200 import main_calculation as MC
    torch.cuda.set_device(0)
    p = I.config5_fit()
    geos = I.config5_geometries(p, ngeom_total)
    probs = [p.with_geometry(R) for R in geos]
    xyz = np.stack([np.stack([q.xx, q.yy, q.zz], axis=1) for q in probs])
    ng = len(probs)
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        iref = pl.execute()
        nquart = pl.info()["nquart"]
        # plain per-geometry path
        nplain = min(ng, nplain_max)
        for k in range(3):
            pl.set_centres(*xyz[k].T)
            I0 = pl.execute()
            pl.vjp(2 * (I0 - iref))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(nplain):
            pl.set_centres(*xyz[k].T)
            Ik = pl.execute()
            pl.vjp(2 * (Ik - iref))
        torch.cuda.synchronize()
        t_plain = (time.perf_counter() - t0) / nplain
        # batched path
        pl.use_graph(True)
        G, qt, gps_tune = pl.autotune_batch(gmax)
        nb = (ng + G - 1) // G
        gbuf = np.zeros((nb * G, p.ng, 3))
        ibuf = np.zeros((nb * G, p.nq))
        pad = np.concatenate([xyz, np.repeat(xyz[:1], nb * G - ng, axis=0)])
        for b in range(min(nb, 2)):
            pl.set_centres_batch(pad[b * G:(b + 1) * G])
            Ib = pl.execute_batch()
            pl.vjp_batch(2 * (Ib - iref))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for b in range(nb):
            pl.set_centres_batch(pad[b * G:(b + 1) * G])
            Ib = pl.execute_batch()
            ibuf[b * G:(b + 1) * G] = Ib
            gbuf[b * G:(b + 1) * G] = pl.vjp_batch(2 * (Ib - iref))
        torch.cuda.synchronize()
        t_batch = (time.perf_counter() - t0) / ng
        stages = fit6_stage_table(pl, xyz, iref, pad, G, min(nplain, 8))
        # spot check: the batched answer of the last geometry against the plain path
        pl.set_batch(1)
        pl.set_centres(*xyz[ng - 1].T)
        Ichk = pl.execute()
        gchk = pl.vjp(2 * (Ichk - iref))
    err_i = float(np.max(np.abs(ibuf[ng - 1] - Ichk)) / np.max(np.abs(Ichk)))
    err_g = float(np.max(np.abs(gbuf[ng - 1] - gchk)) / np.max(np.abs(gchk)))
    line = {
        "metric": "geometries/s, forward I(q) + adjoint dLoss/dR (fit6, 400 q)", "value": 1.0 / t_batch,
        "unit": "geometries/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded; BASELINE configuration 5 shapes)",
        "config": {"workload": f"fit6: 6-atom ring, {p.ngto} primitives ({p.ng} shells), {p.nmo} MOs, dense 2-RDM "
                               f"({p.mat.shape[0]} rows), {p.nq} q, {ng} geometries (sigma 0.1 bohr)",
                   "quartets_per_geometry": int(nquart), "autotuned_batch": G, "autotuned_qtile": qt},
        "plain_geometries_per_s": 1.0 / t_plain, "plain_sample_geometries": nplain,
        "batched_over_plain": t_plain / t_batch,
        "quartet_q_per_s_forward_and_adjoint": nquart * p.nq / t_batch,
        "check_vs_plain": {"I_rel": err_i, "grad_rel": err_g},
        "path": "host arrays in and out per batch (set_centres_batch, execute_batch, vjp_batch)",
        "per_stage_ms_per_geometry": stages,
    }
    return line


def fit6_stage_table(pl, xyz, iref, pad, G, nplain):
    """Per-geometry device time by stage, plain (one geometry per call) and
    batched (G per call, without CUDA graphs so that the stage events are
    recorded): the forward stages from the plan's stage events, and the
    forward and the adjoint call each timed with a synchronize on both sides
    (host copies included)."""
    import torch

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    pl.use_graph(False)
    pl.set_batch(1)
    pl.stage_totals()
    tf = tv = 0.0
    for k in range(nplain):
        pl.set_centres(*xyz[k].T)
        Ik, dt = timed(pl.execute)
        tf += dt
        _, dt = timed(lambda: pl.vjp(2 * (Ik - iref)))
        tv += dt
    st = pl.stage_totals()
    plain = {k: st[k] / max(st["executions"], 1) for k in ("pair_tables", "stage1", "stage2", "reduce")}
    plain.update(forward_call=1e3 * tf / nplain, adjoint_call=1e3 * tv / nplain)
    pl.set_batch(G)
    pl.set_centres_batch(pad[:G])
    Ib = pl.execute_batch()
    pl.vjp_batch(2 * (Ib - iref))
    pl.stage_totals()
    tf = tv = 0.0
    nb = min(2, len(pad) // G)
    for b in range(nb):
        pl.set_centres_batch(pad[b * G:(b + 1) * G])
        Ib, dt = timed(pl.execute_batch)
        tf += dt
        _, dt = timed(lambda: pl.vjp_batch(2 * (Ib - iref)))
        tv += dt
    st = pl.stage_totals()
    ng = nb * G
    batched = {k: st[k] / max(st["executions"], 1) / G for k in ("pair_tables", "stage1", "stage2", "reduce")}
    batched.update(forward_call=1e3 * tf / ng, adjoint_call=1e3 * tv / ng)
    pl.use_graph(True)
    return {"plain": plain, "batched_no_graph": batched,
            "what": "ms per geometry; pair_tables / stage1 / stage2 / reduce from the plan's stage events "
                    "(device), forward_call / adjoint_call wall time of one call with host copies"}


def run_batch4(args):
    print(json.dumps(batch4_section(args.batch_molecules, args.batch_chunk, args.batch_gb, min(args.steps, 10))),
          flush=True)
    return 0


def batch4_section(nmol, chunk, gb, reps_arg):
    """Configuration 4: uneven molecules (2-12 atoms, s4p2d1 per atom, 4-24
    MOs, sparse 2-RDMs, total j0 on 256 q).  Molecules are taken in chunks that
    fit the device; per chunk every molecule gets its plan (density transform,
    quartet list), then the chunk's I(q) is computed twice: once plan by plan
    (the plain GPU path, one integrator call per molecule) and once as a
    molecule batch (stage 2 one persistent launch over every (molecule,
    class, block) item, the other stages one launch per kernel shape,
    replayed from a CUDA graph) at the stage-2 pair tile the batch tuner
    picks for the chunk.  Both integrator paths start from the same plans and
    copy I(q) to host memory; set-up and tuning time are reported
    separately."""
    import torch
    from thistle_b200 import _abi
    from thistle_b200 import inputs as I
    from thistle_b200 import main_calculation as MC
    import ctypes as C
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    mols = I.config4_batch(nmol=nmol)
    t_gen = time.perf_counter() - t0
    budget = gb * 1e9
    t_setup = t_plain = t_batch = 0.0
    qq = 0
    nchunks, launches, tiles, err, t_tune = 0, [], [], 0.0, 0.0
    i = 0
    while i < len(mols):
        plans = []
        cached, used = C.c_int64(0), C.c_int64(0)
        while i < len(mols) and len(plans) < chunk:
            t0 = time.perf_counter()
            pl = MC.ScatteringPlan.from_problem(mols[i], MC.TOTAL_J0)
            pl.execute()  # first execution allocates the records
            t_setup += time.perf_counter() - t0
            plans.append(pl)
            qq += pl.info()["nquart"] * pl.nq
            i += 1
            _abi.check(_abi.lib().thistle_device_cache_bytes(C.byref(cached), C.byref(used)))
            if used.value > budget:
                break
        # plain: one integrator call per molecule
        for pl in plans[:2]:
            pl.execute()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        singles = [pl.execute() for pl in plans]
        t_plain += time.perf_counter() - t0
        # batched: stage 2 of every molecule of the chunk in one persistent launch
        with MC.MoleculeBatch(plans) as b:
            b.use_graph(True)
            t0 = time.perf_counter()
            k, nw, _ = b.autotune()
            t_tune += time.perf_counter() - t0
            tiles.append([k, nw])
            for _ in range(2):
                b.execute()
            torch.cuda.synchronize()
            reps = max(1, reps_arg)
            t0 = time.perf_counter()
            for _ in range(reps):
                out = b.execute()
            t_batch += (time.perf_counter() - t0) / reps
            launches.append(b.info()["launches"])
        err = max(err, max(float(np.max(np.abs(o - s)) / np.max(np.abs(s))) for o, s in zip(out, singles)))
        for pl in plans:
            pl.close()
        nchunks += 1
    n = len(mols)
    line = {
        "metric": "molecules/s, total j0 I(q) of an uneven molecule batch (256 q)", "value": n / t_batch,
        "unit": "molecules/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded; BASELINE configuration 4 shapes)",
        "config": {"workload": f"batch4: {n} molecules of 2-12 atoms, s(4)+p(2)+d(1) per atom, 4-24 MOs, "
                               f"sparse 2-RDMs (1-10 %), 256 q", "chunks": nchunks,
                   "max_molecules_per_chunk": chunk, "chunk_budget_gb": gb},
        "plain_molecules_per_s": n / t_plain, "batched_over_plain": t_plain / t_batch,
        "quartet_q_per_s_batched": qq / t_batch, "quartet_q_per_s_plain": qq / t_plain,
        "setup_s_per_molecule": t_setup / n, "input_generation_s": t_gen,
        "kernel_launches_per_chunk": launches[:4], "stage2_tile_per_chunk": tiles[:4],
        "tune_s_per_chunk": t_tune / max(1, nchunks), "check_vs_plain_max_rel": err,
        "path": "integrator only, from plans already built; host I(q) out (MoleculeBatch.execute vs "
                "ScatteringPlan.execute per molecule)",
    }
    return line


def bench_extras(args, p, plan, stream, stage1_ms, peak_tf, fwd_ms):
    """The rest of the benchmark metric on one GPU, after the timed forward
    steps: the adjoint of the same AB6 step, the stage-1 roofline, and the
    batched-versus-plain comparisons of configurations 5 (forward + adjoint
    over geometries) and 4 (uneven molecules)."""
    import torch
    out = {}
    # adjoint: sum_q v(q) dI(q)/dA for the 98 group centres, forward records valid
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    v = torch.randn(p.nq, dtype=torch.float64, device="cuda", generator=g)
    grad = torch.empty(3 * p.ng, dtype=torch.float64, device="cuda")
    for _ in range(2):
        plan.vjp_device(v.data_ptr(), grad.data_ptr())
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.vjp_device(v.data_ptr(), grad.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    adj_ms = e0.elapsed_time(e1) / args.steps
    out["ab6_adjoint"] = {
        "ms": adj_ms, "forward_plus_adjoint_ms": fwd_ms + adj_ms,
        "geometries_per_s_forward_plus_adjoint": 1e3 / (fwd_ms + adj_ms),
        "what": "thistle_plan_vjp_device: sum_q v(q) dI(q)/dA for all 98 group centres (21 nuclear "
                "coordinates), CUDA events over the timed adjoint calls, forward records of the same centres",
        "steps": args.steps, "grad_finite": bool(torch.isfinite(grad).all().item())}
    # stage 1 against its algorithmic FLOPs (counted once by the oracle, oracle/stage1_flops.py)
    prof = os.path.join(ROOT, "profiles", "stage1_ab6_flops.json")
    if WORKLOAD == "ab6" and os.path.exists(prof):
        fl = json.load(open(prof))["flops_per_step"]
        npair = p.ngto * (p.ngto + 1) // 2
        tf = fl / (stage1_ms * 1e-3) / 1e12
        out["roofline_stage1"] = {
            "bound": "fp64", "achieved": tf, "peak": peak_tf, "unit": "TFLOP/s",
            "frac": tf / peak_tf if peak_tf > 0 else None, "kernel_ms": stage1_ms, "flops_per_step": fl,
            "flops_basis": "F_E = 2 (LLmax+1) T_E per quartet (2 T_E on the P = Q branch), T_E counted by the "
                           "oracle under the same cutoffs (profiles/stage1_ab6_flops.json)",
            "rho_unique_half_bytes": 8 * npair * (npair + 1) // 2,
            "hbm_floor_ms": 8 * npair * (npair + 1) / 2 / 6524e9 * 1e3}
    if args.extras != "all":
        return out
    t0 = time.perf_counter()
    out["fit6"] = fit6_section(args.extra_fit_geometries, 16, 64)
    out["fit6"]["section_s"] = time.perf_counter() - t0
    out["fit6"]["config"]["reduction"] = (f"{args.extra_fit_geometries} of the configuration's 512 geometries, "
                                          f"16 timed on the plain path, so the default run stays short; "
                                          f"bench.py --workload fit6 runs all 512")
    t0 = time.perf_counter()
    out["batch4"] = batch4_section(args.extra_batch_molecules, 128, 60.0, 3)
    out["batch4"]["section_s"] = time.perf_counter() - t0
    out["batch4"]["config"]["reduction"] = (f"the first {args.extra_batch_molecules} of the configuration's 1024 "
                                            f"seeded molecules, so the default run stays short; bench.py "
                                            f"--workload batch4 runs all 1024")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120,
                    help="timed steps (AB6: 120 steps are about 2.2 s, so the clock record has samples under load)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="thistle", choices=["thistle", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--workload", default="ab6", choices=["ab6", "ab6_4atom", "fit6", "batch4"],
                    help="ab6_4atom: the first 4 atoms only, a profiling-size case of the same basis; "
                         "fit6: batched forward + adjoint over geometries (configuration 5); "
                         "batch4: uneven molecule batches (configuration 4)")
    ap.add_argument("--extras", default="all", choices=["all", "adjoint", "none"],
                    help="keys of the default line beyond the forward step: all (AB6 adjoint, stage-1 "
                         "roofline, fit6, batch4), adjoint (the first two only) or none")
    ap.add_argument("--extra-fit-geometries", type=int, default=128)
    ap.add_argument("--extra-batch-molecules", type=int, default=256)
    ap.add_argument("--fit-geometries", type=int, default=512)
    ap.add_argument("--fit-plain", type=int, default=32, help="geometries timed on the plain path")
    ap.add_argument("--fit-gmax", type=int, default=64)
    ap.add_argument("--batch-molecules", type=int, default=1024)
    ap.add_argument("--batch-chunk", type=int, default=128, help="molecules per batch at most")
    ap.add_argument("--batch-gb", type=float, default=60.0, help="device memory held per chunk of plans")
    args = ap.parse_args()
    if args.workload == "fit6" and args.impl == "thistle":
        return run_fit(args)
    if args.workload == "batch4" and args.impl == "thistle":
        return run_batch4(args)
    global WORKLOAD
    WORKLOAD = args.workload
    args.warmup = max(args.warmup, 3) if args.impl == "thistle" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from thistle_b200 import _abi
    from thistle_b200 import main_calculation as MC
    import ctypes as C

    p = workload()
    stream = torch.cuda.current_stream()
    plan = MC.ScatteringPlan.from_problem(p, MC.TOTAL_J0)
    plan.set_stream(stream.cuda_stream)
    nquart = plan.info()["nquart"]
    out = torch.empty(p.nq, dtype=torch.float64, device="cuda")

    peak = C.c_double(0.0)
    _abi.check(_abi.lib().thistle_probe_fp64_peak(5, C.byref(peak)))
    peak_tf = peak.value

    for _ in range(args.warmup):
        plan.recompute_device(out.data_ptr())
    torch.cuda.synchronize()
    plan.stage_totals()  # reset
    launches_per_step = plan.info()["launches"]
    counts = plan.class_counts()

    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ
                           else local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.recompute_device(out.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    st = plan.stage_totals()
    if world > 1:
        ms = max_over_ranks(ms, "cuda")
    result = out.cpu().numpy()

    qq_step = nquart * p.nq
    value = whole_job_value(world, qq_step, args.steps, ms)
    n2 = max(st["executions"], 1)
    flops = 0
    for L, (n, n0) in counts.items():
        flops += ((n - n0) * fb_flops(L) + n0 * p0_flops(L)) * p.nq
    # The timed steps overlap each class's stage 2 with the later classes'
    # stage 1, so their stage-2 interval (first class ready -> last class
    # done) also holds stage-1 work.  The kernel's own rate is timed over a
    # second loop of the same steps with the overlap off (stage 2 alone on the
    # GPU, events on its streams' join); both are reported.
    s2_span_ms = st["stage2"] / n2
    k2 = min(args.steps, 30)
    plan.set_pipeline(False)
    for _ in range(2):
        plan.recompute_device(out.data_ptr())
    torch.cuda.synchronize()
    plan.stage_totals()
    for _ in range(k2):
        plan.recompute_device(out.data_ptr())
    torch.cuda.synchronize()
    st_serial = plan.stage_totals()
    plan.set_pipeline(True)
    s2_ms = st_serial["stage2"] / max(st_serial["executions"], 1)
    achieved = flops / (s2_ms * 1e-3) / 1e12
    traffic = None
    prof = os.path.join(ROOT, "profiles", "stage2_ab6_dram.json")
    if WORKLOAD == "ab6" and os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
                "frac": achieved / peak_tf if peak_tf > 0 else None, "traffic": traffic,
                "kernel": "stage2_kernel (quartet x q Bessel sum)", "kernel_ms": s2_ms,
                "flops_per_launch": flops,
                "peak_source": "measured FP64 FMA rate of this GPU (thistle_probe_fp64_peak, in this run)",
                "timed_over": f"{k2} steps with the stage-1/stage-2 overlap off (stage 2 alone); the headline "
                              f"steps overlap them",
                "overlapped": {"stage2_span_ms": s2_span_ms,
                               "frac_of_span": (flops / (s2_span_ms * 1e-3) / 1e12) / peak_tf if peak_tf > 0 else None}}

    extras = {}
    if world == 1 and args.extras != "none":
        extras = bench_extras(args, p, plan, stream, st_serial["stage1"] / max(st_serial["executions"], 1), peak_tf,
                              ms / args.steps)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; BASELINE configuration 3 shapes)",
        "config": dict(workload_config(p, nquart), parallelism=("replicas x%d" % world) if world > 1 else "1 GPU"),
        "roofline": roofline,
        "stage_ms_per_step": {k: v / n2 for k, v in st.items() if k != "executions"},
        "stage_ms_note": "timed steps: the stage-1 and stage-2 intervals overlap (a class's stage 2 starts after "
                         "its own stage 1); stage_ms_per_step_serial: the overlap off",
        "stage_ms_per_step_serial": {k: v / max(st_serial["executions"], 1) for k, v in st_serial.items()
                                     if k != "executions"},
        "p0_quartets_per_step": int(sum(n0 for _, (_, n0) in counts.items())),
        "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clocks,
        "sum_rule_check": float(result[0] / (p.nelec * (p.nelec - 1) * (float(np.float32(np.pi)) / np.pi) ** 3)),
    }
    line.update(extras)
    if rank == 0:
        if args.e2e_steps > 0:
            dt_e2e, res_e2e = e2e_entry1(p, args.e2e_steps, 1)
            line["e2e"] = {"value": qq_step / dt_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d_bytes(p),
                           "d2h_bytes_per_step": 8 * p.nq, "ms_per_step": dt_e2e * 1e3,
                           "path": "thistle_total_scattering (Entry 1), pinned host inputs, plan set-up included"}
            line["e2e_matches_device"] = bool(np.max(np.abs(res_e2e - result)) <= 1e-12 * np.max(np.abs(result)))
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(p)
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
