"""Geometry batches: one plan holding several geometries of its basis, every
stage launched once for all of them, optionally replayed from a CUDA graph,
and the batch-size / q-tile autotuner."""
import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC

pytestmark = pytest.mark.gpu


def _geometries(p, n, seed=3, sigma=0.1):
    rng = np.random.default_rng(seed)
    geos = [p.atoms] + [p.atoms + sigma * rng.standard_normal(p.atoms.shape) for _ in range(n - 1)]
    return [p.with_geometry(R) for R in geos]


def _xyz(probs):
    return np.stack([np.stack([q.xx, q.yy, q.zz], axis=1) for q in probs])


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_single_geometries(use_graph):
    p = I.config2_diatomic()
    probs = _geometries(p, 4)
    v = np.random.default_rng(1).normal(size=(4, p.nq))
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        singles, grads = [], []
        for q, vv in zip(probs, v):
            pl.set_centres(q.xx, q.yy, q.zz)
            singles.append(pl.execute())
            grads.append(pl.vjp(vv))
        pl.set_batch(4)
        pl.use_graph(use_graph)
        pl.set_centres_batch(_xyz(probs))
        out = pl.execute_batch()
        g = pl.vjp_batch(v)
        out2 = pl.execute_batch()   # graph replay (or plain re-run): identical
        g2 = pl.vjp_batch(v)
    for k in range(4):
        assert _rel(out[k], singles[k]) < 1e-12
        assert _rel(g[k], grads[k]) < 1e-11
    assert np.array_equal(out, out2) and np.array_equal(g, g2)


def test_batch_graph_and_plain_agree_bitwise():
    p = I.config1_h2()
    probs = _geometries(p, 3, seed=5)
    res = []
    for use_graph in (False, True):
        with MC.ScatteringPlan.from_problem(p, 1) as pl:
            pl.set_batch(3)
            pl.use_graph(use_graph)
            pl.set_centres_batch(_xyz(probs))
            res.append((pl.execute_batch(), pl.vjp_batch(np.ones((3, p.nq)))))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_autotune_picks_a_batch():
    p = I.config2_diatomic()
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        pl.use_graph(True)
        g, qt, gps = pl.autotune_batch(8)
        assert g in (1, 2, 4, 8) and gps > 0 and 64 <= qt <= p.nq
        assert pl.stage2_tile() in ((2, 4), (2, 8), (1, 4), (1, 8))
        probs = _geometries(p, g, seed=9)
        pl.set_centres_batch(_xyz(probs))
        out = pl.execute_batch()
    ref = MC.scattering(probs[-1], 1)
    assert _rel(out[-1], ref) < 1e-12


@pytest.mark.parametrize("kind", [MC.TOTAL_J0, MC.TOTAL_J2])
def test_stage2_pair_tiles_agree(kind):
    """Every stage-2 pair tile (quartets per lane x warps per block) sums the
    same quartets at the same points: results agree to rounding, and each
    tile is reproducible run to run.  The 3-atom s/p/d case has polynomial
    orders (LB <= 8) and, for j2, recurrence orders (9, 10)."""
    p = I.config3_ab6(nq=200, natoms=3)
    with MC.ScatteringPlan.from_problem(p, kind) as pl:
        assert pl.stage2_tile() == (2, 4)
        ref = pl.execute()
        for k, nw in ((2, 8), (1, 4), (1, 8), (2, 4)):
            pl.set_stage2_tile(k, nw)
            assert pl.stage2_tile() == (k, nw)
            a = pl.execute()
            assert _rel(a, ref) < 1e-13
            assert np.array_equal(a, pl.execute())
        with pytest.raises(MC.ThistleError):
            pl.set_stage2_tile(3, 4)
        with pytest.raises(MC.ThistleError):
            pl.set_stage2_tile(2, 6)


@pytest.mark.parametrize("kind", [MC.TOTAL_J0, MC.ELASTIC_J0, MC.TOTAL_J2])
def test_stage_overlap_is_exact(kind):
    """Stage 2 of a class overlapping the later classes' stage 1 (per-class
    visiting-order sorts) gives bit for bit the result of the serial order."""
    p = I.config3_ab6(nq=200, natoms=3)
    with MC.ScatteringPlan.from_problem(p, kind) as pl:
        on = pl.execute()
        pl.set_pipeline(False)
        off = pl.execute()
        pl.set_pipeline(True)
        again = pl.execute()
    assert np.array_equal(on, off) and np.array_equal(on, again)
