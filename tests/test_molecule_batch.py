"""Molecule batches: plans of different molecules and basis sizes executed
together -- stage 2 as one persistent launch over every (plan, class, block)
item, the other stages one launch per kernel shape (optionally replayed from
a CUDA graph) -- against each plan executed on its own, at every stage-2
pair tile, and the batch tuner."""
import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def molecules():
    # uneven batch of the 2-12 atom generator, the smallest few kept short
    mols = I.config4_batch(nmol=24, nq=256)
    return sorted(mols, key=lambda m: m.ngto)[:6] + [max(mols, key=lambda m: m.ngto)]


@pytest.mark.parametrize("kind", [MC.TOTAL_J0, MC.ELASTIC_J0, MC.TOTAL_J2])
@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_each_plan(molecules, kind, use_graph):
    plans = [MC.ScatteringPlan.from_problem(m, kind) for m in molecules]
    try:
        singles = [p.execute() for p in plans]
        with MC.MoleculeBatch(plans) as b:
            b.use_graph(use_graph)
            out = b.execute()
            again = b.execute()
            info = b.info()
        assert info["plans"] == len(plans) and info["nq"] == sum(p.nq for p in plans)
        assert info["launches"] >= 3
        for o, s in zip(out, singles):
            assert o.shape == s.shape
            assert _rel(o, s) < 1e-12
        for o, a in zip(out, again):
            assert np.array_equal(o, a)
    finally:
        for p in plans:
            p.close()


def test_batch_follows_new_centres(molecules):
    m0, m1 = molecules[0], molecules[1]
    moved = m1.with_geometry(m1.atoms + 0.05)
    plans = [MC.ScatteringPlan.from_problem(m, MC.TOTAL_J0) for m in (m0, m1)]
    ref = MC.ScatteringPlan.from_problem(moved, MC.TOTAL_J0)
    try:
        with MC.MoleculeBatch(plans) as b:
            b.use_graph(True)
            first = b.execute()
            plans[1].set_centres(moved.xx, moved.yy, moved.zz)
            second = b.execute()
        assert np.array_equal(first[0], second[0])
        assert _rel(second[1], ref.execute()) < 1e-12
        # the plans stay usable on their own after the batch
        assert _rel(plans[1].execute(), second[1]) < 1e-12
    finally:
        for p in plans + [ref]:
            p.close()


def test_batch_rejects_mixed_types(molecules):
    a = MC.ScatteringPlan.from_problem(molecules[0], MC.TOTAL_J0)
    b = MC.ScatteringPlan.from_problem(molecules[1], MC.ELASTIC_J0)
    try:
        with pytest.raises(MC.ThistleError):
            MC.MoleculeBatch([a, b])
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("tile", [(2, 8), (1, 4), (1, 8)])
def test_batch_pair_tiles(molecules, tile):
    plans = [MC.ScatteringPlan.from_problem(m, MC.TOTAL_J2) for m in molecules]
    try:
        singles = [p.execute() for p in plans]
        with MC.MoleculeBatch(plans) as b:
            b.use_graph(True)
            b.set_stage2_tile(*tile)
            assert b.stage2_tile() == tile
            out = b.execute()
            again = b.execute()
        for o, s, a in zip(out, singles, again):
            assert _rel(o, s) < 1e-12
            assert np.array_equal(o, a)
    finally:
        for p in plans:
            p.close()


def test_batch_autotune(molecules):
    plans = [MC.ScatteringPlan.from_problem(m, MC.TOTAL_J0) for m in molecules]
    try:
        singles = [p.execute() for p in plans]
        with MC.MoleculeBatch(plans) as b:
            b.use_graph(True)
            k, nw, mps = b.autotune()
            assert (k, nw) in ((2, 4), (2, 8), (1, 4), (1, 8)) and mps > 0
            assert b.stage2_tile() == (k, nw)
            out = b.execute()
            with pytest.raises(MC.ThistleError):
                b.set_stage2_tile(1, 5)
        for o, s in zip(out, singles):
            assert _rel(o, s) < 1e-12
    finally:
        for p in plans:
            p.close()
