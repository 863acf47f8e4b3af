"""Adjoint of total j0 with respect to the nuclear coordinates: the library's
vector-Jacobian product against central finite differences (h = 1e-4 bohr)
of the GPU forward and of the oracle, translation invariance, and the
torch.autograd binding."""
import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC
from oracle import oracle as O

pytestmark = pytest.mark.gpu

H = 1e-4


def _fd(p, plan, v, coords, forward=None, h=H):
    out = []
    for a, ax in coords:
        vals = []
        for sgn in (1, -1):
            R = p.atoms.copy()
            R[a, ax] += sgn * h
            if forward is None:
                q = p.with_geometry(R)
                plan.set_centres(q.xx, q.yy, q.zz)
                vals.append(float(v @ plan.execute()))
            else:
                vals.append(float(v @ forward(p.with_geometry(R))))
        out.append((vals[0] - vals[1]) / (2 * h))
    return np.array(out)


def _vjp_atoms(p, plan, v):
    plan.set_centres(p.xx, p.yy, p.zz)
    return MC.atom_gradient(p, plan.vjp(v))


@pytest.mark.parametrize("cfg", [1, 2])
def test_vjp_matches_central_differences(cfg):
    p = I.config1_h2() if cfg == 1 else I.config2_diatomic()
    rng = np.random.default_rng(cfg)
    v = rng.normal(size=p.nq)
    coords = [(a, ax) for a in range(p.atoms.shape[0]) for ax in range(3)]
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        g = _vjp_atoms(p, pl, v)
        fd = _fd(p, pl, v, coords)
    got = np.array([g[a, ax] for a, ax in coords])
    scale = np.max(np.abs(fd))
    assert scale > 0
    assert np.max(np.abs(got - fd)) < 1e-6 * scale, (got, fd)


def test_vjp_against_oracle_differences():
    """The reference FP64 gradient: central differences of the oracle's I(q)."""
    p = I.config1_h2()
    v = np.random.default_rng(3).normal(size=p.nq)
    coords = [(0, 2), (1, 0), (1, 2)]
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        g = _vjp_atoms(p, pl, v)
    fd = _fd(p, None, v, coords, forward=lambda q: O.scattering(q, 1))
    got = np.array([g[a, ax] for a, ax in coords])
    assert np.max(np.abs(got - fd)) < 1e-6 * np.max(np.abs(fd))


def test_vjp_translation_invariance_and_ab6_sample():
    """AB6 (p and d shells, 7 atoms): the atom gradients sum to zero and
    three coordinates agree with central differences.  The step is 1e-5 bohr
    here: moving the central atom by 1e-4 carries a quartet across the
    reference's P = Q threshold (|H| = cutoffcentre), a jump of the
    reference's own I(q) that a difference quotient cannot tell from a slope."""
    p = I.config3_ab6(nq=120)
    v = np.random.default_rng(7).normal(size=p.nq)
    coords = [(0, 0), (1, 0), (3, 2)]
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        g = _vjp_atoms(p, pl, v)
        fd = _fd(p, pl, v, coords, h=1e-5)
    assert np.max(np.abs(g.sum(axis=0))) < 1e-9 * np.max(np.abs(g))
    got = np.array([g[a, ax] for a, ax in coords])
    assert np.max(np.abs(got - fd)) < 1e-6 * np.max(np.abs(g)), (got, fd)


def test_vjp_is_deterministic_and_rejects_other_types():
    p = I.config2_diatomic()
    v = np.ones(p.nq)
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        a = pl.vjp(v)
        b = pl.vjp(v)
    assert np.array_equal(a, b)
    with MC.ScatteringPlan.from_problem(p, 2) as pl:
        with pytest.raises(MC.ThistleError):
            pl.vjp(v)


def test_autograd_function():
    import torch
    from thistle_b200.autograd import intensity
    p = I.config2_diatomic()
    v = np.random.default_rng(11).normal(size=p.nq)
    with MC.ScatteringPlan.from_problem(p, 1) as pl:
        R = torch.tensor(p.atoms, dtype=torch.float64, device="cuda", requires_grad=True)
        Iq = intensity(R, pl, p.atom_of)
        assert Iq.is_cuda
        assert np.allclose(Iq.detach().cpu().numpy(), pl.execute(), rtol=0, atol=0)
        (Iq * torch.as_tensor(v, device="cuda")).sum().backward()
        ref = _vjp_atoms(p, pl, v)
    assert R.grad.is_cuda
    assert np.allclose(R.grad.cpu().numpy(), ref, rtol=1e-14, atol=0)


def test_batched_autograd_on_device_matches_per_geometry_and_oracle_differences():
    """Configuration 5: a batch of displaced ring geometries through the
    device-resident batched binding, against the per-geometry plan path (the
    same numbers to rounding) and against central differences of the oracle
    at six coordinates of two geometries (committed fixture, h = 1e-4)."""
    import os
    import torch
    from thistle_b200.autograd import intensity_batch
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_cfg5_adjoint.npz"))
    base = I.config5_fit()
    geoms = np.concatenate([g["geoms"], I.config5_geometries(base, 4)[3:]])  # 3 geometries
    v = np.concatenate([g["v"], np.random.default_rng(4).normal(size=(1, base.nq))])
    with MC.ScatteringPlan.from_problem(base, 1) as pl:
        R = torch.tensor(geoms, dtype=torch.float64, device="cuda", requires_grad=True)
        Iq = intensity_batch(R, pl, base.atom_of)
        assert Iq.shape == (3, base.nq) and Iq.is_cuda
        (Iq * torch.as_tensor(v, device="cuda")).sum().backward()
        got_I = Iq.detach().cpu().numpy()
        got_g = R.grad.cpu().numpy()
    with MC.ScatteringPlan.from_problem(base, 1) as single:
        for k in range(3):
            pk = base.with_geometry(geoms[k])
            single.set_centres(pk.xx, pk.yy, pk.zz)
            ref_I = single.execute()
            ref_g = MC.atom_gradient(pk, single.vjp(v[k]))
            assert np.max(np.abs(got_I[k] - ref_I)) < 1e-12 * np.max(np.abs(ref_I))
            assert np.max(np.abs(got_g[k] - ref_g)) < 1e-10 * np.max(np.abs(ref_g))
    for k in range(2):
        fd = g["fd"][k]
        got = np.array([got_g[k, a, ax] for a, ax in g["coords"]])
        assert np.max(np.abs(got - fd)) < 2e-6 * np.max(np.abs(fd)), (got, fd)
