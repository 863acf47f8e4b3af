"""Electron scattering (types 5 and 6): I_e - 2 Ine + Inn, with the
nuclear-electron term Ine of nuclei_electron_integration
(src/Integrals.f90:2493-2596) and the nuclear-nuclear sinc sum Inn
(src/main_calculation.f90:302-311).  The oracle pins are CPU tests; the
CUDA path is checked against the oracle on the GPU."""
import numpy as np
import pytest

from thistle_b200 import inputs as I

from conftest import rel_err

SP15 = (float(np.float32(np.pi)) / np.pi) ** 1.5
TOL = 1e-10


def _zn(p):
    # neutral: the nuclear charges add up to the electron count
    k = len(p.atoms)
    z = np.full(k, p.nelec // k, dtype=np.float64)
    z[0] += p.nelec - z.sum()
    return z


@pytest.mark.parametrize("cfg", [1, 2])
def test_oracle_nuclear_sum_rule(oracle, cfg):
    """q -> 0: the AO density integrates to N, so Ine(0) = sum Zn N (pi_sp/pi)^1.5."""
    p = I.CONFIGS[cfg]()
    zn = _zn(p)
    ine = oracle.nuclear(p, zn)
    assert abs(ine[0] / (zn.sum() * p.nelec * SP15) - 1) < 1e-9


def test_oracle_elastic_electron_vanishes_at_zero_q(oracle):
    """Type 6 at q -> 0: N^2 - 2 Z N + Z^2 = 0 for a neutral molecule (up to the
    reference's single-precision pi in the prefactors)."""
    p = I.config2_diatomic()
    zn = _zn(p)
    r = oracle.electron(p, 6, zn)
    n = p.nelec
    assert abs(r[0]) < 1e-6 * n * n


def test_oracle_bessel_sum_upward_matches_accurate_at_moderate_qh(oracle):
    """BesselSum's upward recurrence (the reference's arithmetic) against the
    stable generator where qH is not small against the order."""
    p = I.config2_diatomic()
    zn = _zn(p)
    q = np.linspace(4.0, 8.0, 5)
    ref = oracle.nuclear(p, zn, bessel_mode=0, q=q)
    acc = oracle.nuclear(p, zn, bessel_mode=1, q=q)
    assert np.max(rel_err(ref, acc)) < 1e-6


def _close(got, ref, scale):
    # I_e - 2 Ine + Inn cancels to roundoff of its terms (size ~scale) at small
    # q: relative tolerance plus an absolute floor at that scale
    return np.all(np.abs(got - ref) <= TOL * np.abs(ref) + 1e-12 * scale)


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [1, 2])
def test_plan_nuclear_matches_oracle(oracle, cfg):
    from thistle_b200 import main_calculation as MC
    p = I.CONFIGS[cfg]()
    zn = _zn(p)
    with MC.ScatteringPlan.from_problem(p, MC.ELASTIC_J0) as pl:
        got = pl.nuclear(zn, p.atoms)
    ref = oracle.nuclear(p, zn, bessel_mode=1)
    assert np.max(rel_err(got, ref)) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [1, 2])
@pytest.mark.parametrize("type_", [5, 6])
def test_entry1_electron_matches_oracle(oracle, cfg, type_):
    from thistle_b200 import main_calculation as MC
    p = I.CONFIGS[cfg]()
    zn = _zn(p)
    got = MC.scattering(p, type_, Zn=zn)
    ref = oracle.electron(p, type_, zn, bessel_mode=1)
    assert _close(got, ref, (p.nelec + zn.sum()) ** 2)


@pytest.mark.gpu
def test_nuclear_term_follows_the_geometry(oracle):
    """Moving the atoms (and their Gaussians) moves the nuclear term with them."""
    from thistle_b200 import main_calculation as MC
    p = I.config2_diatomic()
    zn = _zn(p)
    moved = p.with_geometry(p.atoms * 1.05)
    with MC.ScatteringPlan.from_problem(p, MC.ELASTIC_J0) as pl:
        pl.set_centres(moved.xx, moved.yy, moved.zz)
        got = pl.nuclear(zn, moved.atoms)
    assert np.max(rel_err(got, oracle.nuclear(moved, zn))) < TOL


@pytest.mark.gpu
def test_electron_rejects_mismatched_nuclei():
    from thistle_b200 import main_calculation as MC
    from thistle_b200._abi import ThistleError
    p = I.config1_h2()
    with pytest.raises((ThistleError, ValueError)):
        MC.scattering(p, 6, Zn=np.ones(3))


@pytest.mark.gpu
def test_plan_nuclear_rejects_short_geometry():
    from thistle_b200 import main_calculation as MC
    p = I.config1_h2()
    with MC.ScatteringPlan.from_problem(p, MC.ELASTIC_J0) as pl:
        with pytest.raises(ValueError):
            pl.nuclear(np.ones(2), p.atoms[:1])
