"""The MO -> primitive transform on the FP64 tensor cores against the
oracle's pair density (GPU tests): the whole pair density rho of total
plans (the per-quartet ztot of src/Integrals.f90:109-127, 5163 for every
pair of function pairs) and the AO density Z of elastic plans
(variables_elastic, src/Variables.f90:1199-1217).  Tolerance 1e-12 of the
largest element (FP64 sums of a few thousand terms in another order)."""
import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("cfg", [1, 2, 5])
def test_pair_density_matches_oracle(oracle, cfg):
    p = I.CONFIGS[cfg]()
    with MC.ScatteringPlan.from_problem(p, MC.TOTAL_J0) as pl:
        rho = pl.density()
    ref = oracle.pair_density(p)
    assert rho.shape == ref.shape
    assert _rel(rho, ref) < 1e-12


def test_pair_density_uneven_molecule(oracle):
    """A 12-atom molecule of the uneven batch (21 MOs, sparse 2-RDM)."""
    p = I.config4_batch(5)[4]
    with MC.ScatteringPlan.from_problem(p, MC.TOTAL_J0) as pl:
        rho = pl.density()
    assert _rel(rho, oracle.pair_density(p)) < 1e-12


@pytest.mark.parametrize("cfg", [1, 2])
def test_ao_density_matches_variables_elastic(cfg):
    p = I.CONFIGS[cfg]()
    with MC.ScatteringPlan.from_problem(p, MC.ELASTIC_J0) as pl:
        Z = pl.density()
    k = p.onerdm.shape[0]
    C1 = p.mmod[:k]
    D = 0.5 * (p.onerdm + p.onerdm.T)
    ref = C1.T @ D @ C1
    assert _rel(Z, ref) < 1e-12
