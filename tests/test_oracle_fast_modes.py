"""The oracle's two faster evaluation modes, used to generate the full-size
fixtures, against its reference-order modes (CPU):

* summed pair density (``oracle.pair_density``) in place of the per-quartet
  contraction of the 2-RDM rows (the reference's dgemm pair,
  src/Integrals.f90:109-127);
* the aligned intensity as the weighted five-loop sum with Hermite densities
  (``oracle.aligned_list``) in place of all ng^4 ordered quartets
  (src/Integrals.f90:1425-1573).

Also: the committed large fixtures match the regenerated inputs, the
stratified AB6 sample regenerates identically, and the reference's 2-RDM
files parse to the committed rows (when a reference checkout is present).
"""
import os
import sys

import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC

from conftest import rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
import make_golden_large as MG  # noqa: E402


@pytest.mark.parametrize("cfg", [1, 2])
@pytest.mark.parametrize("type_", [1, 7])
def test_pair_density_mode_matches_row_contraction(oracle, cfg, type_):
    p = I.CONFIGS[cfg]()
    rho = oracle.pair_density(p)
    a = oracle.scattering(p, type_, nthreads=4)
    b = oracle.scattering(p, type_, rho=rho, nthreads=4)
    assert np.max(rel_err(b, a)) < 1e-12


def test_pair_density_mode_ab6_sample(oracle):
    p = I.config3_ab6()
    qs = oracle.enum_quartets(p.ng)
    idx = MG.stratified_sample(p, qs, 0.0, 3, 11)
    sub = qs[idx]
    rho = oracle.pair_density(p)
    a = oracle.scattering(p, 1, quartets=sub, bessel_mode=1, nthreads=8)
    b = oracle.scattering(p, 1, quartets=sub, rho=rho, bessel_mode=1, nthreads=8)
    assert np.max(rel_err(b, a)) < 1e-10


def test_pair_density_is_symmetric(oracle):
    p = I.config2_diatomic()
    rho = oracle.pair_density(p)
    assert np.max(np.abs(rho - rho.T)) <= 1e-14 * np.max(np.abs(rho))


def test_aligned_list_matches_all_ordered_quartets(oracle):
    p = I.config1_h2()
    qal = oracle.qcoord3()[::37]
    re, _ = oracle.aligned(p, qal)
    assert np.max(rel_err(oracle.aligned_list(p, qal), re)) < 1e-12
    p = I.config2_diatomic()
    qal = np.random.default_rng(5).uniform(-6, 6, size=(12, 3))
    re, _ = oracle.aligned(p, qal)
    got = oracle.aligned_list(p, qal, rho=oracle.pair_density(p))
    assert np.max(rel_err(got, re)) < 1e-12


def test_large_fixtures_match_regenerated_inputs():
    g = np.load(os.path.join(GOLD, "golden_cfg5.npz"))
    np.testing.assert_array_equal(g["q"], I.config5_fit().q)
    g = np.load(os.path.join(GOLD, "golden_ab6.npz"))
    np.testing.assert_array_equal(g["q"], I.config3_ab6().q)
    g = np.load(os.path.join(GOLD, "golden_cfg4.npz"))
    mols = I.config4_batch(MG.CFG4_MOLECULES)
    np.testing.assert_array_equal(g["natoms"], [len(p.atoms) for p in mols])
    g = np.load(os.path.join(GOLD, "golden_cfg5_adjoint.npz"))
    base = I.config5_fit()
    np.testing.assert_array_equal(g["geoms"], I.config5_geometries(base, 3)[1:])
    g = np.load(os.path.join(GOLD, "golden_cfg5_aligned.npz"))
    assert g["index"].size >= 2000 and g["index"][-1] < 64 ** 3


def test_ab6_sample_regenerates(oracle):
    p = I.config3_ab6()
    qs = oracle.enum_quartets(p.ng)
    idx = MG.stratified_sample(p, qs, 0.01, 40, 20261204)
    g = np.load(os.path.join(GOLD, "golden_ab6_sample.npz"))
    np.testing.assert_array_equal(idx, g["index"])
    # every shell-type stratum is present
    assert np.unique(MG.strata(p, qs[idx])).size == np.unique(MG.strata(p, qs)).size


@pytest.mark.skipif(not os.path.isdir(MG.REF), reason="no reference checkout")
def test_reference_2rdm_files_parse_to_committed_rows():
    g = np.load(os.path.join(GOLD, "golden_refrdm.npz"))
    for key, rel, reader, nelec, _ in MG.REF_RDMS:
        fn = MC.read_twordm if reader == "rows" else MC.read_twordm_listing
        mat, total = fn(os.path.join(MG.REF, rel))
        np.testing.assert_array_equal(mat, g[f"{key}_mat"])
        np.testing.assert_array_equal(total, g[f"{key}_total"])
        tr = total[(mat[:, 0] == mat[:, 1]) & (mat[:, 2] == mat[:, 3])].sum()
        assert abs(tr - nelec * (nelec - 1)) < 1e-6 * nelec * nelec
