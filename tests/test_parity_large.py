"""Full-size parity of the CUDA path with the oracle (GPU tests).

The oracle's outputs for the large configurations are committed fixtures
(tests/golden/make_golden_large.py): the whole AB6 I(q) (11.9 M group
quartets x 500 q) for total j0, elastic j0 and total j2, a 1 % sample of
it stratified by shell types through the explicit-quartet entry, the
6-atom ring (configuration 5) forward, its adjoint against central
differences of the oracle at two displaced geometries, its aligned intensity
on a 2002-vector slice of the 64^3 Cartesian grid, eight molecules of the
uneven batch (configuration 4, including a 12-atom one) as one molecule
batch, and the reference's own 2-RDM files.  Inputs are regenerated from the
seeded generators.

Tolerance: 1e-10 relative per q point (floor 1e-12 of max |I| where I
crosses zero).  Total j2 is a P2-weighted orientational average, a signed
sum whose terms are bounded by those of total j0 and which is only 1e-3 to
1e-2 of it on these molecules (it changes sign, and on the octahedral AB6
cubic symmetry cancels most of it); its rounding error scales with the j0
intensity, so a j2 point is held to 1e-10 |I_j2(q)| + 1e-12 |I_j0(q)|.  The
adjoint: 2e-6 of the largest difference quotient (the central difference's
own truncation error at h = 1e-4 bohr).
"""
import os
import sys

import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10
J0_SCALE = 1e-12  # j2: |error| <= TOL |I_j2| + J0_SCALE |I_j0| at each q
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
SP = (float(np.float32(np.pi)) / np.pi) ** 3
sys.path.insert(0, GOLD)
import make_golden_large as MG  # noqa: E402


def gold(name):
    return np.load(os.path.join(GOLD, name))


def check(got, ref, tol=TOL, floor=1e-12, j0=None):
    assert np.all(np.isfinite(got))
    if j0 is not None:
        excess = np.abs(got - ref) - (tol * np.abs(ref) + J0_SCALE * np.abs(j0))
        assert np.max(excess) <= 0.0, float(np.max(np.abs(got - ref) / (np.abs(ref) + 1e-300)))
        return
    err = float(np.max(rel_err(got, ref, floor=floor)))
    assert err < tol, err


# ---------------------------------------------------------------- AB6 ------
@pytest.fixture(scope="module")
def ab6():
    return I.config3_ab6()


@pytest.mark.parametrize("type_", [1, 2, 7])
def test_ab6_full_intensity_vs_oracle(ab6, type_):
    """Every quartet class and (LK, side) sub-range of the plan's own
    execution (split contracted-side stage 1 included) at full size."""
    g = gold("golden_ab6.npz")
    np.testing.assert_array_equal(ab6.q, g["q"])
    with MC.ScatteringPlan.from_problem(ab6, type_) as pl:
        got = pl.execute()
    check(got, g[f"type{type_}"], j0=g["type1"] if type_ == 7 else None)
    if type_ == 1:
        # the reference's own Bessel start where it has converged (qH <= 70)
        check(got[g["ref_mask"]], g["type1_ref"])
        assert abs(got[0] / (ab6.nelec * (ab6.nelec - 1) * SP) - 1) < 1e-10


@pytest.mark.parametrize("type_", [1, 2, 7])
def test_ab6_stratified_sample_vs_oracle(ab6, type_):
    """1 % of every shell-type stratum (at least 40 quartets each), through
    the explicit-quartet entry point."""
    g = gold("golden_ab6_sample.npz")
    qs = MG.O.enum_quartets(ab6.ng)[g["index"]]
    assert qs.shape[0] >= 0.01 * 11_920_622
    with MC.ScatteringPlan.from_problem(ab6, type_) as pl:
        got = pl.execute_quartets(qs[:, :4])
    check(got, g[f"type{type_}"], j0=g["type1"] if type_ == 7 else None)


# ------------------------------------------------------- configuration 5 ---
@pytest.fixture(scope="module")
def ring():
    return I.config5_fit()


@pytest.mark.parametrize("type_", [1, 2, 7])
def test_ring_full_intensity_vs_oracle(ring, type_):
    g = gold("golden_cfg5.npz")
    np.testing.assert_array_equal(ring.q, g["q"])
    with MC.ScatteringPlan.from_problem(ring, type_) as pl:
        got = pl.execute()
    check(got, g[f"type{type_}"], j0=g["type1"] if type_ == 7 else None)
    if type_ == 1:
        check(got[g["ref_mask"]], g["type1_ref"])


def test_ring_batched_adjoint_vs_oracle_differences(ring):
    """vjp over a two-geometry batch against central differences of the
    oracle's I(q) (h = 1e-4 bohr) at six coordinates per geometry."""
    g = gold("golden_cfg5_adjoint.npz")
    geoms, v, coords, fd = g["geoms"], g["v"], g["coords"], g["fd"]
    with MC.ScatteringPlan.from_problem(ring, 1) as pl:
        pl.set_batch(2)
        xyz = np.stack([np.stack([ring.with_geometry(R).xx, ring.with_geometry(R).yy,
                                  ring.with_geometry(R).zz], axis=1) for R in geoms])
        pl.set_centres_batch(xyz)
        grads = pl.vjp_batch(v)
    for k in range(2):
        ga = MC.atom_gradient(ring.with_geometry(geoms[k]), grads[k])
        got = np.array([ga[a, ax] for a, ax in coords])
        scale = np.max(np.abs(fd[k]))
        assert scale > 0
        assert np.max(np.abs(got - fd[k])) < 2e-6 * scale, (got, fd[k])


def test_ring_aligned_64cubed_grid_vs_oracle(ring):
    """The aligned intensity on all 262 144 vectors of the 64^3 grid, checked
    on a strided slice of 2002 vectors."""
    g = gold("golden_cfg5_aligned.npz")
    grid = I.config5_aligned_grid()
    assert grid.shape == (64 ** 3, 3)
    re, im = MC.aligned(ring, grid)
    assert np.all(im == 0.0)
    check(re[g["index"]], g["re"])


# ------------------------------------------------------- configuration 4 ---
@pytest.mark.parametrize("type_", [1, 2, 7])
def test_uneven_molecule_batch_vs_oracle(type_):
    g = gold("golden_cfg4.npz")
    mols = I.config4_batch(MG.CFG4_MOLECULES)
    assert max(len(p.atoms) for p in mols) == 12
    plans = [MC.ScatteringPlan.from_problem(p, type_) for p in mols]
    try:
        with MC.MoleculeBatch(plans) as b:
            b.use_graph(True)
            out = b.execute()
    finally:
        for pl in plans:
            pl.close()
    for k, row in enumerate(out):
        check(row, g[f"type{type_}"][k], j0=g["type1"][k] if type_ == 7 else None)


# ------------------------------------------- the reference's own 2-RDMs ----
@pytest.mark.parametrize("key", [r[0] for r in MG.REF_RDMS])
def test_reference_2rdm_files_vs_oracle(key):
    g = gold("golden_refrdm.npz")
    spec = {r[0]: r for r in MG.REF_RDMS}[key]
    p = MG.refrdm_problem(key, g[f"{key}_mat"], g[f"{key}_total"], spec[3], spec[4])
    for type_ in (1, 7):
        got = MC.scattering(p, type_)
        check(got, g[f"{key}_type{type_}"], j0=g[f"{key}_type1"] if type_ == 7 else None)
        if type_ == 1:
            # trace of the file's 2-RDM at q -> 0: N(N-1) (182 for the HF file)
            m = g[f"{key}_mat"]
            tr = g[f"{key}_total"][(m[:, 0] == m[:, 1]) & (m[:, 2] == m[:, 3])].sum()
            assert abs(got[0] / (tr * SP) - 1) < 1e-10
            if key == "hf":
                assert abs(tr - 182.0) < 1e-12


# ------------------------------------------------ documented known answer --
def test_docs_form_factor_through_entry1():
    """docs/src/kernels.md:76-79: one s quartet at H = 1 bohr with
    zcontr + zcontr2 = 0.5 gives F(mu) = 0.5 j0(mu * 0.529177) =
    [0.49976668, 0.49790243] at mu = [0.1, 0.3].  Two s primitives (exponent
    1) at x = 0 and x = 1 bohr, identity MO coefficients and the single 2-RDM
    row (1,1,2,2) = 1 make rho(11, 22) = 0.5 the only nonzero pair density,
    so Entry 1 returns the loop-4 quartet (1,1,2,2): I = 2 F E12_11 E12_22."""
    b = 0.529177210903
    mu = np.array([0.1, 0.3])
    q = mu * b
    ga = np.array([1.0, 1.0])
    z3 = np.zeros(2, np.int32)
    xx = np.array([0.0, 1.0])
    zero = np.zeros(2)
    _, I_q = MC.total_scattering_calculation(
        1, None, None, 0, 0, 0, 2, 2, ga, z3, z3, z3, xx, zero, zero, np.eye(2), q, 2,
        np.array([1, 2], np.int32), 1e-15, 1e-20, 1e-3,
        mat=np.array([[1, 1, 2, 2]], np.int32), total=np.array([1.0]))
    pi_sp = float(np.float32(np.pi))
    e12 = (pi_sp / 2.0) ** 1.5 * np.exp(-q * q / 8.0)
    f = I_q / (2.0 * e12 * e12)
    np.testing.assert_array_equal(np.round(f, 8), [0.49976668, 0.49790243])
