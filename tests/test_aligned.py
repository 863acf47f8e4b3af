"""Aligned (non-averaged) total intensity, tot_integration_aligned
(src/Integrals.f90:1425-1573): the QCOORD3 grid on the host, and the GPU
q-vector kernel against the oracle's all-ng^4 ordered sum."""
import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC
from oracle import oracle as O


def test_qcoord3_matches_the_reference_routine():
    """The library's QCOORD3 grid (host code, no GPU) equals the oracle's restatement."""
    got = MC.qcoord3()
    ref = O.qcoord3()
    assert got.shape == (3131, 3)
    assert np.array_equal(got, ref)
    # the origin slot; the hexagon points lie on the Ewald sphere |(qx, qy, k0 - qz)| = k0
    k0 = 10.583544175
    assert np.all(got[0] == 1e-10)
    hexa = got[2:7]
    assert np.allclose(np.linalg.norm(np.stack([hexa[:, 0], hexa[:, 1], k0 - hexa[:, 2]], 1), axis=1), k0,
                       rtol=1e-13)


def _check(re, im, ref_re, ref_im, tol=1e-10):
    scale = np.max(np.abs(ref_re))
    err = np.abs(re - ref_re) / np.maximum(np.abs(ref_re), 1e-12 * scale)
    assert np.max(err) < tol, np.max(err)
    # the ordered sum is real: the oracle's imaginary part is rounding noise
    assert np.max(np.abs(ref_im)) < 1e-12 * scale
    assert np.all(im == 0.0)


@pytest.mark.gpu
def test_aligned_h2_qcoord3_grid():
    p = I.config1_h2()
    qv = MC.qcoord3()[::9]
    re, im = MC.aligned(p, qv)
    ref_re, ref_im = O.aligned(p, qv)
    _check(re, im, ref_re, ref_im)


@pytest.mark.gpu
def test_aligned_random_vectors_diatomic():
    """p and d shells, all LLmax classes of configuration 2, random directions."""
    p = I.config2_diatomic()
    rng = np.random.default_rng(5)
    qv = rng.normal(size=(40, 3))
    qv *= (rng.uniform(0.05, 6.0, size=40) / np.linalg.norm(qv, axis=1))[:, None]
    re, im = MC.aligned(p, qv)
    ref_re, ref_im = O.aligned(p, qv)
    _check(re, im, ref_re, ref_im)


@pytest.mark.gpu
def test_aligned_entry1_type3():
    """Entry 1 with type 3: the QCOORD3 grid, |q| in q_abs, Re I in result."""
    p = I.config1_h2()
    dummy = np.ones(3131)
    q_abs, res = MC.total_scattering_calculation(
        3, None, p.atoms, 0, 0, 1, p.ngto, p.ng, p.ga, p.l, p.m, p.n, p.xx, p.yy, p.zz, p.mmod, dummy, 3131,
        p.group, p.cutoffz, p.cutoffmd, p.cutoffcentre, mat=p.mat, total=p.total)
    grid = MC.qcoord3()
    assert np.allclose(q_abs, np.linalg.norm(grid, axis=1), rtol=1e-15)
    re, _ = MC.aligned(p, grid)
    assert np.array_equal(res, re)


@pytest.mark.gpu
def test_aligned_forward_direction_is_the_total_j0_limit():
    """At q -> 0 every Bessel and phase factor is 1: aligned = total j0 there."""
    p = I.config2_diatomic()
    qv = np.array([[1e-10, 1e-10, 1e-10]])
    re, _ = MC.aligned(p, qv)
    tot = MC.scattering(p, MC.TOTAL_J0, q=np.array([np.sqrt(3) * 1e-10]))
    assert abs(re[0] - tot[0]) < 1e-10 * abs(tot[0])
