"""Host-side input generation: orthonormal MOs, 2-RDM symmetries and traces."""
import numpy as np

from thistle_b200 import inputs as I


def test_q_grid_replaces_zero():
    q = I.q_grid(10.0, 100)
    assert q[0] == 1e-10 and q[-1] == 10.0 and q.size == 100


def test_mos_orthonormal_in_ao_overlap():
    p = I.config2_diatomic()
    S = I.overlap(p.ga, p.l, p.m, p.n, p.xx, p.yy, p.zz)
    np.testing.assert_allclose(p.mmod @ S @ p.mmod.T, np.eye(p.nmo), atol=1e-10)


def test_overlap_of_normalised_primitives_is_one():
    p = I.config1_h2()
    S = I.overlap(p.ga, p.l, p.m, p.n, p.xx, p.yy, p.zz)
    nrm = I.primitive_norms(p.ga, p.l, p.m, p.n)
    np.testing.assert_allclose(np.diag(S) * nrm ** 2, 1.0, rtol=1e-12)


def test_rdm2_symmetries_trace_and_psd():
    rng = np.random.default_rng(0)
    G = I.rdm2_dense(rng, 5, 6)
    np.testing.assert_allclose(G, G.transpose(2, 3, 0, 1), atol=1e-14)
    np.testing.assert_allclose(G, G.transpose(1, 0, 3, 2), atol=1e-14)
    assert abs(np.einsum('aabb->', G) - 30) < 1e-10
    w = np.linalg.eigvalsh(G.reshape(25, 25))
    assert w.min() > -1e-10 * w.max()
    S = I.rdm2_sparse(rng, 8, 6, 0.05)
    frac = np.count_nonzero(S) / S.size
    assert 0.02 < frac < 0.2
    assert abs(np.einsum('aabb->', S) - 30) < 1e-10


def test_config_sizes_match_survey():
    p1 = I.config1_h2()
    assert (p1.ngto, p1.ng, p1.nmo, p1.nq) == (14, 10, 4, 100)
    p2 = I.config2_diatomic()
    assert (p2.ngto, p2.ng, p2.nmo, p2.mat.shape[0], p2.nq) == (42, 20, 10, 10000, 200)
    n = p2.nelec
    assert abs(p2.total[(p2.mat[:, 0] == p2.mat[:, 1]) & (p2.mat[:, 2] == p2.mat[:, 3])].sum() - n * (n - 1)) < 1e-9


def test_onerdm_trace():
    p = I.config2_diatomic()
    assert abs(np.trace(p.onerdm) - p.nelec) < 1e-10


def test_with_geometry_moves_centres():
    p = I.config1_h2()
    q = p.with_geometry(p.atoms + 1.0)
    np.testing.assert_allclose(q.zz - p.zz, 1.0)
    assert q.mat is p.mat
