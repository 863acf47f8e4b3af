"""Seeded synthetic inputs in the reference's data layout.

The reference takes a decontracted Cartesian Gaussian basis (one primitive per
basis function, grouped into shells), MO coefficients with the primitive
normalisation folded in, and a sparse 2-RDM list of ``(p, q, r, s, value)``
rows (the ``read_twordm`` format, src/one_rdm.f90:2112-2147).  The drivers
build these from molden files (src/molden_reader_nikola.py:382-429) and put
``q[0] = 1e-10`` when the grid starts at 0 (src/scattering_main_routine.py:186-187).

Nothing here needs a GPU.  The arrays use the reference conventions:

* ``ga, l, m, n, xx, yy, zz`` per primitive function (length ngto);
* ``group`` 1-based shell index per function, functions of a shell contiguous;
* ``mmod`` (nmo, ngto): MO coefficients multiplying *unnormalised* primitives;
* ``mat`` (nmat, 4) int32 1-based MO indices and ``total`` (nmat,) values,
  pair (p,q) on electron 1 and (r,s) on electron 2; sum_{ab} G(a,a,b,b) is
  N(N-1) for orthonormal MOs (the convention of src/HF_NonZero2RM_MO_Coeffs).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# Cartesian component order inside a shell (molden order for d).
_CART = {
    0: [(0, 0, 0)],
    1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
    3: [(3, 0, 0), (0, 3, 0), (0, 0, 3), (1, 2, 0), (2, 1, 0), (2, 0, 1),
        (1, 0, 2), (0, 1, 2), (0, 2, 1), (1, 1, 1)],
    4: [(a, b, 4 - a - b) for a in range(4, -1, -1) for b in range(4 - a, -1, -1)],
}

CUTOFFCENTRE = 1.0e-3   # src/scattering_main_routine.py:174-178
CUTOFFZ = 1.0e-15
CUTOFFMD = 1.0e-20


@dataclass
class Problem:
    """One molecule (or geometry) in the reference's input layout."""
    name: str
    atoms: np.ndarray            # (natoms, 3) bohr
    ga: np.ndarray
    l: np.ndarray
    m: np.ndarray
    n: np.ndarray
    xx: np.ndarray
    yy: np.ndarray
    zz: np.ndarray
    group: np.ndarray            # int32, 1-based
    atom_of: np.ndarray          # int32, 0-based atom of each function
    mmod: np.ndarray             # (nmo, ngto)
    mat: np.ndarray              # (nmat, 4) int32, 1-based
    total: np.ndarray            # (nmat,)
    onerdm: np.ndarray           # (nmo, nmo)
    q: np.ndarray                # (nq,)
    nelec: int
    cutoffz: float = CUTOFFZ
    cutoffmd: float = CUTOFFMD
    cutoffcentre: float = CUTOFFCENTRE
    meta: dict = field(default_factory=dict)

    @property
    def ngto(self) -> int:
        return int(self.ga.size)

    @property
    def ng(self) -> int:
        return int(self.group.max())

    @property
    def nmo(self) -> int:
        return int(self.mmod.shape[0])

    @property
    def nq(self) -> int:
        return int(self.q.size)

    def with_geometry(self, atoms: np.ndarray) -> "Problem":
        """Same basis, MOs and RDMs with the Gaussian centres moved with their atoms."""
        atoms = np.asarray(atoms, dtype=np.float64).reshape(-1, 3)
        p = Problem(**{k: getattr(self, k) for k in self.__dataclass_fields__})
        p.atoms = atoms.copy()
        p.xx = atoms[self.atom_of, 0].copy()
        p.yy = atoms[self.atom_of, 1].copy()
        p.zz = atoms[self.atom_of, 2].copy()
        p.meta = dict(self.meta)
        return p


def q_grid(qmax: float, nq: int) -> np.ndarray:
    """linspace(0, qmax, nq) with q[0] -> 1e-10 as the reference drivers do."""
    q = np.linspace(0.0, qmax, nq)
    if q[0] < 1e-10:
        q[0] = 1e-10
    return q


def geometric(lo: float, hi: float, k: int) -> list:
    if k == 1:
        return [lo]
    return list(lo * (hi / lo) ** (np.arange(k) / (k - 1)))


def build_basis(atoms: np.ndarray, shells_per_atom):
    """Decontracted basis: one group per (atom, l, exponent) shell.

    ``shells_per_atom[a]`` is a list of ``(l, exponent)``.
    """
    ga, L, M, N, X, Y, Z, grp, aof = [], [], [], [], [], [], [], [], []
    g = 0
    for a, shells in enumerate(shells_per_atom):
        for (lsh, alpha) in shells:
            g += 1
            for (i, j, k) in _CART[lsh]:
                ga.append(alpha); L.append(i); M.append(j); N.append(k)
                X.append(atoms[a, 0]); Y.append(atoms[a, 1]); Z.append(atoms[a, 2])
                grp.append(g); aof.append(a)
    f64 = lambda v: np.asarray(v, dtype=np.float64)
    i32 = lambda v: np.asarray(v, dtype=np.int32)
    return f64(ga), i32(L), i32(M), i32(N), f64(X), f64(Y), f64(Z), i32(grp), i32(aof)


def _dfact(k: int) -> float:
    r = 1.0
    while k > 1:
        r *= k
        k -= 2
    return r


def primitive_norms(ga, l, m, n) -> np.ndarray:
    out = np.empty(ga.size)
    for i in range(ga.size):
        a = ga[i]
        lt = l[i] + m[i] + n[i]
        out[i] = ((2 * a / np.pi) ** 0.75 * (4 * a) ** (lt / 2)
                  / np.sqrt(_dfact(2 * l[i] - 1) * _dfact(2 * m[i] - 1) * _dfact(2 * n[i] - 1)))
    return out


def _md_e0(la, lb, PA, PB, a):
    """E^{la,lb}_0 by the Hermite recurrence (vectorised over pairs)."""
    E = {(0, 0): [np.ones_like(PA)]}
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if j == 0:
                prev, P = E[(i - 1, 0)], PA
            else:
                prev, P = E[(i, j - 1)], PB
            new = []
            for t in range(i + j + 1):
                v = np.zeros_like(PA)
                if t >= 1:
                    v = v + a * prev[t - 1]
                if t <= len(prev) - 1:
                    v = v + P * prev[t]
                if t + 1 <= len(prev) - 1:
                    v = v + (t + 1) * prev[t + 1]
                new.append(v)
            E[(i, j)] = new
    return E[(la, lb)][0]


def overlap(ga, l, m, n, xx, yy, zz) -> np.ndarray:
    """AO overlap of unnormalised Cartesian primitives."""
    A = ga[:, None]
    B = ga[None, :]
    p = A + B
    S = (np.pi / p) ** 1.5
    for lax, x in ((l, xx), (m, yy), (n, zz)):
        Px = (A * x[:, None] + B * x[None, :]) / p
        PA = Px - x[:, None]
        PB = Px - x[None, :]
        S = S * np.exp(-A * B / p * (x[:, None] - x[None, :]) ** 2)
        e0 = np.zeros_like(S)
        for la in range(int(lax.max()) + 1):
            for lb in range(int(lax.max()) + 1):
                mask = (lax[:, None] == la) & (lax[None, :] == lb)
                if mask.any():
                    e0[mask] = _md_e0(la, lb, PA[mask], PB[mask], 0.5 / p[mask])
        S = S * e0
    return S


def lowdin_mos(rng, nmo: int, ga, l, m, n, xx, yy, zz) -> np.ndarray:
    """uniform[-1,1] coefficients on normalised primitives, normalisation folded
    in, then symmetric (Loewdin) orthonormalisation in the AO overlap."""
    ngto = ga.size
    c0 = rng.uniform(-1.0, 1.0, size=(nmo, ngto)) * primitive_norms(ga, l, m, n)[None, :]
    S = overlap(ga, l, m, n, xx, yy, zz)
    M = c0 @ S @ c0.T
    w, V = np.linalg.eigh(M)
    Mih = V @ np.diag(w ** -0.5) @ V.T
    return Mih @ c0


def _swap_sym(G: np.ndarray, n: int) -> np.ndarray:
    """Gamma_ijkl = Gamma_klij = Gamma_jilk on the (n*n, n*n) pair matrix."""
    G4 = G.reshape(n, n, n, n)
    G4 = 0.5 * (G4 + G4.transpose(1, 0, 3, 2))
    G4 = 0.5 * (G4 + G4.transpose(2, 3, 0, 1))
    return G4


def rdm2_dense(rng, nmo: int, nelec: int, nterms: int | None = None) -> np.ndarray:
    n2 = nmo * nmo
    k = nterms or min(n2, 2 * nmo)
    V = rng.standard_normal((k, n2))
    w = np.abs(rng.standard_normal(k))
    G = (V.T * w) @ V
    G4 = _swap_sym(G, nmo)
    tr = np.einsum('aabb->', G4)
    return G4 * (nelec * (nelec - 1) / tr)


def rdm2_sparse(rng, nmo: int, nelec: int, density: float) -> np.ndarray:
    """PSD in pair space by construction: a sum of w v v^T over sparse v."""
    n2 = nmo * nmo
    target = density * n2 * n2
    s = max(2, int(round(np.sqrt(target / (2.0 * max(nmo, 4))))))
    s = min(s, n2)
    G = np.zeros((n2, n2))
    diag_pairs = np.arange(nmo) * (nmo + 1)
    nz = 0
    it = 0
    while nz < target and it < 100000:
        it += 1
        idx = rng.choice(n2, size=s, replace=False)
        idx[0] = diag_pairs[rng.integers(nmo)]
        v = rng.standard_normal(s)
        G[np.ix_(idx, idx)] += abs(rng.standard_normal()) * np.outer(v, v)
        if it % 4 == 0:
            nz = np.count_nonzero(_swap_sym(G, nmo))
    G4 = _swap_sym(G, nmo)
    tr = np.einsum('aabb->', G4)
    return G4 * (nelec * (nelec - 1) / tr)


def rdm_rows(G4: np.ndarray):
    idx = np.argwhere(G4 != 0.0)
    mat = (idx + 1).astype(np.int32)
    total = G4[G4 != 0.0].astype(np.float64)
    return mat, total


def onerdm_from_2rdm(G4: np.ndarray, nelec: int) -> np.ndarray:
    D = np.einsum('pqrr->pq', G4) / (nelec - 1)
    return 0.5 * (D + D.T)


def _problem(name, atoms, shells, nmo, nelec, q, rng, G4=None, density=None, meta=None):
    ga, L, M, N, X, Y, Z, grp, aof = build_basis(atoms, shells)
    C = lowdin_mos(rng, nmo, ga, L, M, N, X, Y, Z)
    if G4 is None:
        G4 = rdm2_dense(rng, nmo, nelec) if density is None else rdm2_sparse(rng, nmo, nelec, density)
    mat, total = rdm_rows(G4)
    D = onerdm_from_2rdm(G4, nelec)
    return Problem(name=name, atoms=np.asarray(atoms, float), ga=ga, l=L, m=M, n=N, xx=X, yy=Y, zz=Z,
                   group=grp, atom_of=aof, mmod=C, mat=mat, total=total, onerdm=D, q=q,
                   nelec=nelec, meta=meta or {})


SEED0 = 20261203


def config1_h2() -> Problem:
    """H2: z = +-0.7 bohr; per atom s(0.15, 0.6, 2.5, 12.0) + p(1.0); 4 MOs;
    dense 2-RDM, trace 2; q = 0..10 (100 points)."""
    rng = np.random.default_rng(SEED0 + 1)
    atoms = np.array([[0.0, 0.0, -0.7], [0.0, 0.0, 0.7]])
    shells = [[(0, e) for e in (0.15, 0.6, 2.5, 12.0)] + [(1, 1.0)] for _ in range(2)]
    return _problem("h2", atoms, shells, 4, 2, q_grid(10.0, 100), rng)


def _diatomic_shells():
    return ([(0, e) for e in geometric(0.1, 5000.0, 6)] + [(1, e) for e in geometric(0.2, 30.0, 3)]
            + [(2, 0.8)])


def config2_diatomic() -> Problem:
    """Diatomic, 14 electrons: atoms at z = 0, 2.13; per atom s(6, 0.1-5000),
    p(3, 0.2-30), d(1, 0.8); 10 MOs; dense 2-RDM (10^4 rows), trace 182;
    q = 0..12 (200 points)."""
    rng = np.random.default_rng(SEED0 + 2)
    atoms = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 2.13]])
    shells = [_diatomic_shells() for _ in range(2)]
    return _problem("diatomic", atoms, shells, 10, 14, q_grid(12.0, 200), rng)


def _ab6_shells():
    return ([(0, e) for e in geometric(0.1, 1.0e5, 8)] + [(1, e) for e in geometric(0.15, 200.0, 5)]
            + [(2, 0.6)])


def config3_ab6(nq: int = 500, natoms: int = 7) -> Problem:
    """Octahedral AB6 (S-F 2.95 bohr); per atom s(8, 0.1-1e5), p(5, 0.15-200),
    d(1, 0.6); 40 MOs; 5 % nonzero sparse PSD 2-RDM, trace N(N-1), N = 70;
    q = 0..15 (500 points).  ``natoms < 7`` keeps the first atoms only (a
    smaller case of the same basis, for profiling)."""
    rng = np.random.default_rng(SEED0 + 3)
    r = 2.95
    atoms = np.array([[0, 0, 0], [r, 0, 0], [-r, 0, 0], [0, r, 0], [0, -r, 0], [0, 0, r], [0, 0, -r]],
                     dtype=float)[:natoms]
    shells = [_ab6_shells() for _ in range(natoms)]
    name = "ab6" if natoms == 7 else f"ab6_{natoms}atom"
    return _problem(name, atoms, shells, 40, 70, q_grid(15.0, nq), rng, density=0.05)


def cms_onerdms(prob: Problem, seed: int = SEED0 + 9):
    """Two seeded transition-like 1-RDMs for the resolved CMS (type 9): the
    bra's (states 1-3) and the ket's (states 2-3), nonsymmetric, on the scale
    of ``prob.onerdm``."""
    rng = np.random.default_rng(seed)
    n = prob.onerdm.shape[0]
    s = float(np.max(np.abs(prob.onerdm)))
    a = prob.onerdm + 0.3 * s * rng.standard_normal((n, n))
    b = 0.5 * prob.onerdm + 0.3 * s * rng.standard_normal((n, n))
    return a, b


def hexagon(radius: float = 2.64) -> np.ndarray:
    ang = np.arange(6) * np.pi / 3.0
    return np.stack([radius * np.cos(ang), radius * np.sin(ang), np.zeros(6)], axis=1)


def config5_fit(nq: int = 400) -> Problem:
    """6-atom ring with the config-2 basis per atom; 30 MOs; dense 2-RDM;
    q = 0..14 (400 points)."""
    rng = np.random.default_rng(SEED0 + 5)
    atoms = hexagon()
    shells = [_diatomic_shells() for _ in range(6)]
    return _problem("fit6", atoms, shells, 30, 30, q_grid(14.0, nq), rng)


def config5_aligned_grid(n: int = 64, qmax: float = 14.0) -> np.ndarray:
    """The n^3 Cartesian q vectors of the ring's aligned intensity: every
    component on linspace(-qmax, qmax, n) (bohr^-1), x fastest; shape (n^3, 3)."""
    ax = np.linspace(-qmax, qmax, n)
    qz, qy, qx = np.meshgrid(ax, ax, ax, indexing="ij")
    return np.stack([qx.ravel(), qy.ravel(), qz.ravel()], axis=1)


def config5_geometries(base: Problem, ngeom: int = 512, sigma: float = 0.1, seed: int = SEED0 + 55):
    rng = np.random.default_rng(seed)
    out = [base.atoms.copy()]
    for _ in range(ngeom - 1):
        out.append(base.atoms + sigma * rng.standard_normal(base.atoms.shape))
    return np.stack(out)


def config4_batch(nmol: int = 1024, nq: int = 256, seed: int = SEED0 + 4):
    """Uneven batch: 2-12 atoms placed 1.8-3.0 bohr from a random earlier atom;
    per atom s(4)+p(2)+d(1) with exponents jittered +-20 %; 4-24 MOs; sparse
    PSD 2-RDMs with 1-10 % nonzero entries; q = 0..12 (256 points)."""
    rng = np.random.default_rng(seed)
    base_s = [0.15, 0.8, 4.0, 20.0]
    base_p = [0.3, 1.5]
    base_d = [0.7]
    q = q_grid(12.0, nq)
    mols = []
    for i in range(nmol):
        na = int(rng.integers(2, 13))
        atoms = [np.zeros(3)]
        while len(atoms) < na:
            anchor = atoms[int(rng.integers(len(atoms)))]
            d = rng.standard_normal(3)
            d /= np.linalg.norm(d)
            cand = anchor + d * rng.uniform(1.8, 3.0)
            if min(np.linalg.norm(cand - a) for a in atoms) > 1.5:
                atoms.append(cand)
        atoms = np.array(atoms)
        jit = lambda e: float(e * rng.uniform(0.8, 1.2))
        shells = [[(0, jit(e)) for e in base_s] + [(1, jit(e)) for e in base_p] + [(2, jit(e)) for e in base_d]
                  for _ in range(na)]
        ngto = na * 16
        nmo = int(min(rng.integers(4, 25), ngto))
        nelec = int(max(2, min(2 * nmo - 2, nmo + int(rng.integers(0, nmo)))))
        dens = float(rng.uniform(0.01, 0.10))
        mols.append(_problem(f"batch{i}", atoms, shells, nmo, nelec, q, rng, density=dens))
    return mols


CONFIGS = {1: config1_h2, 2: config2_diatomic, 3: config3_ab6, 5: config5_fit}
