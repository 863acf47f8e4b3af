"""Molden input for the scattering path: the reference's reader of molden
files (src/molden_reader_nikola.py), with its conventions.

``read_orbitals(file, N, decontract)`` returns ``(gtos, atoms)`` like the
reference's ``read_orbitals`` (:496-508): one entry per primitive Cartesian
Gaussian with its exponent, angular exponents, centre, group (the primitive
shell: all Cartesian components of one primitive of one contraction) and MO
coefficients that already carry the contraction coefficient and the
primitive's normalisation (``_normalise_gto``, :437-441), so the MO of the
path is sum_i mo[i] x^l y^m z^n exp(-ga r^2) over unnormalised primitives.
With ``decontract`` the primitives that several contractions share (same
atom, exponent and l, m, n) are merged by adding their MO coefficients, and
the groups are renumbered 1, 2, 3, ... (``_reverse_contraction_scheme``,
:382-422) -- the basis the integrators take.

Conventions kept from the reference:

* Cartesian component order per shell type (:196-240): p x, y, z; d xx, yy,
  zz, xy, xz, yz; f and g as listed there;
* the MOs are read up to N of them and reordered by symmetry label, irrep
  (the digits after the point) first, then index (:258-345);
* the atomic coordinates of [Atoms] are divided by 0.52917721092 whatever
  unit the section header names (:104-110) -- a molden file written in bohr
  (``[Atoms] (AU)``) is therefore scaled; ``units="file"`` honours the header
  instead (AU: as read, Angs: divided by 0.52917721092).

Only the reader is provided; running the electronic-structure programs that
write molden files is upstream of the scattering path.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass

import numpy as np

AU2ANG = 0.52917721092

# Cartesian components of each shell type, in the reference's order
_CART = {
    "s": [(0, 0, 0)],
    "p": [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    "d": [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
    "f": [(3, 0, 0), (0, 3, 0), (0, 0, 3), (1, 2, 0), (2, 1, 0), (2, 0, 1), (1, 0, 2), (0, 1, 2), (0, 2, 1),
          (1, 1, 1)],
    "g": [(4, 0, 0), (0, 4, 0), (0, 0, 4), (3, 1, 0), (3, 0, 1), (1, 3, 0), (0, 3, 1), (1, 0, 3), (0, 1, 3),
          (2, 2, 0), (2, 0, 2), (0, 2, 2), (2, 1, 1), (1, 2, 1), (1, 1, 2)],
}


def _double_factorial(n: int) -> float:
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def primitive_norm(ga: float, l: int, m: int, n: int) -> float:
    """Normalisation of x^l y^m z^n exp(-ga r^2) (PrimitiveGTO.norm, :51-59)."""
    a = (2 / math.pi) ** 0.75 * 2 ** (l + m + n) * ga ** ((2 * l + 2 * m + 2 * n + 3) / 4.0)
    return a / math.sqrt(_double_factorial(2 * l - 1) * _double_factorial(2 * m - 1) * _double_factorial(2 * n - 1))


@dataclass
class Atoms:
    """The [Atoms] section: atomic numbers and positions (bohr, see units)."""
    numbers: np.ndarray
    xyz: np.ndarray

    def atomic_numbers(self):
        return self.numbers

    def geometry(self):
        return self.xyz


@dataclass
class GTOArray:
    """Primitive basis in the layout the integrators take (one row per
    primitive function): mo (nprim, nMO), x, y, z, ga, l, m, n, group (1-based)."""
    mo: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    ga: np.ndarray
    l: np.ndarray
    m: np.ndarray
    n: np.ndarray
    group: np.ndarray
    occ: np.ndarray = None
    energy: np.ndarray = None
    syms: np.ndarray = None


def _section(lines, tag):
    for k, line in enumerate(lines):
        if tag in line:
            return k
    raise ValueError(f"molden file has no {tag} section")


def _read_atoms(lines, units):
    k = _section(lines, "[Atoms]")
    header = lines[k]
    in_au = "AU" in header.upper().replace("ANGS", "")
    nums, xyz = [], []
    for line in lines[k + 1:]:
        if "[GTO]" in line:
            break
        cols = line.split()
        if len(cols) < 6:
            continue
        nums.append(int(cols[2]))
        v = np.array([float(c) for c in cols[3:6]])
        if units == "reference" or not in_au:
            v = v / AU2ANG
        xyz.append(v)
    return Atoms(np.array(nums, dtype=np.int32), np.array(xyz, dtype=np.float64).reshape(-1, 3))


def _read_contractions(lines):
    """Primitives as (atom, contraction, group, ga, c, l, m, n) (:135-250)."""
    k = _section(lines, "[GTO]") + 1
    prims = []
    contraction, group = 1, 0
    atom = None
    while k < len(lines) and "[MO]" not in lines[k]:
        cols = lines[k].split()
        k += 1
        if not cols:
            atom = None
            continue
        if atom is None:
            atom = int(cols[0])
            continue
        shell, nprim = cols[0].lower(), int(cols[1])
        if shell not in _CART:
            raise ValueError(f"shell type {shell!r}: only s, p, d, f and g are read")
        comps = _CART[shell]
        for _ in range(nprim):
            g, c = (float(t.replace("D", "E").replace("d", "e")) for t in lines[k].split()[:2])
            k += 1
            group += 1
            for i, (l, m, n) in enumerate(comps):
                prims.append((atom, contraction + i, group, g, c, l, m, n))
        contraction += len(comps)
    return prims


def _read_mos(lines, N):
    """MO coefficients (ncontracted, nMO), sorted by symmetry label (:258-345)."""
    k = _section(lines, "[MO]") + 1
    syms, energy, occ, table, this = [], [], [], [], []
    count = 0
    while k < len(lines) and count <= N and "[FREQ]" not in lines[k]:
        line = lines[k]
        k += 1
        if "Sym" in line:
            count += 1
            if count <= N:
                s = re.findall(r"\d+\.\d+", line)
                syms.append(s[0] if s else 1.1)
            if this:
                table.append(this)
            this = []
        elif "Ene" in line:
            energy.append(float(re.findall(r"\d+\.\d+", line)[0]))
        elif "Spin" in line:
            continue
        elif "Occup" in line:
            occ.append(float(re.findall(r"\d+\.\d+", line)[0]))
        elif line.split():
            this.append(float(line.split()[1]))
    if this:
        table.append(this)
    table = table[:len(syms)]
    s = np.array([float(v) for v in syms])
    key = (s - s.astype(int)) * 1000 + s.astype(int)
    idx = np.argsort(key, kind="stable")
    mo = np.array(table)[idx, :]
    e = np.array(energy)[:len(syms)][idx] if energy else np.zeros(len(syms))
    o = np.array(occ)[:len(syms)][idx] if occ else np.zeros(len(syms))
    return mo.T, o, e, s[idx]


def read_orbitals(file, N: int = 10000, decontract: bool = False, units: str = "reference"):
    """(gtos, atoms) of a molden file (a path or an open text file), as the
    reference's read_orbitals; see the module docstring for ``units``."""
    if units not in ("reference", "file"):
        raise ValueError("units must be 'reference' or 'file'")
    if isinstance(file, str):
        with open(file) as f:
            lines = f.read().splitlines()
    else:
        lines = file.read().splitlines()
    atoms = _read_atoms(lines, units)
    prims = _read_contractions(lines)
    mo_table, occ, energy, syms = _read_mos(lines, N)
    nmo = mo_table.shape[1]
    rows = []
    for (atom, contraction, group, g, c, l, m, n) in prims:
        mo = c * primitive_norm(g, l, m, n) * mo_table[contraction - 1, :]
        rows.append([atom, group, g, l, m, n, mo])
    if decontract:
        merged = []
        index = {}
        for atom, group, g, l, m, n, mo in rows:
            key = (atom, g, l, m, n)
            if key in index:
                merged[index[key]][6] = merged[index[key]][6] + mo
            else:
                index[key] = len(merged)
                merged.append([atom, group, g, l, m, n, mo.copy()])
        # consecutive group numbers in order of appearance
        counter, prev = 1, merged[0][1]
        for r in merged:
            if r[1] != prev:
                counter += 1
                prev = r[1]
            r[1] = counter
        rows = merged
    at = np.array([r[0] for r in rows]) - 1
    xyz = atoms.xyz[at]
    gtos = GTOArray(
        mo=np.array([r[6] for r in rows]).reshape(len(rows), nmo),
        x=xyz[:, 0].copy(), y=xyz[:, 1].copy(), z=xyz[:, 2].copy(),
        ga=np.array([r[2] for r in rows], dtype=np.float64),
        l=np.array([r[3] for r in rows], dtype=np.int32),
        m=np.array([r[4] for r in rows], dtype=np.int32),
        n=np.array([r[5] for r in rows], dtype=np.int32),
        group=np.array([r[1] for r in rows], dtype=np.int32),
        occ=occ, energy=energy, syms=syms)
    return gtos, atoms
