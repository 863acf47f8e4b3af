"""Command-line front end with the inputs and output of the reference's
``Main.exe`` (src/Main.f90), on the B200 path.

    python -m thistle_b200.main [directory]

reads ``basis.dat``, ``MOs.dat`` and ``options.dat`` from the directory
(default: the working directory), computes the intensity of the calculation
type named there through Entry 1 and writes ``q I(q)`` lines to the output
file named there, as Main.f90's ``readrdm`` branch does (:113-161).

Input formats (written by src/File_creator_pyscf.py:109-255):

* ``basis.dat``: ngtos, then per primitive ``x y z ga l m n group``
  (Main.f90:28-34);
* ``MOs.dat``: ``norbs ngtos``, then one row of ngtos coefficients per MO
  (:38-45);
* ``options.dat`` (:47-125): natoms; the atomic numbers; natoms rows of
  coordinates; cutoffcentre; cutoffz; cutoffmd; three logicals (jeremyR,
  mcci, hf); ``qmin qmax npoints``; the type; ``state1 state2 state3``; the
  output file name; three logicals (molpro, molcas, bagel); then for the
  RDM branch the word ``readrdm`` and the 1-RDM and 2-RDM file names
  (read_onerdm / read_twordm formats, src/one_rdm.f90:2072-2147).  Type 9
  (resolved CMS) reads both names as 1-RDM files: the bra's (states 1-3)
  and the ket's (states 2-3).  Type 10 stops with the reference's reason:
  its tot_integration_j1 stops before integrating (src/Integrals.f90:526-527).

The q grid is linspace_1(qmin, qmax, npoints) (src/linspace.f90).  A q of 0
makes the reference divide by zero (NaN in its output); here it is replaced
by 1e-10, the value the reference's drivers use, with a note on stderr.
The CI branches (molpro, molcas, bagel) build RDMs from CI vectors, which is
upstream of the scattering path: they are rejected with a message.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import main_calculation as MC


def _tokens(path):
    with open(path) as f:
        return [line.split() for line in f if line.strip()]


def _logical(tok: str) -> bool:
    """A Fortran list-directed logical: T/F, .true./.false., True/False."""
    t = tok.strip().lstrip(".").upper()
    if not t or t[0] not in "TF":
        raise ValueError(f"not a logical: {tok!r}")
    return t[0] == "T"


def _word(tok: str) -> str:
    return tok.strip().strip("'\"")


def read_basis(path):
    """basis.dat: (xx, yy, zz, ga, l, m, n, group)."""
    rows = _tokens(path)
    n = int(rows[0][0])
    a = np.array([[float(v) for v in r[:8]] for r in rows[1:1 + n]])
    if a.shape != (n, 8):
        raise ValueError(f"{path}: expected {n} rows of 8 columns")
    i32 = lambda c: a[:, c].astype(np.int32)
    return a[:, 0], a[:, 1], a[:, 2], a[:, 3], i32(4), i32(5), i32(6), i32(7)


def read_mos(path):
    """MOs.dat: (norbs, ngtos) coefficients, read row after row as Fortran's
    list-directed read does (values may wrap over lines)."""
    vals = [v for r in _tokens(path) for v in r]
    norbs, ngtos = int(vals[0]), int(vals[1])
    c = np.array([float(v) for v in vals[2:2 + norbs * ngtos]])
    if c.size != norbs * ngtos:
        raise ValueError(f"{path}: expected {norbs} x {ngtos} coefficients")
    return c.reshape(norbs, ngtos)


def read_options(path):
    """options.dat as a dict (see the module docstring)."""
    rows = _tokens(path)
    k = 0

    def nxt():
        nonlocal k
        r = rows[k]
        k += 1
        return r

    o = {}
    natoms = int(nxt()[0])
    o["natoms"] = natoms
    zs = []
    while len(zs) < natoms:
        zs.extend(float(v) for v in nxt())
    o["atoms"] = np.array(zs[:natoms])
    o["geom"] = np.array([[float(v) for v in nxt()[:3]] for _ in range(natoms)]).reshape(natoms, 3)
    o["cutoffcentre"] = float(nxt()[0].replace("D", "E").replace("d", "e"))
    o["cutoffz"] = float(nxt()[0].replace("D", "E").replace("d", "e"))
    o["cutoffmd"] = float(nxt()[0].replace("D", "E").replace("d", "e"))
    o["jeremyR"] = _logical(nxt()[0])
    o["mcci"] = _logical(nxt()[0])
    o["hf"] = _logical(nxt()[0])
    r = nxt()
    o["qmin"], o["qmax"], o["npoints"] = float(r[0]), float(r[1]), int(r[2])
    o["type"] = int(nxt()[0])
    r = nxt()
    o["state1"], o["state2"], o["state3"] = (int(v) for v in r[:3])
    o["file_out"] = _word(nxt()[0])
    o["molpro"] = _logical(nxt()[0])
    o["molcas"] = _logical(nxt()[0])
    o["bagel"] = _logical(nxt()[0])
    o["var"] = _word(nxt()[0]) if k < len(rows) else ""
    if o["var"] == "readrdm":
        o["file_onerdm"] = _word(nxt()[0])
        o["file_twordm"] = _word(nxt()[0])
    return o


def linspace_1(qmin: float, qmax: float, n: int) -> np.ndarray:
    """linspace_1 of src/linspace.f90: from + range (i - 1) / (n - 1)."""
    i = np.arange(1, n + 1, dtype=np.float64)
    return qmin + (qmax - qmin) * (i - 1) / (n - 1)


def run(directory: str = ".") -> str:
    """Reads the three input files of ``directory``, writes the output file
    there and returns its path."""
    path = lambda f: f if os.path.isabs(f) else os.path.join(directory, f)
    xx, yy, zz, ga, l, m, n, group = read_basis(path("basis.dat"))
    mmod = read_mos(path("MOs.dat"))
    o = read_options(path("options.dat"))
    if o["molpro"] or o["molcas"] or o["bagel"] or o["var"] != "readrdm":
        raise SystemExit("thistle_b200.main: only the readrdm branch is provided (the RDMs come from files); "
                         "building RDMs from CI vectors is upstream of the scattering path")
    q = linspace_1(o["qmin"], o["qmax"], o["npoints"])
    if np.any(q <= 0.0):
        print("thistle_b200.main: q <= 0 replaced by 1e-10 (the reference divides by q there)", file=sys.stderr)
        q = np.where(q <= 0.0, 1e-10, q)
    t = o["type"]
    mat = total = onerdm = onerdm2 = None
    if t == MC.TOTAL_J1:
        raise SystemExit("thistle_b200.main: type 10 (total j1) is not computed by the reference either: "
                         "tot_integration_j1 stops before integrating (src/Integrals.f90:526-527)")
    if t in (MC.TOTAL_J0, MC.TOTAL_J2, MC.TOTAL_ELECTRON):
        mat, total = MC.read_twordm(path(o["file_twordm"]))
    if t in (MC.ELASTIC_J0, MC.ELASTIC_J2, MC.ELASTIC_ALIGNED, MC.TOTAL_ELECTRON, MC.ELASTIC_ELECTRON):
        onerdm = MC.read_onerdm(path(o["file_onerdm"]))
    if t == MC.RESOLVED_CMS:
        onerdm = MC.read_onerdm(path(o["file_onerdm"]))
        onerdm2 = MC.read_onerdm(path(o["file_twordm"]))
    nq = o["npoints"] if t not in (MC.TOTAL_ALIGNED,) else 3131
    qabs, result = MC.total_scattering_calculation(
        t, o["atoms"], o["geom"], o["state1"], o["state2"], int(l.max()), l.size, int(group.max()), ga, l, m, n,
        xx, yy, zz, mmod, q if t != MC.TOTAL_ALIGNED else np.zeros(3131), nq, group, o["cutoffz"],
        o["cutoffmd"], o["cutoffcentre"], mat=mat, total=total, onerdm=onerdm, onerdm2=onerdm2)
    qout = q if t not in (MC.TOTAL_ALIGNED, MC.ELASTIC_ALIGNED) else qabs
    out = path(o["file_out"])
    with open(out, "w") as f:
        for a, b in zip(qout, result):
            f.write(f"{a:25.17E} {b:25.17E}\n")
    return out


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    out = run(argv[0] if argv else ".")
    print(out, "created")
    return 0


if __name__ == "__main__":
    sys.exit(main())
