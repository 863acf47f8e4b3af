"""Input formats and the Main.exe-compatible command line.

CPU: the molden reader (thistle_b200.molden, the reference's
src/molden_reader_nikola.py conventions) reproduces the committed parse of
the reference's CO molden file and, with the file's own units honoured,
gives MOs that are orthonormal in the decontracted primitive overlap; the
readers of basis.dat / MOs.dat / options.dat (src/Main.f90:28-125) read back
what the reference's input writer layout holds.

GPU: the command line (python -m thistle_b200.main) on input files written
in the reference's layout for the CO basis with the reference's HF 2-RDM
file and its 1-RDM -- total j0, elastic j0 and total j2 against the oracle
(1e-10 relative per point; j2 also within 1e-12 of the j0 intensity).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from thistle_b200 import inputs as I
from thistle_b200 import main as M
from thistle_b200 import molden

from conftest import rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
import make_golden_large as MG  # noqa: E402

REF_MOLDEN = os.path.join(MG.REF, MG.CO_MOLDEN)


def write_inputs(d, p, type_, qmin, qmax, npoints, out="result.dat"):
    """basis.dat, MOs.dat, options.dat and the RDM files in the layout of
    src/File_creator_pyscf.py:109-255 (readrdm branch)."""
    with open(os.path.join(d, "basis.dat"), "w") as f:
        f.write(f"{p.ngto}\n")
        for i in range(p.ngto):
            f.write(f"{float(p.xx[i])!r} {float(p.yy[i])!r} {float(p.zz[i])!r} {float(p.ga[i])!r} "
                    f"{p.l[i]} {p.m[i]} {p.n[i]} {p.group[i]}\n")
    with open(os.path.join(d, "MOs.dat"), "w") as f:
        f.write(f"{p.mmod.shape[0]} {p.mmod.shape[1]}\n")
        for row in p.mmod:
            f.write(" ".join(repr(float(v)) for v in row) + " \n")
    with open(os.path.join(d, "twordm.txt"), "w") as f:
        for r, v in zip(p.mat, p.total):
            f.write(f"{r[0]} {r[1]} {r[2]} {r[3]} {float(v)!r}\n")
    D = p.onerdm
    with open(os.path.join(d, "onerdm.txt"), "w") as f:
        for i in range(D.shape[0]):
            for j in range(D.shape[1]):
                f.write(f"{i + 1} {j + 1} {float(D[i, j])!r}\n")
    with open(os.path.join(d, "options.dat"), "w") as f:
        f.write(f"{len(p.atoms)}\n")
        f.write(" ".join(str(int(z)) for z in p.meta.get("Z", [6] * len(p.atoms))) + " \n")
        for a in p.atoms:
            f.write(" ".join(repr(float(v)) for v in a) + "\n")
        f.write(f"{p.cutoffcentre}\n{p.cutoffz}\n{p.cutoffmd}\nFalse\nFalse\nFalse\n")
        f.write(f"{qmin} {qmax} {npoints} \n{type_}\n1 1 1\n{out}\nFalse\nFalse\nFalse\n")
        f.write("readrdm\nonerdm.txt\ntwordm.txt")


def co_problem():
    g = np.load(os.path.join(GOLD, "golden_co.npz"))
    p = MG.co_problem(g, np.load(os.path.join(GOLD, "golden_refrdm.npz")))
    p.meta["Z"] = [int(z) for z in g["numbers"]]
    return p, g


@pytest.mark.skipif(not os.path.exists(REF_MOLDEN), reason="no reference checkout")
def test_molden_reader_reproduces_committed_parse():
    g = np.load(os.path.join(GOLD, "golden_co.npz"))
    gt, at = molden.read_orbitals(REF_MOLDEN, N=100, decontract=True)
    for k in ("ga", "l", "m", "n", "x", "y", "z", "group"):
        np.testing.assert_array_equal(getattr(gt, k), g[k])
    np.testing.assert_array_equal(gt.mo.T, g["mmod"])
    np.testing.assert_array_equal(at.xyz, g["atoms"])


@pytest.mark.skipif(not os.path.exists(REF_MOLDEN), reason="no reference checkout")
def test_molden_mos_orthonormal_in_primitive_overlap():
    """Decontraction and normalisation folded into the MO coefficients: the
    alpha MOs (the first 18 of the UCCSD file) are orthonormal over the
    unnormalised primitives when the [Atoms] (AU) header is honoured."""
    gt, _ = molden.read_orbitals(REF_MOLDEN, N=100, decontract=True, units="file")
    S = I.overlap(gt.ga, gt.l, gt.m, gt.n, gt.x, gt.y, gt.z)
    Mo = gt.mo.T[:18]
    assert np.max(np.abs(Mo @ S @ Mo.T - np.eye(18))) < 1e-12
    # groups are consecutive and each holds one primitive shell
    assert gt.group[0] == 1 and np.all(np.diff(gt.group) >= 0) and np.all(np.diff(gt.group) <= 1)


def test_input_files_round_trip(tmp_path):
    p, _ = co_problem()
    write_inputs(str(tmp_path), p, 1, 0.0, 8.0, 60)
    xx, yy, zz, ga, l, m, n, group = M.read_basis(str(tmp_path / "basis.dat"))
    np.testing.assert_array_equal(ga, p.ga)
    np.testing.assert_array_equal(zz, p.zz)
    np.testing.assert_array_equal(group, p.group)
    np.testing.assert_array_equal(M.read_mos(str(tmp_path / "MOs.dat")), p.mmod)
    o = M.read_options(str(tmp_path / "options.dat"))
    assert o["natoms"] == 2 and o["type"] == 1 and o["npoints"] == 60 and o["var"] == "readrdm"
    assert o["file_onerdm"] == "onerdm.txt" and o["file_twordm"] == "twordm.txt" and not o["molpro"]
    np.testing.assert_array_equal(o["geom"], p.atoms)
    q = M.linspace_1(0.0, 8.0, 60)
    assert q[0] == 0.0 and abs(q[-1] - 8.0) < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("type_", [1, 2, 7])
def test_command_line_co_molden_vs_oracle(tmp_path, type_):
    p, g = co_problem()
    write_inputs(str(tmp_path), p, type_, 0.0, 8.0, 60)
    r = subprocess.run([sys.executable, "-m", "thistle_b200.main", str(tmp_path)], cwd=ROOT,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.loadtxt(str(tmp_path / "result.dat"))
    np.testing.assert_allclose(out[1:, 0], g["q"][1:], rtol=1e-15)
    ref = g[f"type{type_}"]
    if type_ == 7:
        assert np.all(np.abs(out[:, 1] - ref) <= 1e-10 * np.abs(ref) + 1e-12 * np.abs(g["type1"]))
    else:
        assert np.max(rel_err(out[:, 1], ref)) < 1e-10


def _write_onerdm(path, D):
    with open(path, "w") as f:
        for i in range(D.shape[0]):
            for j in range(D.shape[1]):
                f.write(f"{i + 1} {j + 1} {float(D[i, j])!r}\n")


def test_command_line_refuses_total_j1(tmp_path):
    """Type 10 stops as the reference's does (tot_integration_j1 stops before
    integrating, src/Integrals.f90:526-527), before any device work."""
    p = I.config1_h2()
    write_inputs(str(tmp_path), p, 10, 0.0, 4.0, 20)
    with pytest.raises(SystemExit) as e:
        M.run(str(tmp_path))
    assert "stops before integrating" in str(e.value)


@pytest.mark.gpu
def test_command_line_resolved_cms_vs_golden(tmp_path):
    """Type 9 reads its two 1-RDM files (the bra's, then the ket's) from the
    two RDM names of the readrdm branch."""
    p = I.config2_diatomic()
    d1, d2 = I.cms_onerdms(p)
    p = I.Problem(**{**p.__dict__, "onerdm": d1})
    write_inputs(str(tmp_path), p, 9, 0.0, float(p.q[-1]), p.nq)
    _write_onerdm(str(tmp_path / "twordm.txt"), d2)
    r = subprocess.run([sys.executable, "-m", "thistle_b200.main", str(tmp_path)], cwd=ROOT,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.loadtxt(str(tmp_path / "result.dat"))
    g = np.load(os.path.join(GOLD, "golden_cfg2.npz"))
    np.testing.assert_allclose(out[1:, 0], g["q"][1:], rtol=1e-14)
    assert np.max(rel_err(out[:, 1], g["type9"])) < 1e-10
