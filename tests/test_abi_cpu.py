"""The C-ABI library without a GPU: it loads, exports every declared symbol,
and rejects bad input with the documented status codes (validation runs
before any CUDA call)."""
import os
import re

import numpy as np
import pytest

from thistle_b200 import _abi
from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC
from thistle_b200._abi import ThistleError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "thistle_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(thistle_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_header_symbols():
    L = _abi.lib()
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(_abi.EXPORTS) == syms
    assert L.thistle_version() >= 100


def _call(p, **over):
    kw = dict(type=1, ngto=p.ngto, ng=p.ng, ga=p.ga, l=p.l, m=p.m, n=p.n, xx=p.xx, yy=p.yy, zz=p.zz,
              mmod=p.mmod, q=p.q, group=p.group, mat=p.mat, total=p.total, onerdm=None)
    kw.update(over)
    return MC.total_scattering_calculation(kw["type"], None, None, 0, 0, 1, kw["ngto"], kw["ng"], kw["ga"],
                                           kw["l"], kw["m"], kw["n"], kw["xx"], kw["yy"], kw["zz"], kw["mmod"],
                                           kw["q"], len(kw["q"]), kw["group"], p.cutoffz, p.cutoffmd,
                                           p.cutoffcentre, mat=kw["mat"], total=kw["total"],
                                           onerdm=kw["onerdm"])


@pytest.fixture(scope="module")
def h2():
    return I.config1_h2()


def code_of(fn):
    with pytest.raises(ThistleError) as e:
        fn()
    return e.value.code


def test_q_zero_rejected(h2):
    q = h2.q.copy()
    q[0] = 0.0
    assert code_of(lambda: _call(h2, q=q)) == -8


def test_angular_momentum_above_g_rejected(h2):
    l = h2.l.copy()
    l[0] = 5
    assert code_of(lambda: _call(h2, l=l)) == -3


def test_nonfinite_rejected(h2):
    xx = h2.xx.copy()
    xx[3] = np.nan
    assert code_of(lambda: _call(h2, xx=xx)) == -4
    tot = h2.total.copy()
    tot[0] = np.inf
    assert code_of(lambda: _call(h2, total=tot)) == -4


def test_bad_type_rejected(h2):
    assert code_of(lambda: _call(h2, type=11)) == -7


def test_total_j1_refused_with_the_references_reason(h2):
    """Type 10: the reference's tot_integration_j1 stops before it integrates
    (src/Integrals.f90:526-527), so the library refuses it by name."""
    with pytest.raises(ThistleError) as e:
        _call(h2, type=10)
    assert e.value.code == -7 and "stops before integrating" in str(e.value)


def test_noncontiguous_group_rejected(h2):
    g = h2.group.copy()
    g[5] = g[0]          # function 5 (inside the p shell) joins group 1
    assert code_of(lambda: _call(h2, group=g)) == -2


def test_mixed_shell_group_rejected(h2):
    ga = h2.ga.copy()
    i = int(np.flatnonzero(h2.l + h2.m + h2.n == 1)[1])
    ga[i] *= 1.1
    assert code_of(lambda: _call(h2, ga=ga)) == -2


def test_rdm_index_out_of_range_rejected(h2):
    mat = h2.mat.copy()
    mat[0, 2] = h2.nmo + 1
    assert code_of(lambda: _call(h2, mat=mat)) == -2


def test_elastic_needs_onerdm(h2):
    assert code_of(lambda: _call(h2, type=2, onerdm=None)) == -1


def test_static_bessel_sum_rejects_table_not_starting_at_zero():
    """thistle_bessel_sum_static walks quartets from 0: a class table whose
    first range starts later is rejected before any device work."""
    import ctypes as C
    b = np.array([5], np.int64)
    e = np.array([9], np.int64)
    o = np.zeros(1, np.int64)
    s = np.full(1, 8, np.int32)
    rc = _abi.lib().thistle_bessel_sum_static(
        C.c_void_p(8), 1, b.ctypes.data_as(_abi.I64), e.ctypes.data_as(_abi.I64), o.ctypes.data_as(_abi.I64),
        s.ctypes.data_as(_abi.I32), C.c_void_p(8), 16, C.c_void_p(8), C.c_void_p(0))
    assert rc == -2
    assert b"quartet 0" in _abi.lib().thistle_last_error_string()
