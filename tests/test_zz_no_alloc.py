"""Stage 2 with static scratch (thistle_bessel_sum_static), for callers that
cannot allocate device memory when they evaluate.

Kept in a file of its own that pytest collects last.  It runs the new entry
point twice in a row on the records of a plan and checks each result against
the plan's own execution (the existing entry point), at the tolerance of the
other parity tests.
"""
import ctypes as C

import numpy as np
import pytest

from thistle_b200 import _abi
from thistle_b200 import inputs as I
from thistle_b200 import main_calculation as MC

from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_static_scratch_bessel_sum_matches_plan():
    import torch

    p = I.config2_diatomic()
    with MC.ScatteringPlan.from_problem(p, MC.TOTAL_J0) as plan:
        ref = plan.execute()
        r = plan.records()
        out = torch.empty(p.nq, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()
        for _ in range(2):
            out.fill_(float("nan"))
            rc = _abi.lib().thistle_bessel_sum_static(
                C.c_void_p(r["rec"]), r["ncls"], r["begin"].ctypes.data_as(_abi.I64),
                r["end"].ctypes.data_as(_abi.I64), r["recoff"].ctypes.data_as(_abi.I64),
                r["rs"].ctypes.data_as(_abi.I32), C.c_void_p(r["q"]), p.nq, C.c_void_p(out.data_ptr()),
                C.c_void_p(stream.cuda_stream))
            _abi.check(rc)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.max(rel_err(got, ref)) < 1e-10


def test_static_scratch_rejects_too_many_q():
    r_b = np.zeros(1, np.int64)
    r_e = np.ones(1, np.int64)
    r_o = np.zeros(1, np.int64)
    r_s = np.full(1, 8, np.int32)
    rc = _abi.lib().thistle_bessel_sum_static(
        C.c_void_p(8), 1, r_b.ctypes.data_as(_abi.I64), r_e.ctypes.data_as(_abi.I64),
        r_o.ctypes.data_as(_abi.I64), r_s.ctypes.data_as(_abi.I32), C.c_void_p(8), 4096, C.c_void_p(8),
        C.c_void_p(0))
    assert rc == -1
    assert b"1024" in _abi.lib().thistle_last_error_string()
