"""The oracle reproduces the committed golden vectors (pins it across edits)."""
import os

import numpy as np
import pytest

from thistle_b200 import inputs as I

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("cfg", [1, 2])
def test_oracle_golden(oracle, cfg):
    g = np.load(os.path.join(HERE, "golden", f"golden_cfg{cfg}.npz"))
    p = I.CONFIGS[cfg]()
    for t in (1, 2, 7):
        got = oracle.scattering(p, t, nthreads=8)
        np.testing.assert_allclose(got, g[f"type{t}"], rtol=1e-13, atol=1e-13 * np.max(np.abs(got)))
