"""Build recipe for the C oracle (test infrastructure).

``python -m oracle.build`` (or ``build()``) compiles ``thistle_oracle.c`` into
``oracle/liboracle_thistle.so`` with ``-ffp-contract=off`` so that no fused
multiply-add changes the reference's rounding order.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose: bool = False) -> str:
    src = os.path.join(HERE, "thistle_oracle.c")
    out = os.path.join(HERE, "liboracle_thistle.so")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-Wall",
           "-Wno-unused-function", "-o", out, src, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return out


if __name__ == "__main__":
    print(build(verbose=True))
