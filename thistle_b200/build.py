"""Build recipe for libthistle_b200.so (sm_100a), in-tree.

``python -m thistle_b200.build`` compiles every CUDA source under
``thistle_b200/csrc`` with nvcc for ``compute_100a/sm_100a`` into
``thistle_b200/libthistle_b200.so``.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libthistle_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        sorted(glob.glob(os.path.join(HERE, "csrc", "*.h"))) + [os.path.join(ROOT, "include", "thistle_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(verbose: bool = False, force: bool = False, extra=None, out: str | None = None,
          objdir: str | None = None) -> str:
    """Compile into ``out`` (default: the in-tree library); ``extra`` nvcc flags
    and a separate ``objdir`` give a differently configured build."""
    if out is None and up_to_date() and not force:
        return LIB
    LIBOUT = out or LIB
    objdir = objdir or os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "csrc"),
              "--expt-relaxed-constexpr", "-Xptxas", "-v" if verbose else "-O3"]
    if extra:
        common += list(extra)
    headers = [d for d in deps() if not d.endswith(".cu")]
    newest_header = max(os.path.getmtime(h) for h in headers)
    todo = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= newest_header):
            continue
        todo.append(common + ["-c", src, "-o", obj])
    # one nvcc per translation unit, in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        procs = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), todo))
    for cmd, pr in zip(todo, procs):
        if verbose:
            print(" ".join(cmd))
            print(pr.stdout + pr.stderr)
        if pr.returncode != 0:
            raise RuntimeError("nvcc failed: " + " ".join(cmd) + "\n" + pr.stdout + pr.stderr)
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIBOUT, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIBOUT


if __name__ == "__main__":
    import sys
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
