"""Build libzb.so (every CUDA source under csrc/) for sm_100a with nvcc.

    python zoomy-jax_b200/build.py [--force] [-j N]

Objects go to zoomy-jax_b200/_build/, the library to zoomy-jax_b200/lib/.
A source is recompiled only when it or a header is newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "lib" / "libzb.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -prec-div/-prec-sqrt/-ftz affect single precision only: the float kernels
# use fast division and square root (stated tolerance).  These flags leave
# double arithmetic IEEE; the Cartesian float64 kernels nonetheless divide and
# take square roots through their own Newton-refined routines (ndiv / nsqrt /
# nrsqrt in csrc/common.cuh, within 1 ulp of IEEE), and float64 parity with
# the oracle stays at 1e-12
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-prec-div=false", "-prec-sqrt=false", "-ftz=true",
         "--expt-relaxed-constexpr", "-I", str(INCLUDE), "-I", str(CSRC)]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libzb")
    return exe


def _newest_header():
    hs = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: pathlib.Path, force: bool, verbose: bool):
    obj = BUILD / (src.stem + ".o")
    if (not force and obj.exists()
            and obj.stat().st_mtime >= max(src.stat().st_mtime, _newest_header())):
        return obj, ""
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    jobs = jobs or min(len(srcs), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    if (force or not LIB.exists()
            or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs)):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB),
               *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("-v", action="store_true", help="print ptxas resource usage")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
