"""Builds the CUDA library libdream_das.so in-tree for sm_100a with nvcc.

    python -m dream_b200.build            # incremental
    python -m dream_b200.build --force    # rebuild everything
    python -m dream_b200.build --checked  # bounds-checked gathers -> libdream_das_checked.so

The shared object is written next to this file so that it travels with the
source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdream_das.so")
BUILD_CHECKED = os.path.join(HERE, "_build_checked")
LIB_CHECKED = os.path.join(HERE, "libdream_das_checked.so")
PEAKS_SRC = os.path.join(HERE, "peaks", "peaks.cu")
PEAKS_LIB = os.path.join(HERE, "libdream_peaks.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math",
           "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-Werror=infinite-recursion",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _deps_mtime() -> float:
    files = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max([os.path.getmtime(f) for f in files] + [0.0])


def _compile(src: str, force: bool, verbose: bool, checked: bool = False) -> str:
    obj = os.path.join(BUILD_CHECKED if checked else BUILD, os.path.basename(src) + ".o")
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= _deps_mtime()):
        return obj
    cmd = [nvcc(), *ARCH, *NVFLAGS, *(["-DDREAM_DAS_CHECKED"] if checked else []), "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Builds libdream_das.so (or, with checked=True, libdream_das_checked.so,
    whose gathers test every index against the extent of Y) and the roofline
    microbenchmark library."""
    bdir, lib = (BUILD_CHECKED, LIB_CHECKED) if checked else (BUILD, LIB)
    os.makedirs(bdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose, checked), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # roofline microbenchmarks (separate library, used by bench.py)
    if force or not os.path.exists(PEAKS_LIB) or os.path.getmtime(PEAKS_LIB) < os.path.getmtime(PEAKS_SRC):
        cmd = [nvcc(), *ARCH, *NVFLAGS, "-shared", PEAKS_SRC, "-o", PEAKS_LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {PEAKS_SRC}:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill report")
    ap.add_argument("--checked", action="store_true", help="bounds-checked gathers (libdream_das_checked.so)")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, checked=a.checked))
