"""Build the CUDA library in place: every csrc/*.cu compiled for sm_100a and linked into
zebsdsolve_b200/libzebsdsolve_b200.so (the file the package loads); and, with gcc,
zebsdsolve_b200/libzebsdsolve.so, the reference's own C ABI over the package (csrc/ze_abi.c).

    python -m zebsdsolve_b200.build [--force] [--verbose]

Objects go to zebsdsolve_b200/_build/; a source is recompiled when it or any csrc header is newer
than its object.  nvcc cross-compiles without a GPU.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libzebsdsolve_b200.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--use_fast_math=false", "-Xptxas", "-v"]


def nvcc():
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def _compile(src, obj, verbose):
    cmd = [nvcc(), *ARCH, *[f for f in FLAGS if f != "--use_fast_math=false"], "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
    return src.name, r.stderr if verbose else ""


def write_twiddles():
    """csrc/twiddles.cuh: e^{-2πi t/N} for the register FFTs, from float64 rounded to float."""
    import math

    lines = ["// Twiddles e^{-2πi t/N} as float literals (written by build.py from the float64 values",
             "// rounded to the nearest float), for the register FFTs of the slab kernel.",
             "#pragma once", "", "namespace zeb {", ""]
    for n in (16, 32, 64, 128, 256):
        re = ", ".join(f"{math.cos(-2 * math.pi * t / n):.9e}f" for t in range(n))
        im = ", ".join(f"{math.sin(-2 * math.pi * t / n):.9e}f" for t in range(n))
        lines.append(f"__device__ constexpr float kTwRe{n}[{n}] = {{{re}}};")
        lines.append(f"__device__ constexpr float kTwIm{n}[{n}] = {{{im}}};")
    lines += ["", "}  // namespace zeb", ""]
    text = "\n".join(lines)
    path = CSRC / "twiddles.cuh"
    if not path.exists() or path.read_text() != text:
        path.write_text(text)


def build(force=False, verbose=False):
    BUILD.mkdir(exist_ok=True)
    write_twiddles()
    sources = sorted(CSRC.glob("*.cu"))
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    newest_header = max((h.stat().st_mtime for h in headers), default=0)
    jobs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for name, log in ex.map(lambda j: _compile(j[0], j[1], verbose), jobs):
                if verbose and log:
                    print(f"== {name}\n{log}", file=sys.stderr)
    objs = [BUILD / (s.stem + ".o") for s in sources]
    if jobs or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_abi(force)
    return LIB


ABI_SRC = CSRC / "ze_abi.c"
ABI_LIB = HERE / "libzebsdsolve.so"


def build_abi(force=False):
    """libzebsdsolve.so: the reference's own C ABI (csrc/ze_abi.c, include/zebsdsolve.h) with gcc.
    The Python C API is left to be resolved where the library is loaded (a Python process, or a
    native host that links libpython)."""
    import sysconfig

    deps = [ABI_SRC, INCLUDE / "zebsdsolve.h"]
    if force or not ABI_LIB.exists() or ABI_LIB.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        cmd = [os.environ.get("CC", "gcc"), "-O2", "-std=c11", "-Wall", "-Wextra", "-Wno-unused-parameter", "-fPIC",
               "-shared", "-fvisibility=hidden", "-I", sysconfig.get_paths()["include"], str(ABI_SRC), "-o",
               str(ABI_LIB), "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"gcc failed on {ABI_SRC.name}:\n{r.stderr}")
    return ABI_LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
