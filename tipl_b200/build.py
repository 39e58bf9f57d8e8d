"""Builds tipl_b200/libregb200.so in-tree for sm_100a.

CUDA sources: nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -fmad=false.
Host sources: g++ -O2 -ffp-contract=off (no -march=native), so host float arithmetic
(the transform algebra) rounds like the reference's own build.
The CUDA runtime is linked statically; the library shares the device's primary
context with any other runtime in the process.

    python -m tipl_b200.build [--force] [-v]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libregb200.so")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-pthread", f"-I{CUDA_HOME}/include"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    hdr = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))
    return cu, cpp, hdr


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths) if paths else 0.0


def _compile(src, verbose, extra, hdr_time=0.0):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not extra and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
        return obj  # up to date (every header counts as a dependency of every source)
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + extra + [f"-I{INCLUDE}", "-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + [f"-I{INCLUDE}", "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    cu, cpp, hdr = _sources()
    srcs = [os.path.join(CSRC, f) for f in cu + cpp]
    deps = srcs + [os.path.join(CSRC, f) for f in hdr] + [os.path.join(INCLUDE, "regb200.h"), __file__]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _newest(deps):
        return OUT
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    hdr_time = float("inf") if force else _newest([os.path.join(CSRC, f) for f in hdr] +
                                                  [os.path.join(INCLUDE, "regb200.h"), __file__])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose or ptxas_info, extra, hdr_time), srcs))
    tmp = OUT + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + ["-lz", "-lpthread", "-ldl", "-lrt"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


def clean():
    if os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    if os.path.exists(OUT):
        os.remove(OUT)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args()
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose, ptxas_info=a.ptxas_info))
    sys.exit(0)
