"""Build the engine's shared library in-tree for sm_100a.

    python -m cudamica_b200.build          # -> cudamica_b200/libamica_b200.so
    python -m cudamica_b200.build --cli    # also the cudaamica-compatible CLI

One nvcc invocation per source (parallel), linked into a single C-ABI shared
library; no torch types cross the boundary.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libamica_b200.so")
CLI = os.path.join(PKG, "cudaamica")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
SOURCES = ["engine.cu", "mstep.cu", "estep_plain.cu", "estep_tc.cu", "estep_tc_wg2.cu", "gemm_tc.cu",
           "preprocess.cu", "adjoint.cu", "estep_noalloc.cu", "estep_dens.cu"]


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    inp = os.path.join(CSRC, src)
    # every shared header and included kernel body can change any object
    deps = [inp, os.path.join(ROOT, "include", "amica_b200.h")] + [
        os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".inc"))]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps
                                   if os.path.exists(d)):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-c", inp, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, cli: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if (not os.path.exists(LIB)) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "--cudart=static", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if cli and os.path.exists(os.path.join(CSRC, "cli.cpp")):
        src = os.path.join(CSRC, "cli.cpp")
        if (not os.path.exists(CLI)) or os.path.getmtime(src) > os.path.getmtime(CLI) or \
                os.path.getmtime(LIB) > os.path.getmtime(CLI):
            cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), src, "-o", CLI,
                   "-L" + PKG, "-lamica_b200", "-Wl,-rpath,$ORIGIN"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas resource usage")
    args = ap.parse_args()
    print(build(verbose=args.verbose))
