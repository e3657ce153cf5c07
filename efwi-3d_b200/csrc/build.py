"""Builds efwi-3d_b200/libefwi.so (the C-ABI engine) with nvcc for sm_100a.

Usage: python efwi-3d_b200/csrc/build.py [--force] [--verbose]

Each .cu file is compiled separately (in parallel) into _build/ and linked
into one shared library next to the Python package, so that it travels with
the repository snapshot.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "libefwi.so")
BUILD = os.path.join(PKG, "_build")
SOURCES = ["efwi_fwd.cu", "efwi_fwd_tma.cu", "efwi_rev.cu", "efwi_rev_tma.cu", "efwi_aux.cu",
           "efwi_abi.cu", "efwi_noalloc.cu", "efwi_exact.cu", "efwi_cnn.cu"]
HEADERS = ["efwi_common.cuh", "efwi_kernels.h", "efwi_tma.cuh", "efwi_window.cuh", "efwi_exact.h",
           "efwi_revolve.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
           "--expt-relaxed-constexpr"]


def nvcc() -> str:
    cand = [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def host_compiler() -> list:
    # The image exports CXX pointing at a separate toolchain; nvcc is
    # validated against the system g++.
    if os.path.exists("/usr/bin/g++"):
        return ["-ccbin", "/usr/bin/g++"]
    return []


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(HERE, h) for h in HEADERS] + [os.path.join(ROOT, "include", "efwi.h")]
    cc = nvcc()
    extra = list(extra or [])

    def compile_one(src):
        s = os.path.join(HERE, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if not force and _newer(o, [s] + headers):
            return o, ""
        cmd = [cc] + host_compiler() + ARCH + NVFLAGS + extra + ["-I", HERE, "-I",
                                                                  os.path.join(ROOT, "include"),
                                                                  "-c", s, "-o", o]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return o, r.stderr

    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for o, log in results:
            if log:
                print(f"--- {os.path.basename(o)}\n{log}")
    if force or not _newer(OUT, objs):
        cmd = [cc] + host_compiler() + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
