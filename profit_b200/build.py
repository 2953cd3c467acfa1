"""Builds profit_b200/lib/libprofit_b200.so for sm_100a with nvcc.

Each .cu file is its own translation unit so the FP64 parity kernels
(render64.cu) can be compiled with --fmad=false: libprofit's scalar C++ does
not contract a*b+c into fused multiply-adds, and the plain form must round
the same way to take the same subsampling decisions.

Usage:  python -m profit_b200.build  [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libprofit_b200.so")
PEAKS_LIB = os.path.join(LIBDIR, "libpf_peaks.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
          "-I" + CSRC, "--expt-relaxed-constexpr"]
UNITS = {
    # file: extra flags
    "render64.cu": ["--fmad=false"],
    "render32.cu": [],
    "fft.cu": [],
    "model.cu": ["--fmad=false"],
    "like_noalloc.cu": ["--fmad=false"],
    # the fit-space kernels round like the host copy of the same code (model.cu)
    "fitspace.cu": ["--fmad=false"],
}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_source() -> float:
    t = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            t = max(t, os.path.getmtime(os.path.join(d, f)))
    return max(t, os.path.getmtime(__file__))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.exists(PEAKS_LIB) and os.path.getmtime(LIB) >= _newest_source():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    objs: List[str] = []
    procs = []
    for unit, extra in UNITS.items():
        obj = os.path.join(OBJDIR, unit.replace(".cu", ".o"))
        cmd = [nvcc] + ARCH + COMMON + extra + ["-c", os.path.join(CSRC, unit), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((unit, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    for unit, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {unit}:\n{out.decode()}")
        elif verbose and out:
            print(out.decode())
    tmp = LIB + ".tmp"
    cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout.decode())
    os.replace(tmp, LIB)
    # FMA-throughput probe used by the benchmark for roofline denominators
    cmd = [nvcc] + ARCH + COMMON + ["-shared", "-o", PEAKS_LIB, os.path.join(CSRC, "peaks.cu")]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("peaks build failed:\n" + r.stdout.decode())
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
