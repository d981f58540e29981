"""Build libb200bssn.so in-tree with nvcc for sm_100a.

    python -m sympygr_b200.build            # library only
    python -m sympygr_b200.build --verbose  # also print ptxas register/spill report
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libb200bssn.so")

SOURCES = ["b200bssn.cu", "diagnostics.cu", "noalloc.cu", "rk4.cu", "guard.cu"]
HEADERS = ["rhs_kernels.cuh", "fused_kernel.cuh", "stencils.cuh", "plan_types.h", "plan_internal.h", "constraint_kernels.cuh",
           "generated/bssn_rhs_algebra.cuh", "generated/bssn_rhs_algebra_adv.cuh",
           "generated/bssn_constraints_algebra.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


SHIM_SRC = os.path.join(PKG, "shim", "bssnrhs_shim.cpp")
SHIM_LIB = os.path.join(LIBDIR, "libb200bssn_shim.so")


def build_shim(force: bool = False) -> str:
    """libb200bssn_shim.so: the C++ bssnrhs with the reference's signature, linked
    against libb200bssn.so; its bssn:: globals stay undefined (the host defines them)."""
    lib = build(force=False)
    if force or _stale(SHIM_LIB, [SHIM_SRC, lib, os.path.join(REPO, "include", "b200bssn.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", os.path.join(REPO, "include"),
               SHIM_SRC, "-L", LIBDIR, "-lb200bssn", "-Wl,-rpath,$ORIGIN", "-o", SHIM_LIB + ".tmp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("g++ failed building libb200bssn_shim.so")
        os.replace(SHIM_LIB + ".tmp", SHIM_LIB)
    return SHIM_LIB


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(REPO, "include", "b200bssn.h"), __file__]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-I", os.path.join(REPO, "include"), "-I", CSRC, "-o", LIB + ".tmp", *srcs,
           "-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libb200bssn.so")
    if verbose:
        sys.stdout.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))
    print(build_shim(force=a.force))
