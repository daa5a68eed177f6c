"""Build recipe for libhplb200.so (sm_100a) and the hplb command-line driver.

Everything is compiled in-tree with nvcc so the shared library travels with
the source snapshot; there is no JIT step at import time.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libhplb200.so")
CLI = os.path.join(PKG, "hplb")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _cuda_home() -> str:
    nv = _nvcc()
    if os.path.isabs(nv):
        return os.path.dirname(os.path.dirname(nv))
    return os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = _sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(
        os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    if force or _stale(LIB, deps):
        objdir = os.path.join(PKG, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        procs = []
        for src in _sources():
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            objs.append(obj)
            if force or _stale(obj, [src] + deps[len(_sources()):]):
                cmd = [_nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
                if verbose:
                    print(" ".join(cmd))
                procs.append((src, subprocess.Popen(cmd)))
        for src, p in procs:
            if p.wait() != 0:
                raise RuntimeError(f"nvcc failed on {src}")
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.check_call(cmd)
    cli_src = os.path.join(PKG, "cli", "hplb_main.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB])):
        cuda = _cuda_home()
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, "-I", os.path.join(cuda, "include"),
               cli_src, "-o", CLI, "-L", PKG, "-lhplb200", "-Wl,-rpath,$ORIGIN",
               "-L", os.path.join(cuda, "lib64"), "-lcudart"]
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
