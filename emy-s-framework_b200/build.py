"""Builds the engine library (librsb.so) for sm_100a with nvcc, in place.

The physics headers are compiled with FMA contraction disabled (--fmad=false), so that
every multiply and add rounds separately as in the reference simulator's x86 build.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "librsb.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["rsb_engine.cu", "gae.cu"]
CPP_SOURCES = ["arena_build.cpp"]


def _headers() -> list[str]:
    out = [os.path.join(ROOT, "include", "rsb.h")]
    for d in (CSRC, os.path.join(CSRC, "phys")):
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} (exit {r.returncode})")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    """Compiles the engine if any source changed; returns the library path."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    hdrs = _headers()
    objs = []
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cxx = shutil.which("g++") or "g++"
            _run([cxx, "-std=c++17", "-O2", "-fPIC", "-c", s, "-o", o] + inc, verbose)
        objs.append(o)
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
                   "--extended-lambda", "-c", s, "-o", o] + inc
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose or ptxas_info)
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-Xlinker", "-Bsymbolic", "-o", LIB] + objs + ["-lcudart"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv, force="--force" in sys.argv)
    print(LIB)
