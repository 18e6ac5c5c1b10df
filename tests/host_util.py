"""Builds the host harness (tests/cpp/host_engine.cpp): the engine's physics headers
compiled with g++ behind part of the C ABI, used by the CPU parity tests."""
from __future__ import annotations

import os
import shutil
import subprocess

from conftest import PKG_DIR, ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "host_engine.cpp")
ARENA_BUILD = os.path.join(PKG_DIR, "csrc", "arena_build.cpp")
LIB = os.path.join(ROOT, "tests", "_build", "librsbhost.so")


def _deps():
    out = [SRC, ARENA_BUILD, os.path.join(ROOT, "include", "rsb.h")]
    for d in (os.path.join(PKG_DIR, "csrc"), os.path.join(PKG_DIR, "csrc", "phys")):
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return out


def build_host_engine() -> str:
    """Compiles (when stale) and returns the path of librsbhost.so.  Same code generation as
    the reference's CPU build: x86-64 SSE2, no FMA, no contraction."""
    if os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in _deps()):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", "-ffp-contract=off",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG_DIR, "csrc"),
           SRC, ARENA_BUILD, "-o", LIB + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("host harness build failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(LIB + ".tmp", LIB)
    return LIB
