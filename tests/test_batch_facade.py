"""The C++ facade with the reference batch class's method names (include/rsb_batch.hpp),
compiled against librsb.so and driven the way CudaEnvSet drives the reference batch
(tests/cpp/batch_facade_test.cpp).  Without a GPU: it compiles, links, and reports the missing
device as an error.  On the GPU: its results equal the C ABI's, step for step."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from conftest import PKG_DIR, ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "batch_facade_test.cpp")
EXE = os.path.join(ROOT, "tests", "_build", "batch_facade_test")


def _build():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", PKG_DIR, "-lrsb", f"-Wl,-rpath,{PKG_DIR}", "-o", EXE]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def test_facade_builds_and_reports_missing_device(pkg, meshes_dir):
    import torch

    exe = _build()
    if torch.cuda.is_available():
        pytest.skip("a GPU is present (the GPU test runs the facade)")
    r = subprocess.run([exe, meshes_dir, "--no-gpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "facade reports" in r.stdout


@pytest.mark.gpu
def test_facade_equals_c_abi(pkg, meshes_dir):
    exe = _build()
    r = subprocess.run([exe, meshes_dir], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "facade ok" in r.stdout, r.stdout + r.stderr
