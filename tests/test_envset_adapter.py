"""The CudaEnvSet-compatible adapter (include/rsb_envset.hpp), compiled against librsb.so and
checked step for step against the same collector step written as raw C-ABI calls in the
reference's order (tests/cpp/envset_adapter_test.cpp).  Without a GPU: it compiles, links, and
reports the missing device as an error."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from conftest import PKG_DIR, ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "envset_adapter_test.cpp")
EXE = os.path.join(ROOT, "tests", "_build", "envset_adapter_test")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA_HOME, "include"), SRC, "-L", PKG_DIR, "-lrsb", f"-Wl,-rpath,{PKG_DIR}",
           "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(CUDA_HOME, 'lib64')}",
           "-o", EXE]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def test_adapter_builds_and_reports_missing_device(pkg, meshes_dir):
    import torch

    exe = _build()
    if torch.cuda.is_available():
        pytest.skip("a GPU is present (the GPU test runs the adapter)")
    r = subprocess.run([exe, meshes_dir, "--no-gpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "adapter reports" in r.stdout


@pytest.mark.gpu
def test_adapter_equals_raw_abi_sequence(pkg, meshes_dir):
    exe = _build()
    r = subprocess.run([exe, meshes_dir], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "envset adapter ok" in r.stdout, r.stdout + r.stderr
