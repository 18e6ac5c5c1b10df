"""The restated float functions of phys/refmath.h against the host's own: the x86 rsqrtss
estimate (through the 2 x 4096 table the engine samples and uploads) and the C library's
sinf / cosf / asinf / atan2f, whose results the reference's CPU build takes.  On the CPU the
host build of the restatements is compared on strided samples of all 2^32 floats; on the GPU
the device's results are compared with the host library on the same kind of sample."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from host_util import build_host_engine

FUNCS = {"rsqrt": 0, "sin": 1, "cos": 2, "asin": 3, "atan2": 4}


@pytest.fixture(scope="module")
def harness():
    lib = C.CDLL(build_host_engine())
    lib.rsb_host_refmath_check.restype = C.c_int64
    lib.rsb_host_refmath_check.argtypes = [C.c_int32, C.c_uint32, C.c_uint32, C.c_int32, C.POINTER(C.c_int64)]
    lib.rsb_host_libm.restype = C.c_int32
    lib.rsb_host_libm.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    return lib


@pytest.mark.parametrize("name", list(FUNCS))
def test_restatement_equals_host_library(harness, name):
    # every 61st float pattern (70 M inputs; a prime stride reaches every exponent and mantissa
    # residue), plus a dense band of small angles where sinf / cosf are evaluated every tick
    tested = C.c_int64()
    bad = harness.rsb_host_refmath_check(FUNCS[name], 61, 7, 8, C.byref(tested))
    assert tested.value > 10_000_000
    assert bad == 0, f"{name}: {bad} of {tested.value} inputs differ from the host library"
    if name in ("sin", "cos"):
        lo = np.float32(1e-4).view(np.uint32)
        bad = harness.rsb_host_refmath_check(FUNCS[name], 3, int(lo), 8, C.byref(tested))
        assert bad == 0, f"{name}: {bad} small-angle inputs differ"


def _host_values(harness, fn, x, y=None):
    out = np.empty_like(x)
    st = harness.rsb_host_libm(fn, x.ctypes.data, None if y is None else y.ctypes.data, out.ctypes.data, len(x))
    assert st == 0
    return out


def _sample(seed, n):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    x = bits.view(np.float32)
    x = x[np.isfinite(x)]
    small = rng.uniform(-0.1, 0.1, n // 4).astype(np.float32)
    unit = rng.uniform(-4, 4, n // 4).astype(np.float32)
    return np.concatenate([x, small, unit])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(FUNCS))
def test_device_equals_host_library(pkg, harness, meshes_dir, name):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    rsb.Batch(lib, 1, team_size=1, meshes_path=meshes_dir).close()  # loads the rsqrt table
    x = _sample(11 + FUNCS[name], 4_000_000)
    y = None
    if name in ("sin", "cos"):
        x = x[np.abs(x) < 120]
    if name == "atan2":
        y = np.random.default_rng(5).permutation(x)
    dev = rsb.eval_refmath(lib, FUNCS[name], x, y)
    host = _host_values(harness, FUNCS[name], x, y)
    same = (dev.view(np.uint32) == host.view(np.uint32)) | (np.isnan(dev) & np.isnan(host))
    assert same.all(), f"{name}: {int((~same).sum())} of {len(x)} differ, first x={x[~same][:3]}"
