"""GAE test helpers: the oracle libraries behind ctypes and input generators.

libgaeoracle.so is the C restatement of the reference's device GAE (oracle/gae_oracle.c);
libgaeref.so holds the reference's own code compiled from its tree (oracle/gae_pin.cpp):
the CPU recurrence of RocketSimCuda/tests/test_gae_parity.cpp:24-81 and
rsc::ComputeGAEOnDevice (RocketSimCuda/src/GAECuda.cu:247-300).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from conftest import ROOT

GAE_ORACLE = os.path.join(ROOT, "oracle", "_ref", "libgaeoracle.so")
GAE_REF = os.path.join(ROOT, "oracle", "_ref", "libgaeref.so")
CHUNK = 4096  # elements per block of the engine's segment kernel

_P = C.c_void_p
_F = C.c_float
_I = C.c_int32

# (T, terminal probability, returnStd, clipRange, final step truncated) — the cases of the
# reference's GAE parity test (RocketSimCuda/tests/test_gae_parity.cpp:91-97)
REFERENCE_CASES = [
    (200000, 1.0 / 300.0, 1.7, 4.0, True),
    (50000, 1.0 / 50.0, 0.0, 0.0, True),
    (1000, 0.0, 1.0, 2.0, False),
    (777, 1.0 / 20.0, 1.0, 2.0, False),
    (1, 0.0, 1.0, 2.0, True),
]


def load_oracle():
    lib = C.CDLL(GAE_ORACLE)
    lib.gae_oracle.restype = C.c_int
    lib.gae_oracle.argtypes = [_P, _P, _P, _P, _I, _P, _P, _P, _P, _I, _F, _F, _F, _F]
    return lib


def load_ref():
    lib = C.CDLL(GAE_REF)
    lib.gaeref_cpu.restype = C.c_int
    lib.gaeref_cpu.argtypes = [_P, _P, _P, _I, _P, _I, _I, _F, _F, _F, _F, _P, _P, _P, _P]
    lib.gaeref_device.restype = C.c_int
    lib.gaeref_device.argtypes = [_P, _P, _P, _P, _I, _P, _P, _P, _P, _I, _F, _F, _F, _F, _P]
    return lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else None


def make_case(T, p_term, return_std, clip_range, end_terminal, seed, trunc_share=0.4, values=(-2.0, 2.0)):
    """Inputs shaped as the reference test draws them: rewards and values U(-2, 2), a terminal
    with probability p_term (TRUNCATED with probability 0.4, else NORMAL), the final step
    TRUNCATED or running; a running final step gets the extra value the recurrence reads."""
    rng = np.random.default_rng(seed)
    rews = rng.uniform(*values, T).astype(np.float32)
    vals = rng.uniform(*values, T).astype(np.float32)
    term = np.zeros(T, np.int8)
    hit = rng.random(T) < p_term
    kind = np.where(rng.random(T) < trunc_share, 2, 1).astype(np.int8)
    term[hit] = kind[hit]
    if T > 0:
        if end_terminal:
            term[T - 1] = 2
        elif T > 1:
            term[T - 1] = 0
    if T > 0 and term[T - 1] == 0:
        vals = np.append(vals, np.float32(0.0))
    nt = int((term == 2).sum())
    trunc = rng.uniform(*values, nt).astype(np.float32)
    return dict(rews=rews, term=term, vals=vals, trunc=trunc, gamma=0.99, lam=0.95, std=return_std, clip=clip_range)


def run_oracle(lib, c, num_truncs=None):
    T = len(c["rews"])
    nt = len(c["trunc"]) if num_truncs is None else num_truncs
    adv, tgt, ret = (np.zeros(T, np.float32) for _ in range(3))
    clip = np.zeros(1, np.float32)
    st = lib.gae_oracle(_p(c["rews"]), _p(c["term"]), _p(c["vals"]), _p(c["trunc"]), nt, _p(adv), _p(tgt), _p(ret),
                        _p(clip), T, c["gamma"], c["lam"], c["std"], c["clip"])
    return adv, tgt, ret, float(clip[0]), st


def run_ref_cpu(lib, c):
    T = len(c["rews"])
    adv, tgt, ret = (np.zeros(T, np.float32) for _ in range(3))
    clip = np.zeros(1, np.float32)
    st = lib.gaeref_cpu(_p(c["rews"]), _p(c["term"]), _p(c["vals"]), len(c["vals"]), _p(c["trunc"]), len(c["trunc"]),
                        T, c["gamma"], c["lam"], c["std"], c["clip"], _p(adv), _p(tgt), _p(ret), _p(clip))
    assert st == 0
    return adv, tgt, ret, float(clip[0])


def same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))
