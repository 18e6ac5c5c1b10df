"""GAE oracle pins and host-side checks (no GPU).

The C restatement (oracle/gae_oracle.c) must reproduce, bit for bit, the reference's own CPU
recurrence for the device GAE (RocketSimCuda/tests/test_gae_parity.cpp:24-81, compiled from
the reference tree) on the reference test's own case shapes, and the committed fixture that
recurrence wrote (tests/golden/gae_cases.npz).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT
from gae_util import (GAE_ORACLE, GAE_REF, REFERENCE_CASES, load_oracle, load_ref, make_case, run_oracle,
                      run_ref_cpu, same_bits)

GOLDEN = os.path.join(ROOT, "tests", "golden", "gae_cases.npz")


@pytest.fixture(scope="module")
def oracle():
    if not os.path.exists(GAE_ORACLE):
        pytest.fail(f"{GAE_ORACLE} missing: run `make -C oracle gae`")
    return load_oracle()


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(GAE_REF):
        pytest.fail(f"{GAE_REF} missing: run `make -C oracle gae` (needs the reference sources)")
    return load_ref()


@pytest.mark.parametrize("case", range(len(REFERENCE_CASES)))
def test_oracle_matches_reference_recurrence(oracle, ref, case):
    T, p, std, clip, end = REFERENCE_CASES[case]
    c = make_case(T, p, std, clip, end, seed=1234 + case)
    a, t, r, cp, st = run_oracle(oracle, c)
    ra, rt, rr, rcp = run_ref_cpu(ref, c)
    assert st == 0
    assert same_bits(a, ra) and same_bits(r, rr) and same_bits(t, rt)
    assert abs(cp - rcp) < 1e-4  # the reference test's own tolerance for the clip portion


def test_oracle_matches_reference_with_clipping(oracle, ref):
    """Rewards clipped after standardisation: the clip portion is nonzero."""
    c = make_case(30000, 1.0 / 60.0, 0.5, 1.5, True, seed=77)
    a, t, r, cp, st = run_oracle(oracle, c)
    ra, rt, rr, rcp = run_ref_cpu(ref, c)
    assert same_bits(a, ra) and same_bits(r, rr) and same_bits(t, rt)
    assert rcp > 0.1 and abs(cp - rcp) < 1e-4


def test_oracle_matches_golden_fixture(oracle):
    d = np.load(GOLDEN)
    for i in range(int(d["count"][0])):
        g, l, std, clip = (float(x) for x in d[f"c{i}_params"])
        c = dict(rews=d[f"c{i}_rews"], term=d[f"c{i}_term"], vals=d[f"c{i}_vals"], trunc=d[f"c{i}_trunc"], gamma=g,
                 lam=l, std=std, clip=clip)
        a, t, r, cp, st = run_oracle(oracle, c)
        assert st == 0
        assert same_bits(a, d[f"c{i}_adv"]) and same_bits(r, d[f"c{i}_ret"]) and same_bits(t, d[f"c{i}_tgt"]), i
        assert abs(cp - float(d[f"c{i}_clip"][0])) < 1e-4, i


def test_oracle_no_standardisation_portion_is_one(oracle):
    """With returnStd = 0 nothing is added to the clipped sum, so the portion is 1
    (GAECuda.cu:87-90 and :126-128)."""
    c = make_case(500, 0.02, 0.0, 3.0, True, seed=5)
    assert run_oracle(oracle, c)[3] == 1.0


def test_oracle_segments_reset_carries(oracle):
    """A NORMAL terminal zeroes the bootstrap, a TRUNCATED one bootstraps from its value,
    and neither carries the advantage of the step after it."""
    rews = np.array([1.0, 1.0, 1.0, 1.0], np.float32)
    vals = np.array([0.5, 0.5, 0.5, 0.5], np.float32)
    term = np.array([0, 1, 0, 2], np.int8)
    trunc = np.array([2.0], np.float32)
    c = dict(rews=rews, term=term, vals=vals, trunc=trunc, gamma=0.5, lam=1.0, std=0.0, clip=0.0)
    a, t, r, cp, st = run_oracle(oracle, c)
    f = np.float32
    d3 = f(1.0) + f(0.5) * f(2.0) - f(0.5)                 # truncated: bootstrap 2.0
    d2 = f(1.0) + f(0.5) * f(0.5) - f(0.5)                 # running: bootstrap vals[3]
    d1 = f(1.0) - f(0.5)                                   # normal end: bootstrap 0
    d0 = f(1.0) + f(0.5) * f(0.5) - f(0.5)
    assert a[3] == d3 and a[2] == d2 + f(0.5) * d3 and a[1] == d1 and a[0] == d0 + f(0.5) * d1
    assert r.tolist() == [1.5, 1.0, 1.5, 1.0]


def test_oracle_flags_a_short_truncation_list(oracle):
    c = make_case(400, 0.05, 1.0, 2.0, True, seed=9)
    assert len(c["trunc"]) >= 2
    st = run_oracle(oracle, c, num_truncs=len(c["trunc"]) - 1)[4]
    assert st == -1


def test_host_api_without_gpu(pkg):
    """The engine's GAE entry points check arguments first and, without a device, fail with
    RSB_ERR_CUDA instead of computing on the CPU."""
    import torch

    rsb = pkg.rsb
    lib = pkg.engine_library()
    p = rsb.gae_params(lib)
    assert abs(p.gamma - 0.99) < 1e-7 and abs(p.lam - 0.95) < 1e-7 and p.return_std == 0 and p.clip_range == 0
    with pytest.raises(rsb.RsbError) as e:
        rsb.compute_gae(lib, np.zeros(4), np.zeros(4, np.int8), np.zeros(4))  # final step running: needs T + 1 values
    assert e.value.code == -1
    st = lib.rsb_compute_gae(None, None, None, None, 0, None, None, None, None, -1, C.byref(p), None)
    assert st == -1
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(rsb.RsbError) as e:
        rsb.compute_gae(lib, np.zeros(4), np.array([0, 0, 0, 1], np.int8), np.zeros(4))
    assert e.value.code == -2
