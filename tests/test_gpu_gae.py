"""The engine's device GAE (rsb_compute_gae) against the oracle and the reference.

Advantages, returns and target values must be bit-identical to the C restatement
(oracle/gae_oracle.c) and to the reference's own device function, rsc::ComputeGAEOnDevice
built for sm_100a from the reference tree (oracle/_ref/libgaeref.so); the clip portion agrees
within 1e-4, the reference test's tolerance (its sums are added in another order).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from gae_util import CHUNK, GAE_REF, REFERENCE_CASES, load_oracle, load_ref, make_case, run_oracle, same_bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def oracle():
    return load_oracle()


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(GAE_REF):
        pytest.skip("the reference's GAE library was not built")
    return load_ref()


def _dev(torch, c):
    T = len(c["rews"])
    d = dict(rews=torch.from_numpy(c["rews"]).cuda(), term=torch.from_numpy(c["term"]).cuda(),
             vals=torch.from_numpy(c["vals"]).cuda(),
             trunc=torch.from_numpy(c["trunc"] if len(c["trunc"]) else np.zeros(1, np.float32)).cuda())
    for k in ("adv", "tgt", "ret"):
        d[k] = torch.full((max(T, 1),), float("nan"), device="cuda")
    d["clip"] = torch.full((1,), float("nan"), device="cuda")
    return d


def run_engine(pkg, torch, c, num_truncs=None, stream=None):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    d = _dev(torch, c)
    T = len(c["rews"])
    p = rsb.gae_params(lib, gamma=c["gamma"], lam=c["lam"], return_std=c["std"], clip_range=c["clip"])
    nt = len(c["trunc"]) if num_truncs is None else num_truncs
    rsb.compute_gae_device(lib, d["rews"].data_ptr(), d["term"].data_ptr(), d["vals"].data_ptr(),
                           d["trunc"].data_ptr(), nt, d["adv"].data_ptr(), d["tgt"].data_ptr(), d["ret"].data_ptr(),
                           d["clip"].data_ptr(), T, p, stream or torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return (d["adv"][:T].cpu().numpy(), d["tgt"][:T].cpu().numpy(), d["ret"][:T].cpu().numpy(),
            float(d["clip"].item()))


def run_reference_device(ref, torch, c):
    d = _dev(torch, c)
    T = len(c["rews"])
    st = ref.gaeref_device(d["rews"].data_ptr(), d["term"].data_ptr(), d["vals"].data_ptr(),
                           d["trunc"].data_ptr() if len(c["trunc"]) else None, len(c["trunc"]), d["adv"].data_ptr(),
                           d["tgt"].data_ptr(), d["ret"].data_ptr(), d["clip"].data_ptr(), T, c["gamma"], c["lam"],
                           c["std"], c["clip"], None)
    torch.cuda.synchronize()
    assert st == 0
    return (d["adv"][:T].cpu().numpy(), d["tgt"][:T].cpu().numpy(), d["ret"][:T].cpu().numpy(),
            float(d["clip"].item()))


def _check(got, want, what=""):
    a, t, r, cp = got
    wa, wt, wr, wcp = want[:4]
    assert same_bits(a, wa), f"{what}: advantages differ at {np.nonzero(a.view(np.uint32) != wa.view(np.uint32))[0][:5]}"
    assert same_bits(r, wr), f"{what}: returns differ"
    assert same_bits(t, wt), f"{what}: target values differ"
    assert abs(cp - wcp) < 1e-4, f"{what}: clip portion {cp} vs {wcp}"


@pytest.mark.parametrize("case", range(len(REFERENCE_CASES)))
def test_reference_cases_match_oracle_and_reference_device(pkg, torch_cuda, oracle, ref, case):
    T, p, std, clip, end = REFERENCE_CASES[case]
    c = make_case(T, p, std, clip, end, seed=4321 + case)
    got = run_engine(pkg, torch_cuda, c)
    _check(got, run_oracle(oracle, c), "oracle")
    _check(got, run_reference_device(ref, torch_cuda, c), "reference device GAE")


def test_clipping_and_chunk_spanning_segments(pkg, torch_cuda, oracle, ref):
    """Rewards clipped after standardisation; segments far longer than a block's chunk."""
    c = make_case(7 * CHUNK + 123, 1.0 / 9000.0, 0.5, 1.5, False, seed=11)
    _check(run_engine(pkg, torch_cuda, c), run_oracle(oracle, c), "oracle")
    _check(run_engine(pkg, torch_cuda, c), run_reference_device(ref, torch_cuda, c), "reference device GAE")


def test_terminals_on_chunk_edges(pkg, torch_cuda, oracle, ref):
    T = 4 * CHUNK + 17
    c = make_case(T, 0.0, 1.3, 0.9, True, seed=12)
    for pos, kind in ((0, 1), (CHUNK - 1, 2), (CHUNK, 1), (2 * CHUNK - 1, 1), (2 * CHUNK, 2), (3 * CHUNK + 1, 2)):
        c["term"][pos] = kind
    c["trunc"] = np.random.default_rng(3).uniform(-2, 2, int((c["term"] == 2).sum())).astype(np.float32)
    _check(run_engine(pkg, torch_cuda, c), run_oracle(oracle, c), "oracle")
    _check(run_engine(pkg, torch_cuda, c), run_reference_device(ref, torch_cuda, c), "reference device GAE")


def test_every_step_terminal_and_no_terminal(pkg, torch_cuda, oracle, ref):
    for p, end, seed in ((1.0, True, 13), (0.0, False, 14)):
        c = make_case(3 * CHUNK + 5, p, 1.0, 2.0, end, seed=seed)
        _check(run_engine(pkg, torch_cuda, c), run_oracle(oracle, c), f"p={p}")
        _check(run_engine(pkg, torch_cuda, c), run_reference_device(ref, torch_cuda, c), f"p={p} reference")


def test_other_nonzero_terminals_end_segments(pkg, torch_cuda, oracle, ref):
    """A terminal value other than 1 / 2 ends a segment but bootstraps from the next value
    (GAECuda.cu:31 marks every nonzero terminal)."""
    c = make_case(20000, 1.0 / 100.0, 1.0, 2.0, True, seed=15)
    c["term"][np.random.default_rng(1).choice(19999, 40, replace=False)] = 3
    c["trunc"] = c["trunc"][:int((c["term"] == 2).sum())]
    _check(run_engine(pkg, torch_cuda, c), run_oracle(oracle, c), "oracle")
    _check(run_engine(pkg, torch_cuda, c), run_reference_device(ref, torch_cuda, c), "reference device GAE")


def test_empty_and_single(pkg, torch_cuda, oracle):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    clip = torch_cuda.full((1,), 5.0, device="cuda")
    p = rsb.gae_params(lib)
    rsb.compute_gae_device(lib, 0, 0, 0, 0, 0, 0, 0, 0, clip.data_ptr(), 0, p)
    torch_cuda.cuda.synchronize()
    assert clip.item() == 0.0
    for end in (True, False):
        c = make_case(1, 0.0, 0.0, 0.0, end, seed=16)
        c["term"][0] = 2 if end else 0
        _check(run_engine(pkg, torch_cuda, c), run_oracle(oracle, c), f"T=1 end={end}")


def test_short_truncation_list_reads_nothing_out_of_range(pkg, torch_cuda, oracle):
    """num_truncs below the TRUNCATED count: the extra truncations bootstrap from 0, as in the
    oracle (the reference would read before the array; it is not run on such input)."""
    c = make_case(9000, 1.0 / 30.0, 1.0, 2.0, True, seed=17)
    nt = len(c["trunc"]) - 3
    got = run_engine(pkg, torch_cuda, c, num_truncs=nt)
    want = run_oracle(oracle, c, num_truncs=nt)
    assert want[4] == -1
    _check(got, want, "short list")


def test_rollout_sized_buffer(pkg, torch_cuda, oracle):
    """393,216 player trajectories of 32 steps (3v3 x 65,536 arenas), each truncated at the
    rollout's end, goals at random: bit-identical to the oracle over 12.6 M elements."""
    players, steps = 393216, 32
    rng = np.random.default_rng(18)
    T = players * steps
    term = np.zeros((players, steps), np.int8)
    term[rng.random((players, steps)) < 1.0 / 300.0] = 1
    term[:, -1] = 2
    c = dict(rews=rng.standard_normal(T).astype(np.float32), term=term.ravel(),
             vals=rng.standard_normal(T).astype(np.float32),
             trunc=rng.standard_normal(int((term == 2).sum())).astype(np.float32),
             gamma=0.99, lam=0.95, std=1.7, clip=4.0)
    _check(run_engine(pkg, torch_cuda, c), run_oracle(oracle, c), "rollout")


def test_host_entry_point_and_stream(pkg, torch_cuda, oracle):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    c = make_case(50000, 1.0 / 77.0, 1.7, 1.0, False, seed=19)
    p = rsb.gae_params(lib, return_std=c["std"], clip_range=c["clip"])
    host = rsb.compute_gae(lib, c["rews"], c["term"], c["vals"], c["trunc"], p)
    _check(host, run_oracle(oracle, c), "host entry point")
    s = torch_cuda.cuda.Stream()
    with torch_cuda.cuda.stream(s):
        dev = run_engine(pkg, torch_cuda, c, stream=s.cuda_stream)
    _check(dev, host, "side stream")
