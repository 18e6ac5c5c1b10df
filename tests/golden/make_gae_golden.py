"""Writes tests/golden/gae_cases.npz: GAE inputs and the outputs of the reference's own CPU
recurrence for them (RocketSimCuda/tests/test_gae_parity.cpp:24-81, compiled from the
reference tree into oracle/_ref/libgaeref.so by oracle/Makefile).

    make -C oracle gae && python tests/golden/make_gae_golden.py

The cases are smaller copies of the reference test's own cases (test_gae_parity.cpp:91-97)
plus one with real reward clipping and a NORMAL terminal at the first element.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from gae_util import load_ref, make_case, run_ref_cpu  # noqa: E402

CASES = [
    # (T, p_term, returnStd, clipRange, end truncated, seed)
    (5000, 1.0 / 300.0, 1.7, 4.0, True, 1),
    (3000, 1.0 / 50.0, 0.0, 0.0, True, 2),
    (1000, 0.0, 1.0, 2.0, False, 3),
    (777, 1.0 / 20.0, 1.0, 2.0, False, 4),
    (1, 0.0, 1.0, 2.0, True, 5),
    (2000, 1.0 / 40.0, 0.5, 1.5, True, 6),
]


def main():
    ref = load_ref()
    out = {}
    for i, (T, p, std, clip, end, seed) in enumerate(CASES):
        c = make_case(T, p, std, clip, end, seed)
        if i == 5:
            c["term"][0] = 1
            c["trunc"] = c["trunc"][:int((c["term"] == 2).sum())]
        adv, tgt, ret, cp = run_ref_cpu(ref, c)
        for k in ("rews", "term", "vals", "trunc"):
            out[f"c{i}_{k}"] = c[k]
        out[f"c{i}_params"] = np.array([c["gamma"], c["lam"], c["std"], c["clip"]], np.float32)
        out[f"c{i}_adv"], out[f"c{i}_tgt"], out[f"c{i}_ret"] = adv, tgt, ret
        out[f"c{i}_clip"] = np.array([cp], np.float32)
    out["count"] = np.array([len(CASES)])
    np.savez_compressed(os.path.join(HERE, "gae_cases.npz"), **out)


if __name__ == "__main__":
    main()
