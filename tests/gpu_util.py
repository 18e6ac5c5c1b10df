"""Helpers shared by the GPU parity tests."""
from __future__ import annotations

import numpy as np

# Per-quantity tolerance of the parity tests: |engine - oracle| <= ABS + REL * |oracle|
POS_ABS_UU = 1e-2
VEL_ABS_UU = 1e-2
REL = 1e-4


def identity_rot(arr):
    for k, f in enumerate(("forward", "right", "up")):
        for c in "xyz":
            arr["rot"][f][c] = 1.0 if "xyz"[k] == c else 0.0


def random_balls(rsb, n, seed, rest_fraction=0.25):
    rng = np.random.default_rng(seed)
    b = np.zeros(n, rsb.BALL_DTYPE)
    identity_rot(b)
    b["pos"]["x"] = rng.uniform(-3900, 3900, n)
    b["pos"]["y"] = rng.uniform(-5000, 5000, n)
    b["pos"]["z"] = rng.uniform(100, 1900, n)
    rest = rng.random(n) < rest_fraction
    b["pos"]["z"][rest] = 93.15 + rng.uniform(0, 10, rest.sum())
    for c in "xyz":
        b["vel"][c] = rng.uniform(-3000, 3000, n)
        b["ang_vel"][c] = rng.uniform(-5, 5, n)
    return b


def vec(arr, field):
    return np.stack([arr[field][c] for c in "xyz"], axis=-1).astype(np.float64)


def max_excess(a, b, abs_tol, rel=REL):
    """Largest violation of |a-b| <= abs_tol + rel*|b| (<= 0 means within tolerance)."""
    d = np.abs(a - b)
    return float((d - (abs_tol + rel * np.abs(b))).max())
