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


def random_cars(rsb, cars, seed, speed_max=2300.0):
    """Cars on the ground at random places, headings, speeds and boost (the random-state
    reset distribution): `cars` is the array returned by Batch.get_cars()."""
    rng = np.random.default_rng(seed)
    c = cars.copy()
    n = len(c)
    yaw = rng.uniform(-np.pi, np.pi, n)
    cy, sy = np.cos(yaw), np.sin(yaw)
    c["pos"]["x"] = rng.uniform(-3500, 3500, n)
    c["pos"]["y"] = rng.uniform(-4500, 4500, n)
    c["pos"]["z"] = 17.0
    for f, v in (("forward", (cy, sy, 0 * cy)), ("right", (-sy, cy, 0 * cy)), ("up", (0 * cy, 0 * cy, 1 + 0 * cy))):
        for k, comp in enumerate("xyz"):
            c["rot"][f][comp] = v[k]
    sp = rng.uniform(0, speed_max, n)
    c["vel"]["x"], c["vel"]["y"], c["vel"]["z"] = cy * sp, sy * sp, 0.0
    for comp in "xyz":
        c["ang_vel"][comp] = 0.0
    c["boost"] = rng.uniform(0, 100, n)
    c["is_on_ground"] = 1
    return c


def random_controls(rsb, n, rng):
    """Discrete controls: throttle/steer/pitch/yaw/roll in {-1, 0, 1}, random buttons."""
    c = np.zeros(n, rsb.CONTROLS_DTYPE)
    for f in ("throttle", "steer", "pitch", "yaw", "roll"):
        c[f] = rng.integers(-1, 2, n).astype(np.float32)
    c["jump"] = rng.random(n) < 0.2
    c["boost"] = rng.random(n) < 0.4
    c["handbrake"] = rng.random(n) < 0.15
    return c


CAR_FLAGS = ("is_on_ground", "has_jumped", "has_double_jumped", "has_flipped", "is_flipping", "is_jumping",
             "is_supersonic", "is_auto_flipping", "is_demoed", "world_contact", "ball_hit_valid")


def flag_mismatch(a, b):
    """Per-car boolean: any discrete field differs (flags, wheel contacts, touch ticks, boost)."""
    bad = np.zeros(len(a), bool)
    for f in CAR_FLAGS:
        bad |= a[f] != b[f]
    bad |= (a["wheels_with_contact"] != b["wheels_with_contact"]).any(axis=1)
    bad |= a["ball_hit_tick"] != b["ball_hit_tick"]
    bad |= a["car_contact_other_id"] != b["car_contact_other_id"]
    return bad


def rot_matrix(a):
    return np.stack([vec(a["rot"], f) for f in ("forward", "right", "up")], axis=-2)


def reference_reverse_order(oracle_batch, pkg):
    """Arenas whose reference visits its cars in reverse creation order (the order the
    engine uses).  The reference keeps cars in an unordered_set of pointers, so in rare
    arenas (two cars in one hash bucket) the order differs from run to run."""
    import ctypes as C
    lib = oracle_batch.lib
    fn = lib.rsbref_car_order
    fn.restype = C.c_int32
    fn.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    ok = np.zeros(oracle_batch.num_arenas, bool)
    buf = np.zeros(8, np.int32)
    for a in range(oracle_batch.num_arenas):
        k = fn(oracle_batch._h, a, buf.ctypes.data)
        ok[a] = k >= 0 and np.array_equal(buf[:k], np.arange(k)[::-1])
    return ok
