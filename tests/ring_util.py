"""A Python model of the reference state ring's restore draws (CudaEnvSet.cpp:608-617 and
:755-800): which arenas a restore picks, which slot it reads, and the xorshift32 state at the
first jitter draw of every picked arena.  float32 arithmetic as the reference computes it."""
from __future__ import annotations

import math

import numpy as np

M32 = 0xFFFFFFFF
F = np.float32


def rand01(state: int):
    s = state
    s ^= (s << 13) & M32
    s ^= s >> 17
    s ^= (s << 5) & M32
    return s, F(s & 0xFFFFFF) / F(0xFFFFFF)


def rand_range(state: int, lo, hi):
    s, r = rand01(state)
    lo, hi = F(lo), F(hi)
    return s, F(lo + F(hi - lo) * r)


def lround(x: float) -> int:
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def plan_restore(cars_per_arena, cfg, filled, write_idx, rng, frac=-1.0, lookback=-1, fuzz_scale=1.0,
                 max_arenas=-1):
    """(slot, [(arena, xorshift state at its first jitter draw)], rng after the restore)."""
    n = len(cars_per_arena)
    frac = F(frac) if frac >= 0 else F(cfg["restore_fraction"])
    frac = max(F(0.01), min(F(0.05), frac))
    lookback = lookback if lookback >= 0 else cfg["lookback_slots"]
    lookback = max(1, min(lookback, filled - 1))
    last = write_idx - 1
    if last < 0:
        last = cfg["depth"] - 1
    slot = last - lookback
    while slot < 0:
        slot += cfg["depth"]
    cap = max_arenas if max_arenas > 0 else cfg["max_arenas_per_restore"]
    cap = min(cap, max(1, lround(0.05 * n)))
    k = max(1, lround(float(frac) * n))
    k = min(k, n, cap)
    order = list(range(n))
    for i in range(k):
        rng, r = rand01(rng)
        j = i + int(F(r * F(n - i)))
        if j >= n:
            j = n - 1
        order[i], order[j] = order[j], order[i]
    fp = F(F(cfg["fuzz_pos"]) * F(fuzz_scale))
    fv = F(F(cfg["fuzz_vel"]) * F(fuzz_scale))
    per_body = (3 if fp > 0 else 0) + (3 if fv > 0 else 0)
    jobs = []
    for i in range(k):
        a = order[i]
        jobs.append((a, rng))
        for _ in range((cars_per_arena[a] + 1) * per_body):
            rng, _ = rand01(rng)
    return slot, jobs, rng


def jitter(state: int, pos, vel, fp, fv, z_floor, z_lo, z_hi):
    """One body's jittered position and velocity (ApplyArenaSnap, CudaEnvSet.cpp:708-743)."""
    pos = [F(x) for x in pos]
    vel = [F(x) for x in vel]
    fp, fv = F(fp), F(fv)
    if fp > 0:
        state, d = rand_range(state, -fp, fp)
        pos[0] = F(pos[0] + d)
        state, d = rand_range(state, -fp, fp)
        pos[1] = F(pos[1] + d)
        state, d = rand_range(state, F(-fp * F(z_lo)), F(fp * F(z_hi)))
        z = F(pos[2] + d)
        pos[2] = z if F(z_floor) < z else F(z_floor)
    if fv > 0:
        state, d = rand_range(state, -fv, fv)
        vel[0] = F(vel[0] + d)
        state, d = rand_range(state, -fv, fv)
        vel[1] = F(vel[1] + d)
        state, d = rand_range(state, F(-fv * F(0.5)), F(fv * F(0.5)))
        vel[2] = F(vel[2] + d)
    return state, pos, vel
