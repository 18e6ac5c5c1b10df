"""The oracle's state ring (the reference CudaEnvSet ring restated on RocketSim arenas) against
the Python model of its draws (tests/ring_util.py), on the CPU."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import random_balls, random_cars, vec
from ring_util import F, jitter, plan_restore


def _batch(pkg, oracle_lib, meshes_dir, n, seed, team_sizes=None, team_size=2):
    rsb = pkg.rsb
    b = rsb.Batch(oracle_lib, n, team_size=None if team_sizes is not None else team_size, team_sizes=team_sizes,
                  meshes_path=meshes_dir, threads=4)
    b.set_cars(random_cars(rsb, b.get_cars(), seed))
    b.set_balls(random_balls(rsb, n, seed + 1))
    return b


def _controls(pkg, b, seed):
    rng = np.random.default_rng(seed)
    c = np.zeros(b.num_cars, pkg.rsb.CONTROLS_DTYPE)
    c["throttle"] = 1.0
    c["steer"] = rng.uniform(-1, 1, b.num_cars)
    c["boost"] = rng.integers(0, 2, b.num_cars)
    return c


def test_restore_picks_the_modelled_arenas_and_jitter(pkg, oracle_lib, meshes_dir):
    n = 120
    ts = np.array([1, 2, 3] * (n // 3), np.int32)
    b = _batch(pkg, oracle_lib, meshes_dir, n, 5, team_sizes=ts)
    cfg = b.ring_configure(depth=4, capture_every=1, lookback_slots=2, seed=0x1234567)
    snaps = []
    for k in range(5):
        b.set_controls(_controls(pkg, b, k))
        b.step(8)
        snaps.append((b.get_cars(), b.get_balls(), b.get_pads()))
        b.ring_maybe_capture()
    st = b.ring_stats()
    assert st["filled"] == 4 and st["captures"] == 5 and st["write_idx"] == 1
    before = (b.get_cars(), b.get_balls(), b.get_pads())
    c = {k: getattr(cfg, k) for k, _ in type(cfg)._fields_}
    slot, jobs, _ = plan_restore([2 * t for t in ts], c, st["filled"], st["write_idx"], cfg.seed)
    got = b.ring_restore()
    assert got == len(jobs) == 6  # 5 % of 120
    # slot k holds the capture made after env step (capture index) with slot = capture % depth
    cap_index = [i for i in range(5) if i % 4 == slot][-1]
    cars0, balls0, pads0 = snaps[cap_index]
    cars1, balls1, pads1 = b.get_cars(), b.get_balls(), b.get_pads()
    picked = {a for a, _ in jobs}
    off = b.car_offset
    for a in range(n):
        sl = slice(off[a], off[a + 1])
        if a not in picked:
            assert cars1[sl].tobytes() == before[0][sl].tobytes()
            assert balls1[a].tobytes() == before[1][a].tobytes()
            continue
        state = dict(jobs)[a]
        for i in range(off[a], off[a + 1]):
            state, p, v = jitter(state, vec(cars0[i], "pos"), vec(cars0[i], "vel"), cfg.fuzz_pos, cfg.fuzz_vel,
                                 17.0, 0.25, 0.35)
            # the setters convert uu -> Bullet units and back, a rounding of a few ulp
            assert np.allclose(vec(cars1[i], "pos"), p, rtol=1e-6, atol=1e-3)
            assert np.allclose(vec(cars1[i], "vel"), v, rtol=1e-6, atol=1e-3)
        state, p, v = jitter(state, vec(balls0[a], "pos"), vec(balls0[a], "vel"), cfg.fuzz_pos, cfg.fuzz_vel,
                             93.0, 0.2, 0.4)
        assert np.allclose(vec(balls1[a], "pos"), p, rtol=1e-6, atol=1e-3)
        assert np.allclose(vec(balls1[a], "vel"), v, rtol=1e-6, atol=1e-3)
        assert pads1[a * 34:(a + 1) * 34].tobytes() == pads0[a * 34:(a + 1) * 34].tobytes()


@pytest.fixture(scope="module")
def batches(pkg, oracle_lib, meshes_dir):
    return {n: pkg.rsb.Batch(oracle_lib, n, team_size=1, meshes_path=meshes_dir, threads=8) for n in (10, 60, 200)}


@pytest.mark.parametrize("n,frac,cap,expect", [(200, 0.05, 64, 10), (200, 0.2, 64, 10), (200, 0.001, 64, 2),
                                               (200, 0.05, 3, 3), (60, 0.05, 64, 3), (10, 0.05, 64, 1)])
def test_restore_counts(batches, n, frac, cap, expect):
    """At least 1 %, at most 5 % of the arenas, at most max_arenas (CudaEnvSet.cpp:760-785)."""
    b = batches[n]
    b.ring_configure(depth=3, capture_every=1, max_arenas_per_restore=cap, fuzz_pos=0.0, fuzz_vel=0.0)
    assert b.ring_restore() == 0  # nothing captured yet
    b.ring_capture()
    assert b.ring_restore() == 0  # one capture: nothing to look back to
    b.ring_capture()
    assert b.ring_restore(restore_fraction=frac) == expect


def test_tripwire_and_disable(pkg, oracle_lib, meshes_dir):
    b = pkg.rsb.Batch(oracle_lib, 40, team_size=1, meshes_path=meshes_dir, threads=2)
    b.ring_configure(depth=2, capture_every=2)
    for _ in range(4):
        b.ring_maybe_capture()
    assert b.ring_stats()["captures"] == 2
    for k in range(33):
        assert b.ring_restore() == 2
    st = b.ring_stats()
    assert st["replay_disabled"] == 1 and st["restore_calls"] == 33
    assert b.ring_restore() == 0
    b.ring_configure(depth=0)
    assert b.ring_stats()["depth"] == 0


def test_configure_clamps_like_the_reference(pkg, oracle_lib, meshes_dir):
    b = pkg.rsb.Batch(oracle_lib, 8, team_size=1, meshes_path=meshes_dir, threads=1)
    b.ring_configure(depth=1, capture_every=0, lookback_slots=9)
    for _ in range(3):
        b.ring_maybe_capture()
    st = b.ring_stats()
    assert st["depth"] == 2 and st["captures"] == 3 and st["filled"] == 2
