"""The engine's device state ring against the oracle's (the reference CudaEnvSet ring restated
on RocketSim arenas).

Both sides hold bit-identical public state before every capture (the oracle's state is
written into both after each env step), so the captured slots agree; a restore must then
leave every car, ball and pad of both batches bit-identical, rewound arenas included (the
same arenas, the same jitter draws, the same Get/SetState conversions), and one env step
after it must stay within the per-tick parity bounds.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import random_balls, random_cars, reference_reverse_order, vec
from ring_util import plan_restore

pytestmark = pytest.mark.gpu


def _pair(pkg, oracle_lib, meshes_dir, n, seed, team_sizes):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), n, team_size=None, team_sizes=team_sizes, meshes_path=meshes_dir)
    ora = rsb.Batch(oracle_lib, n, team_size=None, team_sizes=team_sizes, meshes_path=meshes_dir, threads=8)
    cars, balls = random_cars(rsb, ora.get_cars(), seed), random_balls(rsb, n, seed + 1)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    return eng, ora


def _sync(eng, ora):
    cars, balls, pads = ora.get_cars(), ora.get_balls(), ora.get_pads()
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
        b.set_pads(pads)


def _same(eng, ora):
    for get in ("get_cars", "get_balls", "get_pads"):
        a, b = getattr(eng, get)(), getattr(ora, get)()
        bad = np.nonzero(a.view(np.uint8).reshape(len(a), -1) != b.view(np.uint8).reshape(len(b), -1))
        assert a.tobytes() == b.tobytes(), f"{get}: records differ at {np.unique(bad[0])[:8]}"


def _drive(pkg, eng, ora, steps, seed, capture=True):
    rng = np.random.default_rng(seed)
    for _ in range(steps):
        c = np.zeros(ora.num_cars, pkg.rsb.CONTROLS_DTYPE)
        c["throttle"] = 1.0
        c["steer"] = rng.uniform(-1, 1, ora.num_cars)
        c["boost"] = rng.integers(0, 2, ora.num_cars)
        c["jump"] = rng.random(ora.num_cars) < 0.1
        for b in (eng, ora):
            b.set_controls(c)
            b.step(8)
        _sync(eng, ora)
        if capture:
            for b in (eng, ora):
                b.ring_maybe_capture()


@pytest.mark.parametrize("fuzz_scale", [1.0, 0.0, 3.5])
def test_restore_matches_oracle_bit_for_bit(pkg, oracle_lib, meshes_dir, fuzz_scale):
    n = 300
    ts = np.array([1, 2, 3] * (n // 3), np.int32)
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, n, 40, ts)
    for b in (eng, ora):
        b.ring_configure(depth=5, capture_every=2, lookback_slots=3, seed=0xBEEF1234)
    _drive(pkg, eng, ora, 9, seed=1)
    assert eng.ring_stats() == ora.ring_stats()
    cfg = eng._ring_cfg
    st = eng.ring_stats()
    c = {k: getattr(cfg, k) for k, _ in type(cfg)._fields_}
    _, jobs, _ = plan_restore([2 * t for t in ts], c, st["filled"], st["write_idx"], cfg.seed, fuzz_scale=fuzz_scale)
    before = eng.get_cars()
    ne = eng.ring_restore(fuzz_scale=fuzz_scale)
    no = ora.ring_restore(fuzz_scale=fuzz_scale)
    assert ne == no == len(jobs) == 15
    _same(eng, ora)
    changed = {a for a in range(n)
               if before[eng.car_offset[a]:eng.car_offset[a + 1]].tobytes() !=
               eng.get_cars()[eng.car_offset[a]:eng.car_offset[a + 1]].tobytes()}
    assert changed <= {a for a, _ in jobs}
    assert eng.ring_stats() == ora.ring_stats()

    # one env step from the rewound state, both sides free-running
    keep = reference_reverse_order(ora, pkg)
    for b in (eng, ora):
        b.step(8)
    a, b = eng.get_cars(), ora.get_cars()
    keep_cars = np.repeat(keep, np.diff(ora.car_offset))
    for comp in "xyz":
        d = np.abs(a["pos"][comp] - b["pos"][comp])[keep_cars]
        assert (d <= 1e-2 + 1e-4 * np.abs(b["pos"][comp][keep_cars])).mean() > 0.99


def test_capture_is_stream_ordered_and_leaves_state(pkg, oracle_lib, meshes_dir):
    """A capture queues device copies only: the live state is untouched, later steps do not
    alter the slot, and restoring with no jitter and lookback 1 rewinds to that capture."""
    n = 64
    ts = np.full(n, 2, np.int32)
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, n, 7, ts)
    for b in (eng, ora):
        b.ring_configure(depth=3, capture_every=1, fuzz_pos=0.0, fuzz_vel=0.0, restore_fraction=0.05)
    _drive(pkg, eng, ora, 2, seed=3)
    snap_cars, snap_balls = eng.get_cars(), eng.get_balls()
    _drive(pkg, eng, ora, 1, seed=4)
    _drive(pkg, eng, ora, 2, seed=5, capture=False)
    # newest capture is the third; lookback 1 reads the second (snap_*)
    cfg = eng._ring_cfg
    st = eng.ring_stats()
    c = {k: getattr(cfg, k) for k, _ in type(cfg)._fields_}
    _, jobs, _ = plan_restore([4] * n, c, st["filled"], st["write_idx"], cfg.seed, lookback=1)
    ne = eng.ring_restore(lookback_slots=1)
    no = ora.ring_restore(lookback_slots=1)
    assert ne == no == len(jobs) == 3
    _same(eng, ora)
    cars, balls = eng.get_cars(), eng.get_balls()
    for a, _ in jobs:
        assert np.allclose(vec(balls[a], "pos"), vec(snap_balls[a], "pos"), rtol=1e-6, atol=1e-3)
        sl = slice(eng.car_offset[a], eng.car_offset[a + 1])
        assert np.array_equal(cars[sl]["boost"], snap_cars[sl]["boost"])
        assert np.allclose(cars[sl]["pos"]["x"], snap_cars[sl]["pos"]["x"], rtol=1e-6, atol=1e-3)


def test_disabled_ring_is_a_no_op(pkg, meshes_dir):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), 16, team_size=1, meshes_path=meshes_dir)
    eng.ring_configure(depth=0)
    before = eng.get_cars()
    eng.ring_capture()
    eng.ring_maybe_capture()
    assert eng.ring_restore() == 0
    assert eng.get_cars().tobytes() == before.tobytes()
    assert eng.ring_stats()["depth"] == 0
