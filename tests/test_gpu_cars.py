"""Arenas with cars: the CUDA engine against the oracle.

Two comparisons:
  * per tick: both sides start every tick from the same state (the oracle's, written
    into both), and after the tick every byte of every car, ball and pad state is equal;
  * trajectories: both sides run 480 ticks free, and every byte stays equal after every tick
    (parity_util.run_lockstep).  The device reproduces the reference CPU's rsqrtss estimate
    and its C library's sin / cos / atan2 / asin (phys/refmath.h), so nothing is left to
    drift.
Arenas where the reference visits its cars in an order other than the engine's (its car
set is hashed by heap address; see reference_reverse_order) are left out, and so is an arena
after a demolished car respawns (the reference draws the spot from a process-global random
engine).
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import (POS_ABS_UU, VEL_ABS_UU, flag_mismatch, max_excess, random_balls, random_cars,
                      random_controls, reference_reverse_order, rot_matrix, vec)
from parity_util import rows, run_lockstep

pytestmark = pytest.mark.gpu

def make_pair(pkg, oracle_lib, meshes_dir, n, team_size, seed):
    eng = pkg.rsb.Batch(pkg.engine_library(), n, team_size=team_size, meshes_path=meshes_dir)
    ora = pkg.rsb.Batch(oracle_lib, n, team_size=team_size, meshes_path=meshes_dir, threads=8)
    cars = random_cars(pkg.rsb, ora.get_cars(), seed)
    balls = random_balls(pkg.rsb, n, seed + 1, rest_fraction=0.0)
    balls["pos"]["z"] = np.random.default_rng(seed).uniform(93.15, 1300, n)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    return eng, ora


def car_ok_mask(ora, pkg):
    keep_arena = reference_reverse_order(ora, pkg)
    return np.repeat(keep_arena, np.diff(ora.car_offset)), keep_arena


@pytest.mark.parametrize("team_size", [1, 2, 3])
def test_per_tick_parity(pkg, oracle_lib, meshes_dir, team_size):
    n = 256
    eng, ora = make_pair(pkg, oracle_lib, meshes_dir, n, team_size, seed=100 + team_size)
    keep, keep_arena = car_ok_mask(ora, pkg)
    rng = np.random.default_rng(7 + team_size)
    ctl = None
    for tick in range(120):
        if tick % 8 == 0:
            ctl = random_controls(pkg.rsb, eng.num_cars, rng)
            eng.set_controls(ctl)
            ora.set_controls(ctl)
        eng.step(1)
        ora.step(1)
        a, b = eng.get_cars(), ora.get_cars()
        a, b = a[keep], b[keep]
        where = f"team size {team_size}, tick {tick}"
        assert (rows(a, len(a)) == rows(b, len(b))).all(), f"{where}: car states differ"
        ba, bb = eng.get_balls()[keep_arena], ora.get_balls()[keep_arena]
        assert (rows(ba, len(ba)) == rows(bb, len(bb))).all(), f"{where}: ball states differ"
        assert not flag_mismatch(a, b).any(), f"{where}: discrete car state differs"
        np.testing.assert_allclose(a["boost"], b["boost"], atol=1e-3, err_msg=where)
        assert max_excess(vec(a, "pos"), vec(b, "pos"), POS_ABS_UU) <= 0, f"{where}: position"
        assert max_excess(vec(a, "vel"), vec(b, "vel"), VEL_ABS_UU) <= 0, f"{where}: velocity"
        assert max_excess(vec(a, "ang_vel"), vec(b, "ang_vel"), 1e-3) <= 0, f"{where}: angular velocity"
        assert max_excess(rot_matrix(a), rot_matrix(b), 1e-4) <= 0, f"{where}: rotation"
        ba, bb = eng.get_balls()[keep_arena], ora.get_balls()[keep_arena]
        assert max_excess(vec(ba, "pos"), vec(bb, "pos"), POS_ABS_UU) <= 0, f"{where}: ball position"
        assert max_excess(vec(ba, "vel"), vec(bb, "vel"), VEL_ABS_UU) <= 0, f"{where}: ball velocity"
        pa, pb = eng.get_pads(), ora.get_pads()
        np.testing.assert_array_equal(pa["is_active"], pb["is_active"], err_msg=where)
        np.testing.assert_array_equal(pa["prev_locked_car_id"], pb["prev_locked_car_id"], err_msg=where)
        # next tick starts from the oracle's state on both sides
        cars, balls = ora.get_cars(), ora.get_balls()
        for x in (eng, ora):
            x.set_cars(cars)
            x.set_balls(balls)


@pytest.mark.parametrize("team_size", [1, 2, 3])
def test_free_running_is_bit_exact(pkg, oracle_lib, meshes_dir, team_size):
    compared, differed, respawned, first = run_lockstep(pkg.rsb, pkg, pkg.engine_library(), oracle_lib, meshes_dir,
                                                        team_size, 256, seed=200 + team_size, ticks=480)
    print(f"team size {team_size}: {compared} arenas, {respawned} left out after a respawn, {differed} differed")
    assert compared >= 180
    assert differed == 0, f"{differed} arenas differ; first: arena {first[0]} at tick {first[1]}"


def test_free_running_ragged_batch_is_bit_exact(pkg, oracle_lib, meshes_dir):
    sizes = np.array([1, 2, 3] * 64, np.int32)
    compared, differed, respawned, first = run_lockstep(pkg.rsb, pkg, pkg.engine_library(), oracle_lib, meshes_dir,
                                                        None, len(sizes), seed=78, ticks=240, team_sizes=sizes)
    assert compared >= 150
    assert differed == 0, f"{differed} arenas differ; first: arena {first[0]} at tick {first[1]}"


def test_multi_tick_launch_is_bit_identical_with_cars(pkg, meshes_dir):
    n = 128
    a = pkg.rsb.Batch(pkg.engine_library(), n, team_size=3, meshes_path=meshes_dir)
    b = pkg.rsb.Batch(pkg.engine_library(), n, team_size=3, meshes_path=meshes_dir)
    cars = random_cars(pkg.rsb, a.get_cars(), seed=5)
    balls = random_balls(pkg.rsb, n, seed=6)
    ctl = random_controls(pkg.rsb, a.num_cars, np.random.default_rng(1))
    for x in (a, b):
        x.set_cars(cars)
        x.set_balls(balls)
        x.set_controls(ctl)
    a.step(64)
    for _ in range(8):
        b.step(8)
    assert a.get_cars().tobytes() == b.get_cars().tobytes()
    assert a.get_balls().tobytes() == b.get_balls().tobytes()
    assert a.get_pads().tobytes() == b.get_pads().tobytes()


def test_mixed_team_sizes_in_one_batch(pkg, oracle_lib, meshes_dir):
    """Ragged batch (1v1, 2v2, 3v3 interleaved) against per-size oracle runs."""
    sizes = np.array([1, 2, 3] * 32, np.int32)
    eng = pkg.rsb.Batch(pkg.engine_library(), len(sizes), team_size=None, team_sizes=sizes, meshes_path=meshes_dir)
    ora = pkg.rsb.Batch(oracle_lib, len(sizes), team_size=None, team_sizes=sizes, meshes_path=meshes_dir, threads=8)
    cars = random_cars(pkg.rsb, ora.get_cars(), seed=31)
    balls = random_balls(pkg.rsb, len(sizes), seed=32)
    keep, keep_arena = car_ok_mask(ora, pkg)
    rng = np.random.default_rng(3)
    for x in (eng, ora):
        x.set_cars(cars)
        x.set_balls(balls)
    for tick in range(24):
        if tick % 8 == 0:
            ctl = random_controls(pkg.rsb, eng.num_cars, rng)
            eng.set_controls(ctl)
            ora.set_controls(ctl)
        eng.step(1)
        ora.step(1)
        a, b = eng.get_cars()[keep], ora.get_cars()[keep]
        assert not flag_mismatch(a, b).any(), f"tick {tick}: discrete car state differs"
        assert max_excess(vec(a, "pos"), vec(b, "pos"), POS_ABS_UU) <= 0, f"tick {tick}: position"
        assert max_excess(vec(a, "vel"), vec(b, "vel"), VEL_ABS_UU) <= 0, f"tick {tick}: velocity"
        cars, balls = ora.get_cars(), ora.get_balls()
        for x in (eng, ora):
            x.set_cars(cars)
            x.set_balls(balls)
