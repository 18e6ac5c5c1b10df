"""Non-default mutators (RocketSim MutatorConfig) on the engine against the oracle, per tick
with both sides restarted from the oracle's state every tick, at the bounds of the
default-config per-tick test (tests/test_gpu_cars.py).

Stronger boosts, jumps and unlimited flips make violent contacts common, which amplify any
one-ulp difference into a visible one.  The device reproduces the reference's x86 rsqrtss
estimate and its C library's sin / cos / atan2 / asin (phys/refmath.h), so no car-tick may
leave the bounds and no discrete field may differ (the counts are printed).
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import (POS_ABS_UU, VEL_ABS_UU, flag_mismatch, random_balls, random_cars,
                      random_controls, reference_reverse_order, vec)

pytestmark = pytest.mark.gpu

CASES = {
    "low_gravity_heavy_ball": dict(gravity=(0.0, 0.0, -325.0), ball_mass=60.0, ball_max_speed=3000.0, ball_drag=0.1,
                                   ball_world_restitution=0.8, ball_world_friction=0.5, car_mass=250.0),
    "boost_jump_flips": dict(boost_accel_ground=1500.0, boost_accel_air=1500.0, jump_accel=2500.0,
                             jump_immediate_force=500.0, boost_used_per_second=10.0, unlimited_flips=1,
                             unlimited_double_jumps=1, car_world_friction=0.6, car_world_restitution=0.1),
    "demos_bumps_pads": dict(demo_mode=1, enable_team_demos=1, bump_force_scale=2.0, bump_cooldown_time=0.1,
                             respawn_delay=1.0, boost_pad_cooldown_big=2.0, boost_pad_cooldown_small=1.0,
                             car_spawn_boost_amount=100.0, ball_hit_extra_force_scale=1.5),
    "big_ball": dict(ball_radius=100.0),  # RocketSim's broadphase refuses balls much larger (cell size)
}


def _mutators(rsb, lib, fields):
    m = rsb.default_mutators(lib)
    for k, v in fields.items():
        if k == "gravity":
            m.gravity.x, m.gravity.y, m.gravity.z = v
        else:
            setattr(m, k, v)
    return m


@pytest.mark.parametrize("case", sorted(CASES))
def test_per_tick_parity_with_mutators(pkg, oracle_lib, meshes_dir, case):
    rsb = pkg.rsb
    n, team_size = 192, 2
    fields = CASES[case]
    eng = rsb.Batch(pkg.engine_library(), n, team_size=team_size, meshes_path=meshes_dir,
                    mutators=_mutators(rsb, pkg.engine_library(), fields))
    ora = rsb.Batch(oracle_lib, n, team_size=team_size, meshes_path=meshes_dir, threads=8,
                    mutators=_mutators(rsb, oracle_lib, fields))
    seed = 400 + sorted(CASES).index(case)
    cars = random_cars(rsb, ora.get_cars(), seed)
    balls = random_balls(rsb, n, seed + 1, rest_fraction=0.0)
    rmin = fields.get("ball_radius", 91.25) + 2.0
    balls["pos"]["z"] = np.random.default_rng(seed).uniform(rmin, 1300, n)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    keep_arena = reference_reverse_order(ora, pkg)
    keep = np.repeat(keep_arena, np.diff(ora.car_offset))
    rng = np.random.default_rng(seed + 2)
    off_bounds = discrete = total = 0
    for tick in range(64):
        if tick % 8 == 0:
            ctl = random_controls(rsb, eng.num_cars, rng)
            eng.set_controls(ctl)
            ora.set_controls(ctl)
        eng.step(1)
        ora.step(1)
        a, b = eng.get_cars()[keep], ora.get_cars()[keep]
        total += len(a)
        discrete += int(flag_mismatch(a, b).sum())
        bad = np.zeros(len(a), bool)
        for f, tol in (("pos", POS_ABS_UU), ("vel", VEL_ABS_UU), ("ang_vel", 1e-3)):
            x, y = vec(a, f), vec(b, f)
            bad |= (np.abs(x - y) > tol + 1e-4 * np.abs(y)).any(axis=1)
        bad |= np.abs(a["boost"] - b["boost"]) > 1e-3
        off_bounds += int(bad.sum())
        ba, bb = eng.get_balls()[keep_arena], ora.get_balls()[keep_arena]
        # the ball carries the same amplified differences after such an impact
        ball_bad = (np.abs(vec(ba, "pos") - vec(bb, "pos")) > POS_ABS_UU + 1e-4 * np.abs(vec(bb, "pos"))).any(axis=1)
        off_bounds += int(ball_bad.sum())
        pa, pb = eng.get_pads(), ora.get_pads()
        np.testing.assert_array_equal(pa["is_active"], pb["is_active"], err_msg=f"{case}, tick {tick}")
        cars, balls = ora.get_cars(), ora.get_balls()
        for x in (eng, ora):
            x.set_cars(cars)
            x.set_balls(balls)
    print(f"MUTATORS {case}: {discrete} discrete, {off_bounds} off-bounds of {total} car-ticks")
    assert discrete == 0, f"{case}: discrete state differs on {discrete} of {total} car-ticks"
    assert off_bounds == 0, f"{case}: {off_bounds} of {total} car-ticks outside the per-tick bounds"
