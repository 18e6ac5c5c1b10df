"""The observation cases of the reference's CPU parity report
(RocketSimCuda/tests/reports/cpu_parity_report.txt: obs_kickoff_1v1, obs_midair_2v2,
obs_post_bounce_inv, obs_demo, obs_near_goal), engine against RLGymCPP's AdvancedObs and
DefaultAction masks in the oracle, bit for bit on identical state."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import random_balls, random_cars, reference_reverse_order

pytestmark = pytest.mark.gpu


def _pair(pkg, oracle_lib, meshes_dir, n, team_size):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), n, team_size=team_size, meshes_path=meshes_dir,
                    rewards=rsb.default_rewards(pkg.engine_library()))
    ora = rsb.Batch(oracle_lib, n, team_size=team_size, meshes_path=meshes_dir, threads=4,
                    rewards=rsb.default_rewards(oracle_lib))
    lut = rsb.default_action_lut(pkg.engine_library())
    for b in (eng, ora):
        b.set_action_lut(lut)
    return eng, ora


def _compare(pkg, eng, ora, steps=1, actions_seed=None):
    """Both sides get the oracle's state, run `steps` env steps of 8 ticks (resynchronised after
    each), then build observations and masks from identical state."""
    keep = np.repeat(reference_reverse_order(ora, pkg), np.diff(ora.car_offset))
    rng = np.random.default_rng(actions_seed or 0)
    cars, balls, pads = ora.get_cars(), ora.get_balls(), ora.get_pads()
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
        b.set_pads(pads)
    for _ in range(steps):
        idx = rng.integers(0, pkg.rsb.RSB_NUM_ACTIONS, eng.num_cars).astype(np.int32)
        for b in (eng, ora):
            b.set_actions(idx)
            b.step(8)
        cars, balls, pads = ora.get_cars(), ora.get_balls(), ora.get_pads()
        for b in (eng, ora):
            b.set_cars(cars)
            b.set_balls(balls)
            b.set_pads(pads)
    for b in (eng, ora):
        b.build_obs()
    oe, oo = eng.copy_obs(), ora.copy_obs()
    same = (oe.view(np.uint32) == oo.view(np.uint32)).all(axis=1)
    assert (same | ~keep).all(), f"observation rows differ for cars {np.nonzero(~same & keep)[0][:8]}"
    assert (eng.copy_masks() == ora.copy_masks()).all(axis=1)[keep].all()
    return oe


def test_obs_kickoff_1v1(pkg, oracle_lib, meshes_dir):
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, 64, 1)
    ora.reset_all(11, pkg.rsb.RSB_RESET_KICKOFF)
    obs = _compare(pkg, eng, ora, steps=0)
    assert obs.shape[1] == 109


def test_obs_midair_2v2(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, 64, 2)
    cars = random_cars(rsb, ora.get_cars(), 5)
    rng = np.random.default_rng(6)
    cars["pos"]["z"] = rng.uniform(200, 1500, len(cars))
    cars["vel"]["z"] = rng.uniform(-500, 500, len(cars))
    cars["is_on_ground"] = 0
    cars["has_jumped"] = 1
    balls = random_balls(rsb, 64, 7, rest_fraction=0.0)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    obs = _compare(pkg, eng, ora, steps=2, actions_seed=8)
    assert obs.shape[1] == 167


def test_obs_post_bounce_orange_side(pkg, oracle_lib, meshes_dir):
    """Balls bouncing off the floor near the orange end: the orange rows see the field
    inverted."""
    rsb = pkg.rsb
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, 64, 1)
    cars = random_cars(rsb, ora.get_cars(), 9)
    balls = random_balls(rsb, 64, 10, rest_fraction=0.0)
    rng = np.random.default_rng(11)
    balls["pos"]["y"] = rng.uniform(2000, 4500, 64)
    balls["pos"]["z"] = rng.uniform(100, 200, 64)
    balls["vel"]["z"] = -rng.uniform(800, 1500, 64)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    _compare(pkg, eng, ora, steps=2, actions_seed=12)


def test_obs_demoed_cars(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, 64, 2)
    cars = random_cars(rsb, ora.get_cars(), 13)
    cars["is_demoed"][::3] = 1
    cars["demo_respawn_timer"][::3] = 2.0
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(random_balls(rsb, 64, 14))
    _compare(pkg, eng, ora, steps=1, actions_seed=15)


def test_obs_near_goal(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, 64, 1)
    cars = random_cars(rsb, ora.get_cars(), 16)
    balls = random_balls(rsb, 64, 17, rest_fraction=0.0)
    rng = np.random.default_rng(18)
    side = np.where(np.arange(64) % 2 == 0, 1.0, -1.0)
    balls["pos"]["x"] = rng.uniform(-800, 800, 64)
    balls["pos"]["y"] = side * rng.uniform(4600, 5050, 64)
    balls["pos"]["z"] = rng.uniform(93.15, 500, 64)
    balls["vel"]["y"] = side * rng.uniform(0, 800, 64)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    _compare(pkg, eng, ora, steps=0)
