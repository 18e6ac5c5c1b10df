"""Env layer on the device against the oracle, which runs RLGymCPP's own AdvancedObs,
DefaultAction masks, stub rewards, ZeroSumReward and terminal conditions on the reference
RocketSim.

After every env step the oracle's state is read and written into both sides, so both hold
bit-identical Bullet-unit state (the write converts uu to Bullet units the same way on
both), and observations, masks, rewards and terminals are computed from identical inputs:
all four must be bit-identical.  Arenas whose reference visits its cars in another order
than the engine (see reference_reverse_order) are left out.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import random_balls, random_cars, reference_reverse_order, vec

pytestmark = pytest.mark.gpu

def _within(a, b):
    """Bit-identical floats (+0 and -0 told apart)."""
    return a.view(np.uint32) == b.view(np.uint32)


def _scene(rsb, ora, seed):
    """Cars on the ground at random; in a third of the arenas the ball sits in front of a
    car driving at it (touches), in a sixth it flies at a goal (goal terminals)."""
    n = ora.num_arenas
    rng = np.random.default_rng(seed)
    cars = random_cars(rsb, ora.get_cars(), seed)
    balls = random_balls(rsb, n, seed + 1, rest_fraction=0.0)
    balls["pos"]["z"] = rng.uniform(93.15, 1200, n)
    off = ora.car_offset
    for a in range(n):
        kind = a % 6
        if kind < 2:
            c = cars[off[a]]
            fwd = vec(c["rot"], "forward")
            d = rng.uniform(150, 350)
            balls["pos"]["x"][a] = c["pos"]["x"] + fwd[0] * d
            balls["pos"]["y"][a] = c["pos"]["y"] + fwd[1] * d
            balls["pos"]["z"][a] = 93.15
            for comp in "xyz":
                balls["vel"][comp][a] = 0.0
        elif kind == 2:
            sgn = 1.0 if rng.random() < 0.5 else -1.0
            balls["pos"]["x"][a] = rng.uniform(-600, 600)
            balls["pos"]["y"][a] = sgn * 4800.0
            balls["pos"]["z"][a] = 300.0
            balls["vel"]["x"][a], balls["vel"]["y"][a], balls["vel"]["z"][a] = 0.0, sgn * 3000.0, 0.0
    return cars, balls


def _pair(pkg, oracle_lib, meshes_dir, n, seed, team_size=None, team_sizes=None, **rewards):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), n, team_size=team_size, team_sizes=team_sizes, meshes_path=meshes_dir,
                    rewards=rsb.default_rewards(pkg.engine_library(), **rewards))
    ora = rsb.Batch(oracle_lib, n, team_size=team_size, team_sizes=team_sizes, meshes_path=meshes_dir, threads=8,
                    rewards=rsb.default_rewards(oracle_lib, **rewards))
    cars, balls = _scene(rsb, ora, seed)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    lut = rsb.default_action_lut(pkg.engine_library())
    for b in (eng, ora):
        b.set_action_lut(lut)
    return eng, ora


def _sync(eng, ora):
    cars, balls, pads = ora.get_cars(), ora.get_balls(), ora.get_pads()
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
        b.set_pads(pads)


def _run_env_steps(pkg, eng, ora, steps, seed, reset_mode=0):
    keep_arena = reference_reverse_order(ora, pkg)
    keep = np.repeat(keep_arena, np.diff(ora.car_offset))
    rng = np.random.default_rng(seed)
    seen = {"touch": 0, "goal": 0, "trunc": 0, "rows": 0}
    for step in range(steps):
        idx = rng.integers(0, pkg.rsb.RSB_NUM_ACTIONS, eng.num_cars).astype(np.int32)
        for b in (eng, ora):
            b.snapshot()
            b.set_actions(idx)
            b.step(8)
        _sync(eng, ora)
        for b in (eng, ora):
            b.build_obs()
            b.build_rewards_terminals(8)
        oe, oo = eng.copy_obs(), ora.copy_obs()
        me, mo = eng.copy_masks(), ora.copy_masks()
        re_, ro = eng.copy_rewards(), ora.copy_rewards()
        te, to = eng.copy_terminals(), ora.copy_terminals()
        ok = _within(oe, oo).all(axis=1)
        bad = np.nonzero(keep & ~ok)[0]
        assert bad.size == 0, (f"step {step}: obs rows differ for cars {bad[:8]}; first row diff at cols "
                               f"{np.nonzero(~_within(oe[bad[0]], oo[bad[0]]))[0][:10]}")
        badm = np.nonzero(keep & (me != mo).any(axis=1))[0]
        assert badm.size == 0, f"step {step}: masks differ for cars {badm[:8]}"
        badr = np.nonzero(keep & ~_within(re_, ro))[0]
        assert badr.size == 0, f"step {step}: rewards differ for cars {badr[:8]}: {re_[badr[:4]]} vs {ro[badr[:4]]}"
        badt = np.nonzero(keep_arena & (te != to))[0]
        assert badt.size == 0, f"step {step}: terminals differ in arenas {badt[:8]}: {te[badt[:4]]} vs {to[badt[:4]]}"
        seen["goal"] += int((to == 1).sum())
        seen["trunc"] += int((to == 2).sum())
        seen["rows"] += int(keep.sum())
        done = np.nonzero(to)[0].astype(np.int32)
        if done.size:
            for b in (eng, ora):
                b.reset_arenas(done, seed + step, reset_mode)
            # both sides restart from the oracle's reset state
            _sync(eng, ora)
            for b in (eng, ora):
                b.build_obs()
            oe, oo = eng.copy_obs(), ora.copy_obs()
            ok = _within(oe, oo).all(axis=1)
            assert (ok | ~keep).all(), f"step {step}: obs after reset differ"
    return seen


@pytest.mark.parametrize("team_size", [1, 2, 3])
def test_obs_masks_rewards_terminals_match_oracle(pkg, oracle_lib, meshes_dir, team_size):
    n = 192
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, n, seed=300 + team_size, team_size=team_size,
                     no_touch_timeout_s=0.5, episode_max_ticks=160)
    seen = _run_env_steps(pkg, eng, ora, steps=24, seed=41 + team_size)
    # the scene must exercise goal terminals and truncations
    assert seen["goal"] > 0 and seen["trunc"] > 0, seen


def test_zero_sum_and_weights_match_oracle(pkg, oracle_lib, meshes_dir):
    n = 96
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, n, seed=77, team_size=3, w_goal=10.0, w_touch=3.0,
                     w_vel_ball_to_goal=2.0, w_vel_player_to_ball=0.5, goal_concede_scale=-0.8, zero_sum=0b1110,
                     team_spirit=0.3, opponent_scale=0.9, no_touch_timeout_s=1.0)
    _run_env_steps(pkg, eng, ora, steps=12, seed=5)


def test_ragged_batch_rows_and_padding(pkg, oracle_lib, meshes_dir):
    n = 96
    ts = np.array([1, 2, 3] * (n // 3), np.int32)
    eng, ora = _pair(pkg, oracle_lib, meshes_dir, n, seed=9, team_sizes=ts)
    assert eng.obs_stride == ora.obs_stride == 51 + 29 * 6
    _run_env_steps(pkg, eng, ora, steps=8, seed=13)
    obs = eng.copy_obs()
    for a in range(n):
        m = 2 * ts[a]
        rows = obs[eng.car_offset[a]:eng.car_offset[a + 1]]
        assert not rows[:, 51 + 29 * m:].any(), "padding beyond an arena's row length must be zero"


def test_kickoff_reset_obs_match_oracle(pkg, oracle_lib, meshes_dir):
    """After a device kickoff reset the engine's state, written into the oracle, gives the
    same observations (zero previous actions, fresh pads)."""
    n = 64
    for ts in (1, 2, 3):
        eng, ora = _pair(pkg, oracle_lib, meshes_dir, n, seed=3, team_size=ts)
        eng.reset_all(1234, pkg.rsb.RSB_RESET_KICKOFF)
        ora.reset_all(1234, pkg.rsb.RSB_RESET_KICKOFF)
        _sync(ora, eng)
        keep = np.repeat(reference_reverse_order(ora, pkg), np.diff(ora.car_offset))
        for b in (eng, ora):
            b.build_obs()
        oe, oo = eng.copy_obs(), ora.copy_obs()
        assert (_within(oe, oo).all(axis=1) | ~keep).all()
        assert not oe[:, 9:17].any(), "previous actions are zero after a reset"
        assert np.array_equal(eng.copy_masks()[keep], ora.copy_masks()[keep])


def _kickoff_table(pkg, oracle_lib, meshes_dir):
    """(x, y) -> car state fields the reference's Arena::ResetToRandomKickoff produces."""
    rsb = pkg.rsb
    table = {}
    ora = rsb.Batch(oracle_lib, 64, team_size=3, meshes_path=meshes_dir, threads=4)
    for seed in range(4):
        ora.reset_all(seed, rsb.RSB_RESET_KICKOFF)
        for c in ora.get_cars():
            table[(float(c["pos"]["x"]), float(c["pos"]["y"]))] = c
    return table


def test_kickoff_reset_is_the_reference_layout(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    table = _kickoff_table(pkg, oracle_lib, meshes_dir)
    assert len(table) == 10, "5 kickoff spawns per team"
    ref = rsb.Batch(oracle_lib, 1, team_size=1, meshes_path=meshes_dir, threads=1)
    ref.reset_all(0, rsb.RSB_RESET_KICKOFF)
    ref_ball = ref.get_balls()[0]
    for ts in (1, 2, 3):
        eng = rsb.Batch(pkg.engine_library(), 256, team_size=ts, meshes_path=meshes_dir)
        eng.step(5)
        eng.reset_all(99 + ts, rsb.RSB_RESET_KICKOFF)
        cars, balls, pads, info = eng.get_cars(), eng.get_balls(), eng.get_pads(), eng.get_arena_info()
        fields = ["pos", "rot", "vel", "ang_vel", "boost", "is_on_ground", "has_jumped", "ball_hit_valid",
                  "ball_hit_tick", "demo_respawn_timer", "last_controls"]
        for c in cars:
            ref = table[(float(c["pos"]["x"]), float(c["pos"]["y"]))]
            for f in fields:
                assert c[f].tobytes() == ref[f].tobytes(), f
        # each team takes distinct spawns; orange rank i mirrors blue rank i
        for a in range(eng.num_arenas):
            blue = cars[eng.car_offset[a]:eng.car_offset[a] + ts]
            orange = cars[eng.car_offset[a] + ts:eng.car_offset[a + 1]]
            assert len({(float(c["pos"]["x"]), float(c["pos"]["y"])) for c in blue}) == ts
            for b, o in zip(blue, orange):
                assert o["pos"]["x"] == -b["pos"]["x"] and o["pos"]["y"] == -b["pos"]["y"]
        assert all(b.tobytes() == ref_ball.tobytes() for b in balls)
        assert pads["is_active"].all() and not pads["cooldown"].any()
        assert not info["episode_ticks"].any() and not info["status"].any()
        # controls are zeroed by the reset: the cars stay at their spawns
        eng.step(8)
        after = eng.get_cars()
        assert np.abs(vec(after, "pos") - vec(cars, "pos")).max() < 5.0


def test_random_state_reset_distribution(pkg, meshes_dir):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), 4096, team_size=3, meshes_path=meshes_dir)
    eng.reset_all(5, rsb.RSB_RESET_RANDOM_STATE)
    cars, balls = eng.get_cars(), eng.get_balls()
    bp, bv = vec(balls, "pos"), vec(balls, "vel")
    assert (np.abs(bp[:, 0]) <= 3500).all() and (np.abs(bp[:, 1]) <= 4000).all()
    assert (bp[:, 2] >= 92.74).all() and (bp[:, 2] <= 1820).all()
    assert (np.linalg.norm(bv, axis=1) <= 4000.5).all() and np.linalg.norm(bv, axis=1).max() > 3500
    cp, cv = vec(cars, "pos"), vec(cars, "vel")
    ground = np.abs(cp[:, 2] - 17.0) < 1e-3
    assert 0.4 < ground.mean() < 0.6
    assert (np.abs(cv[ground, 2]) == 0).all() and not vec(cars, "ang_vel")[ground].any()
    assert (np.linalg.norm(cv, axis=1) <= 2300.5).all()
    assert (cars["boost"] >= 0).all() and (cars["boost"] <= 100).all()
    rot = np.stack([vec(cars["rot"], f) for f in ("forward", "right", "up")], axis=1)
    assert np.abs(rot @ rot.transpose(0, 2, 1) - np.eye(3)).max() < 1e-5
    # deterministic per seed, different across seeds
    eng.reset_all(5, rsb.RSB_RESET_RANDOM_STATE)
    assert eng.get_cars().tobytes() == cars.tobytes()
    eng.reset_all(6, rsb.RSB_RESET_RANDOM_STATE)
    assert eng.get_cars().tobytes() != cars.tobytes()
    eng.step(16)
    assert not eng.get_arena_info()["status"].any()


def test_high_contact_reset(pkg, meshes_dir):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), 2048, team_size=1, meshes_path=meshes_dir)
    eng.reset_all(11, rsb.RSB_RESET_HIGH_CONTACT)
    cars, balls = eng.get_cars(), eng.get_balls()
    sp = np.linalg.norm(vec(cars, "vel"), axis=1)
    assert (sp >= 1499).all() and (sp <= 2301).all()
    cp = vec(cars, "pos")
    bp = np.repeat(vec(balls, "pos"), 2, axis=0)
    near_ball = np.linalg.norm((cp - bp)[:, :2], axis=1) <= 300.5
    other = cp.reshape(-1, 2, 3)[:, ::-1].reshape(-1, 3)
    near_car = np.linalg.norm((cp - other)[:, :2], axis=1) <= 300.5
    wall = (np.abs(cp[:, 0]) >= 3999) | (cp[:, 2] >= 1949)
    assert (near_ball | near_car | wall).all()
    assert 0.05 < wall.mean() < 0.25
    assert 0.3 < (cp[:, 2] > 17.0).mean() < 0.8
    eng.step(64)
    assert not (eng.get_arena_info()["status"] & rsb.RSB_ARENA_NONFINITE).any()


def test_reset_subset_leaves_other_arenas(pkg, meshes_dir):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), 64, team_size=2, meshes_path=meshes_dir)
    eng.reset_all(1, rsb.RSB_RESET_RANDOM_STATE)
    before = eng.get_cars()
    idx = np.arange(0, 64, 3, dtype=np.int32)
    eng.reset_arenas(idx, 2, rsb.RSB_RESET_KICKOFF)
    after = eng.get_cars()
    changed = np.repeat(np.isin(np.arange(64), idx), 4)
    assert (after[~changed].tobytes() == before[~changed].tobytes())
    assert (np.abs(after["pos"]["z"][changed] - 17.0) < 1e-3).all()
    with pytest.raises(rsb.RsbError):
        eng.reset_arenas(np.array([64], np.int32), 0, 0)
