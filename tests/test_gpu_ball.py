"""Ball-only arenas: the CUDA engine against the oracle, tick by tick."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import POS_ABS_UU, VEL_ABS_UU, max_excess, random_balls, vec

pytestmark = pytest.mark.gpu


def make_pair(pkg, oracle_lib, meshes_dir, n):
    eng = pkg.rsb.Batch(pkg.engine_library(), n, team_size=0, meshes_path=meshes_dir)
    ora = pkg.rsb.Batch(oracle_lib, n, team_size=0, meshes_path=meshes_dir, threads=4)
    return eng, ora


def test_ball_trajectories_match_oracle_120_ticks(pkg, oracle_lib, meshes_dir):
    n = 512
    eng, ora = make_pair(pkg, oracle_lib, meshes_dir, n)
    balls = random_balls(pkg.rsb, n, seed=11)
    eng.set_balls(balls)
    ora.set_balls(balls)
    for tick in range(120):
        eng.step(1)
        ora.step(1)
        a, b = eng.get_balls(), ora.get_balls()
        assert max_excess(vec(a, "pos"), vec(b, "pos"), POS_ABS_UU) <= 0, f"tick {tick} position"
        assert max_excess(vec(a, "vel"), vec(b, "vel"), VEL_ABS_UU) <= 0, f"tick {tick} velocity"
        assert max_excess(vec(a, "ang_vel"), vec(b, "ang_vel"), 1e-4) <= 0, f"tick {tick} angular velocity"
        # and, free-running, byte for byte
        assert a.tobytes() == b.tobytes(), f"tick {tick}: ball states differ"


def test_multi_tick_launch_is_bit_identical(pkg, meshes_dir):
    n = 256
    a = pkg.rsb.Batch(pkg.engine_library(), n, team_size=0, meshes_path=meshes_dir)
    b = pkg.rsb.Batch(pkg.engine_library(), n, team_size=0, meshes_path=meshes_dir)
    balls = random_balls(pkg.rsb, n, seed=5)
    a.set_balls(balls)
    b.set_balls(balls)
    a.step(64)
    for _ in range(8):
        b.step(8)
    sa, sb = a.get_balls(), b.get_balls()
    assert sa.tobytes() == sb.tobytes()


def test_resting_ball_sleeps_like_reference(pkg, oracle_lib, meshes_dir):
    eng, ora = make_pair(pkg, oracle_lib, meshes_dir, 4)
    # the reference puts a ball with exactly zero velocity to sleep: it hangs in the air
    b = random_balls(pkg.rsb, 4, seed=3)
    for f in ("vel", "ang_vel"):
        for c in "xyz":
            b[f][c] = 0.0
    eng.set_balls(b)
    ora.set_balls(b)
    eng.step(30)
    ora.step(30)
    np.testing.assert_array_equal(vec(eng.get_balls(), "pos"), vec(ora.get_balls(), "pos"))


def test_goal_flag_matches_oracle(pkg, oracle_lib, meshes_dir):
    eng, ora = make_pair(pkg, oracle_lib, meshes_dir, 64)
    rng = np.random.default_rng(2)
    b = random_balls(pkg.rsb, 64, seed=9)
    b["pos"]["x"] = rng.uniform(-800, 800, 64)
    b["pos"]["y"] = rng.choice([-1, 1], 64) * rng.uniform(4800, 5300, 64)
    b["pos"]["z"] = rng.uniform(150, 600, 64)
    b["vel"]["y"] = np.sign(b["pos"]["y"]) * rng.uniform(0, 2000, 64)
    eng.set_balls(b)
    ora.set_balls(b)
    for _ in range(40):
        eng.step(1)
        ora.step(1)
        ia, ib = eng.get_arena_info(), ora.get_arena_info()
        np.testing.assert_array_equal(ia["goal_scored"], ib["goal_scored"])
        np.testing.assert_array_equal(ia["goal_team"], ib["goal_team"])


def test_floor_bounce_invariants_and_oracle(pkg, oracle_lib, meshes_dir):
    """The reference's floor-bounce invariants (bounce, no tunnelling, no energy gain) on the
    engine, and the same end state as the oracle."""
    from test_oracle_pins import bounce_invariants

    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), 1, team_size=0, meshes_path=meshes_dir)
    ora = rsb.Batch(oracle_lib, 1, team_size=0, meshes_path=meshes_dir, threads=1)
    be = bounce_invariants(eng)
    bo = bounce_invariants(ora)
    assert be[0] and be[1] >= 0.5 * 91.25 and be[2] <= be[3] * 1.001, be
    assert be[1] == bo[1] and be[2] == bo[2], (be, bo)
    assert eng.get_balls().tobytes() == ora.get_balls().tobytes()
