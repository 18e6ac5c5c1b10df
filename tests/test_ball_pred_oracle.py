"""Ball prediction in the oracle: BallPredTracker's reused ball-only arena
(BallPredTracker.cpp:80-88) gives the same balls as a fresh ball-only batch that takes the
arenas' balls and steps to each slice, and the arenas themselves are not advanced."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def pred_pair(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    ora = rsb.Batch(oracle_lib, 16, team_size=2, meshes_path=meshes_dir, threads=4)
    ora.reset_all(0x5EED0042, rsb.RSB_RESET_RANDOM_STATE)
    return rsb, ora


def _ball_only_steps(rsb, oracle_lib, meshes_dir, balls, slices):
    solo = rsb.Batch(oracle_lib, len(balls), team_size=0, meshes_path=meshes_dir, threads=4)
    solo.set_balls(balls)
    out, t = [], 0
    for s in slices:
        solo.step(s - t)
        t = s
        out.append(solo.get_balls())
    return np.stack(out, axis=1)


def test_prediction_is_a_ball_only_rollout(pred_pair, oracle_lib, meshes_dir):
    rsb, ora = pred_pair
    slices = [1, 8, 120, 360]
    before_balls, before_cars = ora.get_balls(), ora.get_cars()
    for _ in range(2):  # the second call reuses the ball-only arenas
        pred = ora.predict_ball(slices)
        want = _ball_only_steps(rsb, oracle_lib, meshes_dir, before_balls, slices)
        assert pred.shape == (16, 4)
        assert pred.tobytes() == want.tobytes()
        assert ora.get_balls().tobytes() == before_balls.tobytes()
        assert ora.get_cars().tobytes() == before_cars.tobytes()
    moved = np.abs(pred["pos"]["z"][:, 3] - before_balls["pos"]["z"]) + np.abs(pred["pos"]["x"][:, 3] - before_balls["pos"]["x"])
    assert (moved > 1.0).any()


def test_prediction_after_stepping_follows_the_new_ball(pred_pair, oracle_lib, meshes_dir):
    rsb, ora = pred_pair
    ora.set_action_lut(rsb.default_action_lut(oracle_lib))
    ora.set_actions(np.random.default_rng(1).integers(0, rsb.RSB_NUM_ACTIONS, ora.num_cars).astype(np.int32))
    ora.step(8)
    pred = ora.predict_ball([120, 240, 360])
    want = _ball_only_steps(rsb, oracle_lib, meshes_dir, ora.get_balls(), [120, 240, 360])
    assert pred.tobytes() == want.tobytes()


@pytest.mark.parametrize("slices", [[], [0], [5, 5], [10, 3], [1, 4097], list(range(1, 10))])
def test_bad_slices_are_refused(pred_pair, slices):
    rsb, ora = pred_pair
    with pytest.raises(Exception):
        ora.predict_ball(slices)
