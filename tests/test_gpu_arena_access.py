"""Per-arena state access on the engine against the oracle: the same one-arena reads and
writes leave both batches bit-identical."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import random_balls, random_cars

pytestmark = pytest.mark.gpu


def test_one_arena_access_matches_oracle(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    n = 90
    ts = np.array([1, 2, 3] * 30, np.int32)
    eng = rsb.Batch(pkg.engine_library(), n, team_sizes=ts, meshes_path=meshes_dir)
    ora = rsb.Batch(oracle_lib, n, team_sizes=ts, meshes_path=meshes_dir, threads=4)
    cars, balls = random_cars(rsb, ora.get_cars(), 11), random_balls(rsb, n, 12)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    rng = np.random.default_rng(5)
    off = ora.car_offset
    for a in rng.choice(n, 20, replace=False):
        a = int(a)
        for c in range(off[a + 1] - off[a]):
            assert eng.get_car(a, c).tobytes() == ora.get_car(a, c).tobytes()
        assert eng.get_ball(a).tobytes() == ora.get_ball(a).tobytes()
        assert eng.get_arena_pads(a).tobytes() == ora.get_arena_pads(a).tobytes()
        info_e, info_o = eng.get_arena_info_at(a), ora.get_arena_info_at(a)
        for f in ("num_cars", "team_size", "goal_scored", "goal_team"):
            assert info_e[f] == info_o[f]
        car = ora.get_car(a, 0)
        car["pos"]["y"] += rng.uniform(-500, 500)
        car["vel"]["x"] = rng.uniform(-1000, 1000)
        ball = ora.get_ball(a)
        ball["pos"]["z"] = rng.uniform(100, 1500)
        pads = ora.get_arena_pads(a)
        pads["is_active"][::3] = 0
        pads["cooldown"][::3] = 7.5
        for b in (eng, ora):
            b.set_car(a, 0, car)
            b.set_ball(a, ball)
            b.set_arena_pads(a, pads)
    for get in ("get_cars", "get_balls", "get_pads"):
        assert getattr(eng, get)().tobytes() == getattr(ora, get)().tobytes(), get
