"""Per-arena state access (rsb_get/set_*_at) on the oracle: each call reads or writes one car,
ball, pad set or arena info, equal to the whole-batch calls, and leaves the other arenas alone."""
from __future__ import annotations

import numpy as np

from gpu_util import random_balls, random_cars


def test_one_arena_access_matches_batch_access(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    n = 12
    b = rsb.Batch(oracle_lib, n, team_sizes=np.array([1, 2, 3] * 4, np.int32), meshes_path=meshes_dir, threads=2)
    b.set_cars(random_cars(rsb, b.get_cars(), 3))
    b.set_balls(random_balls(rsb, n, 4))
    b.step(16)
    cars, balls, pads, info = b.get_cars(), b.get_balls(), b.get_pads(), b.get_arena_info()
    off = b.car_offset
    for a in range(n):
        for c in range(off[a + 1] - off[a]):
            assert b.get_car(a, c).tobytes() == cars[off[a] + c].tobytes()
        assert b.get_ball(a).tobytes() == balls[a].tobytes()
        assert b.get_arena_pads(a).tobytes() == pads[a * 34:(a + 1) * 34].tobytes()
        assert b.get_arena_info_at(a).tobytes() == info[a].tobytes()
    # writes touch one arena only
    c = cars[off[5] + 1].copy()
    c["pos"]["x"] += 100.0
    c["boost"] = 12.5
    b.set_car(5, 1, c)
    bl = balls[7].copy()
    bl["vel"]["z"] = 321.0
    b.set_ball(7, bl)
    pd = pads[9 * 34:10 * 34].copy()
    pd["is_active"] = 0
    pd["cooldown"] = 4.0
    b.set_arena_pads(9, pd)
    cars2, balls2, pads2 = b.get_cars(), b.get_balls(), b.get_pads()
    changed_cars = np.nonzero([cars2[i].tobytes() != cars[i].tobytes() for i in range(len(cars))])[0]
    assert changed_cars.tolist() == [off[5] + 1]
    assert abs(cars2[off[5] + 1]["pos"]["x"] - c["pos"]["x"]) < 1e-3 and cars2[off[5] + 1]["boost"] == 12.5
    assert [a for a in range(n) if balls2[a].tobytes() != balls[a].tobytes()] == [7]
    assert abs(balls2[7]["vel"]["z"] - 321.0) < 1e-3
    assert [a for a in range(n) if pads2[a * 34:(a + 1) * 34].tobytes() != pads[a * 34:(a + 1) * 34].tobytes()] == [9]
