"""rsb_autotune: every launch configuration of the step kernel is timed on a copy of the
state (the handle's own state does not move), and the chosen configuration computes the
same arenas bit for bit as the default one."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import random_balls, random_cars

pytestmark = pytest.mark.gpu


def test_autotune_keeps_state_and_results(pkg, meshes_dir):
    rsb = pkg.rsb
    n = 512
    a = rsb.Batch(pkg.engine_library(), n, team_size=3, meshes_path=meshes_dir)
    b = rsb.Batch(pkg.engine_library(), n, team_size=3, meshes_path=meshes_dir)
    cars = random_cars(rsb, a.get_cars(), 17)
    balls = random_balls(rsb, n, 18)
    for x in (a, b):
        x.set_cars(cars)
        x.set_balls(balls)
    before = a.get_cars().tobytes(), a.get_balls().tobytes(), a.get_arena_info().tobytes()
    res = a.autotune(8)
    # 6 variants x 3 block sizes at full residency, plus 2 x 5 residency caps
    assert len(res) == 28 and all(r["ms"] > 0 for r in res)
    assert sum(r["persistent"] for r in res) == 19
    assert sum(r["warps_per_sm"] > 0 for r in res) == 10
    assert (a.get_cars().tobytes(), a.get_balls().tobytes(), a.get_arena_info().tobytes()) == before
    ctl = np.zeros(a.num_cars, rsb.CONTROLS_DTYPE)
    ctl["throttle"] = 1
    ctl["boost"] = 1
    for x in (a, b):
        x.set_controls(ctl)
        x.step(16)
    assert a.get_cars().tobytes() == b.get_cars().tobytes()
    assert a.get_balls().tobytes() == b.get_balls().tobytes()


@pytest.mark.parametrize("min_blocks,block,warps", [(1, 64, 0), (3, 32, 0), (4, 128, 0), (1, 32, 1), (1, 64, 3)])
def test_persistent_launch_is_bit_identical(pkg, meshes_dir, min_blocks, block, warps):
    """Warps claiming 32 arenas at a time compute every arena exactly as one-thread-per-arena
    blocks do (ragged batch, with an arena count that is not a multiple of 32), at full and at
    capped residency."""
    rsb = pkg.rsb
    ts = np.array([1, 2, 3] * 341 + [2], np.int32)
    n = len(ts)
    a = rsb.Batch(pkg.engine_library(), n, team_sizes=ts, meshes_path=meshes_dir)
    b = rsb.Batch(pkg.engine_library(), n, team_sizes=ts, meshes_path=meshes_dir)
    a.set_step_config(min_blocks, block, persistent=True, warps_per_sm=warps)
    b.set_step_config(1, 64, persistent=False)
    cars = random_cars(rsb, a.get_cars(), 21)
    balls = random_balls(rsb, n, 22)
    ctl = np.zeros(a.num_cars, rsb.CONTROLS_DTYPE)
    ctl["throttle"] = 1
    ctl["boost"] = 1
    ctl["steer"] = np.random.default_rng(3).uniform(-1, 1, a.num_cars)
    for x in (a, b):
        x.set_cars(cars)
        x.set_balls(balls)
        x.set_controls(ctl)
        for _ in range(3):
            x.step(8)
    assert a.get_cars().tobytes() == b.get_cars().tobytes()
    assert a.get_balls().tobytes() == b.get_balls().tobytes()
    assert a.get_pads().tobytes() == b.get_pads().tobytes()
    with pytest.raises(rsb.RsbError):
        a.set_step_config(2, 64)
    with pytest.raises(rsb.RsbError):
        a.set_step_config(1, 64, persistent=False, warps_per_sm=2)
