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
    assert len(res) == 9 and all(r["ms"] > 0 for r in res)
    assert (a.get_cars().tobytes(), a.get_balls().tobytes(), a.get_arena_info().tobytes()) == before
    ctl = np.zeros(a.num_cars, rsb.CONTROLS_DTYPE)
    ctl["throttle"] = 1
    ctl["boost"] = 1
    for x in (a, b):
        x.set_controls(ctl)
        x.step(16)
    assert a.get_cars().tobytes() == b.get_cars().tobytes()
    assert a.get_balls().tobytes() == b.get_balls().tobytes()
