"""The CUDA engine against the committed golden rollouts of the reference CPU RocketSim
(tests/golden/soccar_trajectories.npz): the same states and actions, 120 free-running ticks.
Discrete car flags and car and ball positions must equal the recorded ones at every tick;
arenas whose recorded car order is not reverse creation order are left out (the reference's
car set is hashed by heap address)."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_engine_follows_golden(pkg, meshes_dir):
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg

    rsb = pkg.rsb
    g = dict(np.load(os.path.join(HERE, "golden", "soccar_trajectories.npz")))
    ts = g["team_sizes"]
    b = rsb.Batch(pkg.engine_library(), len(ts), team_sizes=ts, meshes_path=meshes_dir)
    b.set_action_lut(np.frombuffer(g["lut"].tobytes(), rsb.CONTROLS_DTYPE))
    cars = np.frombuffer(g["init_cars"].tobytes(), rsb.CAR_DTYPE).copy()
    balls = np.frombuffer(g["init_balls"].tobytes(), rsb.BALL_DTYPE).copy()
    car_kin, car_flags, car_boost, ball_kin = mg.run(b, cars, balls, g["actions"], rsb)
    order = g["car_order"]
    reverse = np.array([np.array_equal(order[a, :2 * t], np.arange(2 * t)[::-1]) for a, t in enumerate(ts)])
    keep = np.repeat(reverse, 2 * ts)
    flag_ok = (car_flags[:, keep] == g["car_flags"][:, keep]).mean()
    drift_all = np.linalg.norm(car_kin[:, keep, 0] - g["car_kin"][:, keep, 0], axis=-1)
    print(f"GOLDEN flags equal {flag_ok:.6f}; car drift max {drift_all.max():.4g} uu, cars with any drift "
          f"{int((drift_all.max(axis=0) > 0).sum())} of {int(keep.sum())}")
    assert flag_ok == 1.0, flag_ok
    assert drift_all.max() == 0, float(drift_all.max())
    bdrift = np.linalg.norm(ball_kin[:, reverse, 0] - g["ball_kin"][:, reverse, 0], axis=-1)
    assert bdrift.max() == 0, float(bdrift.max())
