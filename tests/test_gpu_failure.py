"""Failure detection on the device, driven from the host (no fault, trap or hang is made on the
GPU: the failures are bad inputs the host uploads).

  * a non-finite car state raises RSB_ARENA_NONFINITE in its own arena only, leaves every
    other arena bit-identical to a run without it, and a reset clears the bit;
  * a culler bound that is deliberately wrong (the network answers 1e6 uu everywhere, so every
    body looks clear of the arena) in audit mode: the skipped static tests still run, every contact they find
    is counted as a missed contact, the arenas that saw one carry RSB_ARENA_CULL_MISS and are
    counted as reverted, and the state stays bit-identical to the exact path; a reset clears
    the bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import random_balls, random_cars, random_controls

pytestmark = pytest.mark.gpu


def _pair(pkg, meshes_dir, n, team_size, **kw):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    return [rsb.Batch(lib, n, team_size=team_size, meshes_path=meshes_dir, **kw) for _ in range(2)]


def test_nonfinite_state_is_flagged_and_contained(pkg, meshes_dir):
    rsb = pkg.rsb
    n, bad_arena = 16, 5
    a, b = _pair(pkg, meshes_dir, n, 2)
    cars = random_cars(rsb, a.get_cars(), seed=41)
    balls = random_balls(rsb, n, seed=42)
    ctl = random_controls(rsb, a.num_cars, np.random.default_rng(43))
    for x in (a, b):
        x.set_cars(cars)
        x.set_balls(balls)
        x.set_controls(ctl)
    broken = cars.copy()
    broken["pos"]["x"][a.car_offset[bad_arena] + 1] = np.nan
    b.set_cars(broken)
    for x in (a, b):
        x.step(8)
    ia, ib = a.get_arena_info(), b.get_arena_info()
    assert (ia["status"] == 0).all()
    assert ib["status"][bad_arena] & rsb.RSB_ARENA_NONFINITE
    others = np.arange(n) != bad_arena
    assert (ib["status"][others] == 0).all()
    ca, cb = a.get_cars(), b.get_cars()
    keep = np.repeat(others, np.diff(a.car_offset))
    assert ca[keep].tobytes() == cb[keep].tobytes()
    assert a.get_balls()[others].tobytes() == b.get_balls()[others].tobytes()
    assert b.stats()["status_bits_seen"] & rsb.RSB_ARENA_NONFINITE
    # a reset of the arena clears the bit and the arena steps normally again
    b.reset_arenas(np.array([bad_arena], np.int32), 9, rsb.RSB_RESET_KICKOFF)
    assert b.get_arena_info()["status"][bad_arena] == 0
    b.step(8)
    assert (b.get_arena_info()["status"] == 0).all()
    c = b.get_cars()
    s = slice(b.car_offset[bad_arena], b.car_offset[bad_arena + 1])
    assert np.isfinite(np.stack([c["pos"][k][s] for k in "xyz"])).all()


def test_wrong_culler_bound_is_caught_by_the_audit(pkg, meshes_dir):
    rsb = pkg.rsb
    n = 256
    exact, audit = (rsb.Batch(pkg.engine_library(), n, team_size=1, meshes_path=meshes_dir, cull_mode=m)
                    for m in (rsb.RSB_CULL_EXACT, rsb.RSB_CULL_LEARNED_AUDIT))
    # a network that answers 1e6 km everywhere (zero weights, output bias 1e6): every bound
    # clears every body's reach
    params = np.zeros(rsb.RSB_CULLER_PARAMS, np.float32)
    params[-1] = 1e6
    audit.culler_set(params, 0.0)
    # cars and balls at mid height, far from the floor, ceiling and side-wall planes (whose
    # exact distances the culler keeps), flying into a back wall, which is an arena mesh
    rng = np.random.default_rng(14)
    cars = random_cars(rsb, exact.get_cars(), seed=15)
    side = np.where(np.arange(len(cars)) % 2 == 0, 1.0, -1.0)
    cars["pos"]["x"] = rng.uniform(-2500, 2500, len(cars))
    cars["pos"]["y"] = side * 5000
    cars["pos"]["z"] = rng.uniform(900, 1100, len(cars))
    cars["vel"]["x"], cars["vel"]["y"], cars["vel"]["z"] = 0.0, side * 1800, 0.0
    cars["is_on_ground"] = 0
    balls = random_balls(rsb, n, seed=16)
    balls["pos"]["x"] = rng.uniform(-2500, 2500, n)
    balls["pos"]["y"] = rng.choice([-4900.0, 4900.0], n)
    balls["pos"]["z"] = rng.uniform(900, 1100, n)
    balls["vel"]["x"], balls["vel"]["y"], balls["vel"]["z"] = 0.0, np.sign(balls["pos"]["y"]) * 2500, 0.0
    ctl = np.zeros(exact.num_cars, rsb.CONTROLS_DTYPE)
    for x in (exact, audit):
        x.set_cars(cars)
        x.set_balls(balls)
        x.set_controls(ctl)
        x.step(8)
        x.step(8)
    st = audit.stats()
    info = audit.get_arena_info()
    flagged = (info["status"] & rsb.RSB_ARENA_CULL_MISS) != 0
    assert st["culled_queries"] > 0
    assert st["missed_contacts"] > 0
    assert flagged.sum() > n // 2
    assert st["arenas_reverted"] == int(flagged.sum())
    assert exact.get_cars().tobytes() == audit.get_cars().tobytes()
    assert exact.get_balls().tobytes() == audit.get_balls().tobytes()
    assert exact.get_pads().tobytes() == audit.get_pads().tobytes()
    audit.reset_arenas(np.arange(n, dtype=np.int32), 13, rsb.RSB_RESET_KICKOFF)
    assert (audit.get_arena_info()["status"] == 0).all()
