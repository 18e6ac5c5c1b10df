"""Contact scenarios with the default mutators, engine against the oracle, per tick with both
sides restarted from the oracle's state every tick (bounds of tests/test_gpu_cars.py):

  * head-on pairs at supersonic speed (demolitions) and at 600-1,400 uu/s (bumps),
  * cars driving at a side wall, a back wall and a corner at 1,000-2,300 uu/s,
  * cars driving at a resting or incoming ball at 500-2,300 uu/s (car-ball hits),
  * airborne cars landing on the ramps.

The scenarios make each contact kind common, so they must happen on both sides on the same
tick: the demo, bump, ball-touch and wheel-contact fields are compared exactly, and no
car-tick may leave the float bounds (the device's arithmetic is the reference's, see
phys/refmath.h; the counts are printed).
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import POS_ABS_UU, VEL_ABS_UU, flag_mismatch, random_balls, reference_reverse_order, vec

pytestmark = pytest.mark.gpu


def _place(c, i, pos, yaw, speed, z=17.0, vz=0.0, pitch=0.0):
    cy, sy = np.cos(yaw), np.sin(yaw)
    cp, sp = np.cos(pitch), np.sin(pitch)
    fwd = (cy * cp, sy * cp, sp)
    right = (-sy, cy, 0.0)
    up = (-cy * sp, -sy * sp, cp)
    for f, v in (("forward", fwd), ("right", right), ("up", up)):
        for k, comp in enumerate("xyz"):
            c["rot"][f][comp][i] = v[k]
    for comp, v in zip("xyz", (pos[0], pos[1], z)):
        c["pos"][comp][i] = v
    for comp, v in zip("xyz", (cy * speed, sy * speed, vz)):
        c["vel"][comp][i] = v
        c["ang_vel"][comp][i] = 0.0
    c["is_on_ground"][i] = 1 if z < 20 else 0
    c["boost"][i] = 50.0
    c["is_supersonic"][i] = 1 if speed >= 2200 else 0
    c["supersonic_time"][i] = 0.0


def _scenes(rsb, cars, balls, off, n, rng):
    """Arena a gets scene a % 6 (2v2: cars 0, 1 blue, 2, 3 orange)."""
    for a in range(n):
        kind = a % 6
        cx, cy = rng.uniform(-2000, 2000), rng.uniform(-3000, 3000)
        o = off[a]
        # keep the spare cars out of the way
        _place(cars, o + 1, (-3000 + 50 * (a % 7), -4000), 0.0, 0.0)
        _place(cars, o + 3, (3000 - 50 * (a % 7), 4000), np.pi, 0.0)
        for comp, v in zip("xyz", (0.0, 4500.0, 93.15)):
            balls["pos"][comp][a] = v
            balls["vel"][comp][a] = 0.0
            balls["ang_vel"][comp][a] = 0.0
        if kind == 0:  # head-on, supersonic: demolitions
            d = rng.uniform(150, 400)
            _place(cars, o + 0, (cx - d, cy), 0.0, 2300.0)
            _place(cars, o + 2, (cx + d, cy), np.pi, rng.uniform(0, 2300))
        elif kind == 1:  # head-on, slower: bumps
            d = rng.uniform(150, 400)
            _place(cars, o + 0, (cx - d, cy), 0.0, rng.uniform(600, 1400))
            _place(cars, o + 2, (cx + d + rng.uniform(-30, 30), cy + rng.uniform(-40, 40)), np.pi + rng.uniform(-0.3, 0.3),
                   rng.uniform(600, 1400))
        elif kind == 2:  # side wall, back wall or corner
            which = a % 3
            if which == 0:
                _place(cars, o + 0, (3800, cy), 0.0, rng.uniform(1000, 2300))
            elif which == 1:
                _place(cars, o + 0, (cx, 4800), np.pi / 2, rng.uniform(1000, 2300))
            else:
                _place(cars, o + 0, (3500, 4500), np.pi / 4, rng.uniform(1000, 2300))
            _place(cars, o + 2, (cx, cy - 1500), np.pi, 0.0)
        elif kind == 3:  # ball at rest in front
            d = rng.uniform(150, 450)
            yaw = rng.uniform(-np.pi, np.pi)
            _place(cars, o + 0, (cx, cy), yaw, rng.uniform(500, 2300))
            balls["pos"]["x"][a], balls["pos"]["y"][a] = cx + np.cos(yaw) * d, cy + np.sin(yaw) * d
            balls["pos"]["z"][a] = rng.choice([93.15, 160.0, 250.0])
            _place(cars, o + 2, (cx, cy + 1500), 0.0, 0.0)
        elif kind == 4:  # ball flying at the car
            d = rng.uniform(300, 600)
            _place(cars, o + 0, (cx, cy), 0.0, rng.uniform(500, 1500))
            balls["pos"]["x"][a], balls["pos"]["y"][a], balls["pos"]["z"][a] = cx + d, cy, rng.uniform(93.15, 200)
            balls["vel"]["x"][a] = -rng.uniform(1000, 3000)
            _place(cars, o + 2, (cx, cy + 1500), 0.0, 0.0)
        else:  # airborne over a ramp corner, falling
            _place(cars, o + 0, (rng.uniform(3300, 3900), rng.uniform(-4700, 4700)), rng.uniform(-np.pi, np.pi),
                   rng.uniform(0, 1500), z=rng.uniform(150, 400), vz=-rng.uniform(0, 800), pitch=rng.uniform(-0.4, 0.4))
            _place(cars, o + 2, (cx, cy), 0.0, 0.0)


def test_contact_scenarios_per_tick(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    n = 360
    eng = rsb.Batch(pkg.engine_library(), n, team_size=2, meshes_path=meshes_dir)
    ora = rsb.Batch(oracle_lib, n, team_size=2, meshes_path=meshes_dir, threads=8)
    rng = np.random.default_rng(2024)
    cars, balls = ora.get_cars(), random_balls(rsb, n, 1)
    _scenes(rsb, cars, balls, ora.car_offset, n, rng)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    ctl = np.zeros(ora.num_cars, rsb.CONTROLS_DTYPE)
    ctl["throttle"] = 1.0
    ctl["boost"] = 1
    for b in (eng, ora):
        b.set_controls(ctl)
    keep_arena = reference_reverse_order(ora, pkg)
    keep = np.repeat(keep_arena, np.diff(ora.car_offset))
    seen = {"demo": 0, "bump": 0, "touch": 0, "wall": 0}
    off_bounds = discrete = total = 0
    for tick in range(60):
        eng.step(1)
        ora.step(1)
        a, b = eng.get_cars()[keep], ora.get_cars()[keep]
        total += len(a)
        discrete += int(flag_mismatch(a, b).sum())
        bad = np.zeros(len(a), bool)
        for f, tol in (("pos", POS_ABS_UU), ("vel", VEL_ABS_UU), ("ang_vel", 1e-3)):
            x, y = vec(a, f), vec(b, f)
            bad |= (np.abs(x - y) > tol + 1e-4 * np.abs(y)).any(axis=1)
        off_bounds += int(bad.sum())
        seen["demo"] += int(b["is_demoed"].sum())
        seen["bump"] += int((b["car_contact_cooldown"] > 0).sum())
        seen["touch"] += int((b["ball_hit_tick"] != np.uint64(0xFFFFFFFFFFFFFFFF)).sum())
        seen["wall"] += int(b["world_contact"].sum())
        co, bo = ora.get_cars(), ora.get_balls()
        for x in (eng, ora):
            x.set_cars(co)
            x.set_balls(bo)
    assert min(seen.values()) > 0, seen
    print(f"CONTACTS {discrete} discrete, {off_bounds} off-bounds of {total} car-ticks ({seen})")
    assert discrete == 0, f"discrete state differs on {discrete} of {total} car-ticks ({seen})"
    assert off_bounds == 0, f"{off_bounds} of {total} car-ticks outside the per-tick bounds ({seen})"
