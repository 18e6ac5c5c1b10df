"""Generates soccar_trajectories.npz: 120-tick rollouts of the reference CPU RocketSim (the
oracle, oracle/_ref/librsref.so, built from the reference's sources) for a ragged batch of
1v1 / 2v2 / 3v3 arenas from seeded states, with a new discrete action per car every 8 ticks.

    python tests/golden/make_golden.py

Stored: the initial car / ball states (the C ABI's rsb_car_state / rsb_ball_state bytes),
the action indices, the action table, every tick's car and ball kinematics and car flags,
and the order in which the reference visited each arena's cars (its car set is hashed by
heap address, so the order can differ between processes).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from conftest import ORACLE_LIB, load_pkg  # noqa: E402
from gpu_util import random_balls, random_cars  # noqa: E402

TEAM_SIZES = np.array([1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3], np.int32)
TICKS = 120
ACTION_EVERY = 8
SEED = 0x5EED0000
FLAG_FIELDS = ("is_on_ground", "has_jumped", "has_double_jumped", "has_flipped", "is_flipping", "is_jumping",
               "is_supersonic", "is_auto_flipping", "is_demoed", "world_contact", "ball_hit_valid")


def car_flags(cars):
    f = np.zeros(len(cars), np.uint32)
    for k, name in enumerate(FLAG_FIELDS):
        f |= (cars[name].astype(np.uint32) & 1) << k
    for w in range(4):
        f |= (cars["wheels_with_contact"][:, w].astype(np.uint32) & 1) << (16 + w)
    return f


def kin(arr):
    return np.stack([np.stack([arr[f][c] for c in "xyz"], -1) for f in ("pos", "vel", "ang_vel")], 1).astype(np.float32)


def initial_state(rsb, batch):
    n = batch.num_arenas
    cars = random_cars(rsb, batch.get_cars(), SEED)
    balls = random_balls(rsb, n, SEED + 1, rest_fraction=0.0)
    rng = np.random.default_rng(SEED + 2)
    balls["pos"]["z"] = rng.uniform(93.15, 1300, n)
    # every other arena: ball just in front of the first car (touches early)
    off = batch.car_offset
    for a in range(0, n, 2):
        c = cars[off[a]]
        fwd = np.array([c["rot"]["forward"][k] for k in "xy"])
        balls["pos"]["x"][a] = c["pos"]["x"] + fwd[0] * 250
        balls["pos"]["y"][a] = c["pos"]["y"] + fwd[1] * 250
        balls["pos"]["z"][a] = 93.15
        for k in "xyz":
            balls["vel"][k][a] = 0.0
    return cars, balls


def run(batch, cars, balls, actions, rsb):
    batch.set_cars(cars)
    batch.set_balls(balls)
    car_kin, car_flag, car_boost, ball_kin = [], [], [], []
    for t in range(TICKS):
        if t % ACTION_EVERY == 0:
            batch.set_actions(actions[t // ACTION_EVERY])
        batch.step(1)
        c, b = batch.get_cars(), batch.get_balls()
        car_kin.append(kin(c))
        car_flag.append(car_flags(c))
        car_boost.append(c["boost"].astype(np.float32))
        ball_kin.append(kin(b))
    return np.stack(car_kin), np.stack(car_flag), np.stack(car_boost), np.stack(ball_kin)


def car_order(batch):
    import ctypes as C
    fn = batch.lib.rsbref_car_order
    fn.restype = C.c_int32
    fn.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    out = np.full((batch.num_arenas, 6), -1, np.int32)
    buf = np.zeros(8, np.int32)
    for a in range(batch.num_arenas):
        k = fn(batch._h, a, buf.ctypes.data)
        out[a, :k] = buf[:k]
    return out


def main():
    rsb = load_pkg().rsb
    lib = rsb.load_library(ORACLE_LIB)
    pkg = load_pkg()
    # the reference visits an arena's cars in the order of its pointer set; record a batch in
    # which every arena visits them in reverse creation order (the engine's order)
    kept, batch = [], None
    for _ in range(200):
        b = rsb.Batch(lib, len(TEAM_SIZES), team_sizes=TEAM_SIZES, meshes_path=pkg.MESHES_DIR, threads=1)
        order = car_order(b)
        if all(np.array_equal(order[a, :2 * t], np.arange(2 * t)[::-1]) for a, t in enumerate(TEAM_SIZES)):
            batch = b
            break
        kept.append(b)  # keep it alive so the next batch's cars get other addresses
    if batch is None:
        raise RuntimeError("no batch with every arena in reverse creation order")
    lut = rsb.default_action_lut(lib)
    batch.set_action_lut(lut)
    cars, balls = initial_state(rsb, batch)
    rng = np.random.default_rng(SEED + 3)
    actions = rng.integers(0, rsb.RSB_NUM_ACTIONS, (TICKS // ACTION_EVERY, batch.num_cars)).astype(np.int32)
    car_kin, car_flag, car_boost, ball_kin = run(batch, cars, balls, actions, rsb)
    np.savez_compressed(os.path.join(HERE, "soccar_trajectories.npz"),
                        team_sizes=TEAM_SIZES, init_cars=np.frombuffer(cars.tobytes(), np.uint8),
                        init_balls=np.frombuffer(balls.tobytes(), np.uint8), actions=actions,
                        lut=np.frombuffer(lut.tobytes(), np.uint8), car_kin=car_kin, car_flags=car_flag,
                        car_boost=car_boost, ball_kin=ball_kin, car_order=car_order(batch),
                        ticks=np.int32(TICKS), action_every=np.int32(ACTION_EVERY))


if __name__ == "__main__":
    main()
