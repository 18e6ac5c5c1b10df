"""Free-running lockstep comparison of an engine build (CUDA or host) with the oracle.

Both sides step from identical state with identical controls and are compared byte for
byte after every step: every car, ball and boost-pad state of every arena.  An arena leaves
the comparison only for reasons that lie in the reference's process, not in the simulation:
  * the reference visits its cars in another order than the engine (its car set is an
    unordered_set hashed by heap address): gpu_util.reference_reverse_order;
  * a demolished car respawned: RocketSim draws the respawn spot from a process-global
    random engine (Car::Respawn, Car.cpp:43-56).  lockstep_gate() resyncs such an arena from
    the oracle and compares it again from the next step on; run_lockstep() drops it.
"""
from __future__ import annotations

import numpy as np

from gpu_util import random_balls, random_cars, random_controls, reference_reverse_order


def rows(a, n):
    return a.view(np.uint8).reshape(n, -1)


def arena_diff(eng, ora, owner, n):
    """Per arena: True where any car, ball or pad byte differs."""
    a, b = eng.get_cars(), ora.get_cars()
    bad = np.zeros(n, bool)
    np.logical_or.at(bad, owner, (rows(a, len(a)) != rows(b, len(b))).any(axis=1))
    bad |= (rows(eng.get_balls(), n) != rows(ora.get_balls(), n)).any(axis=1)
    bad |= (rows(eng.get_pads(), n) != rows(ora.get_pads(), n)).any(axis=1)
    return bad


def run_lockstep(rsb, pkg, eng_lib, ora_lib, meshes_dir, team_size, n, seed, ticks, team_sizes=None):
    """Free-running `ticks` single-tick steps with controls redrawn every 8 ticks.  Returns
    (arenas compared, arenas that differed before leaving, arenas dropped after a respawn,
    (arena, tick) of the first difference or None)."""
    kw = dict(team_size=None, team_sizes=team_sizes) if team_sizes is not None else dict(team_size=team_size)
    eng = rsb.Batch(eng_lib, n, meshes_path=meshes_dir, threads=8, **kw)
    ora = rsb.Batch(ora_lib, n, meshes_path=meshes_dir, threads=8, **kw)
    cars = random_cars(rsb, ora.get_cars(), seed)
    balls = random_balls(rsb, n, seed + 1, rest_fraction=0.0)
    balls["pos"]["z"] = np.random.default_rng(seed).uniform(93.15, 1300, n)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    live = reference_reverse_order(ora, pkg)
    compared = int(live.sum())
    owner = np.repeat(np.arange(n), np.diff(ora.car_offset))
    differed = np.zeros(n, bool)
    respawned = np.zeros(n, bool)
    first = None
    rng = np.random.default_rng(seed + 2)
    prev_demoed = ora.get_cars()["is_demoed"].astype(bool)
    for tick in range(ticks):
        if tick % 8 == 0:
            ctl = random_controls(rsb, eng.num_cars, rng)
            eng.set_controls(ctl)
            ora.set_controls(ctl)
        eng.step(1)
        ora.step(1)
        demoed = ora.get_cars()["is_demoed"].astype(bool)
        resp = np.zeros(n, bool)
        np.logical_or.at(resp, owner, prev_demoed & ~demoed)
        prev_demoed = demoed
        respawned |= resp & live
        live &= ~resp
        bad = arena_diff(eng, ora, owner, n) & live
        if bad.any() and first is None:
            first = (int(np.nonzero(bad)[0][0]), tick)
        differed |= bad
        live &= ~bad
    eng.close()
    ora.close()
    return compared, int(differed.sum()), int(respawned.sum()), first


def sync_arenas(eng, ora, arenas):
    """Writes the oracle's car, ball and pad states of the listed arenas into both sides."""
    for a in arenas:
        a = int(a)
        for c in range(int(ora.car_offset[a + 1] - ora.car_offset[a])):
            s = ora.get_car(a, c)
            eng.set_car(a, c, s)
            ora.set_car(a, c, s)
        b = ora.get_ball(a)
        eng.set_ball(a, b)
        ora.set_ball(a, b)
        p = ora.get_arena_pads(a)
        eng.set_arena_pads(a, p)
        ora.set_arena_pads(a, p)


def sync_all(eng, ora):
    cars, balls, pads = ora.get_cars(), ora.get_balls(), ora.get_pads()
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
        b.set_pads(pads)
