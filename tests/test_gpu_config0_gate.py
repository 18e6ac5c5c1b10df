"""Parity gate on the reference's CPU-runnable workload: soccar 1v1 x 64 arenas, tickSkip 8,
2,000 env steps (16,000 ticks), uniform random discrete actions, goal and 1,800-tick terminals.

Every env step both sides start from the oracle's state (cars, ball, pads written into both),
take the same actions for 8 ticks, and are compared: car and ball positions within 1 uu and
the discrete car state equal on at least 99.9 % of car-steps (8 free ticks let the one-ulp
differences grow a little through contacts; tests/test_gpu_cars.py bounds single ticks).  On
the state both then share, observations, masks, rewards and terminals must be bit-identical;
finished arenas reset on both sides (random-state starts) and the engine takes the oracle's
new state.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import flag_mismatch, reference_reverse_order, vec

pytestmark = pytest.mark.gpu


def test_config0_two_thousand_env_steps(pkg, oracle_lib, meshes_dir):
    rsb = pkg.rsb
    n, steps, tick_skip = 64, 2000, 8
    eng = rsb.Batch(pkg.engine_library(), n, team_size=1, meshes_path=meshes_dir,
                    rewards=rsb.default_rewards(pkg.engine_library(), episode_max_ticks=1800))
    ora = rsb.Batch(oracle_lib, n, team_size=1, meshes_path=meshes_dir, threads=8,
                    rewards=rsb.default_rewards(oracle_lib, episode_max_ticks=1800))
    lut = rsb.default_action_lut(pkg.engine_library())
    for b in (eng, ora):
        b.set_action_lut(lut)
    ora.reset_all(0x5EED0000, rsb.RSB_RESET_KICKOFF)

    def sync():
        cars, balls, pads = ora.get_cars(), ora.get_balls(), ora.get_pads()
        for b in (eng, ora):
            b.set_cars(cars)
            b.set_balls(balls)
            b.set_pads(pads)

    sync()
    keep_arena = reference_reverse_order(ora, pkg)
    keep = np.repeat(keep_arena, np.diff(ora.car_offset))
    rng = np.random.default_rng(0x5EED0000)
    total = off = discrete = goals = truncs = 0
    for step in range(steps):
        idx = rng.integers(0, rsb.RSB_NUM_ACTIONS, eng.num_cars).astype(np.int32)
        for b in (eng, ora):
            b.snapshot()
            b.set_actions(idx)
            b.step(tick_skip)
        a, o = eng.get_cars()[keep], ora.get_cars()[keep]
        total += len(a)
        discrete += int(flag_mismatch(a, o).sum())
        d = np.linalg.norm(vec(a, "pos") - vec(o, "pos"), axis=1)
        off += int((d > 1.0).sum())
        ba, bo = eng.get_balls()[keep_arena], ora.get_balls()[keep_arena]
        off += int((np.linalg.norm(vec(ba, "pos") - vec(bo, "pos"), axis=1) > 1.0).sum())
        sync()
        for b in (eng, ora):
            b.build_obs()
            b.build_rewards_terminals(tick_skip)
        oe, oo = eng.copy_obs(), ora.copy_obs()
        same = (oe.view(np.uint32) == oo.view(np.uint32)).all(axis=1)
        assert (same | ~keep).all(), f"step {step}: observation rows differ"
        assert (eng.copy_masks() == ora.copy_masks()).all(axis=1)[keep].all(), f"step {step}: masks differ"
        re_, ro = eng.copy_rewards(), ora.copy_rewards()
        assert (re_.view(np.uint32) == ro.view(np.uint32))[keep].all(), f"step {step}: rewards differ"
        te, to = eng.copy_terminals(), ora.copy_terminals()
        assert (te == to)[keep_arena].all(), f"step {step}: terminals differ"
        goals += int((to == 1).sum())
        truncs += int((to == 2).sum())
        done = np.nonzero(to)[0].astype(np.int32)
        if done.size:
            # both reset (episode counters), then both take the oracle's new state
            for b in (eng, ora):
                b.reset_arenas(done, 0x5EED1000 + step, rsb.RSB_RESET_RANDOM_STATE)
            sync()
    print(f"GATE car-steps={total} discrete={discrete} off={off} goals={goals} truncations={truncs}")
    assert goals > 0 and truncs > 0, (goals, truncs)
    assert discrete <= 1e-3 * total, f"discrete car state differs on {discrete} of {total} car-steps"
    assert off <= 1e-3 * total, f"{off} of {total} car- or ball-steps more than 1 uu apart"
