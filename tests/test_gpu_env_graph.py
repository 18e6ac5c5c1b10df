"""The captured env step (rsb_env_graph_capture / rsb_env_graph_launch) against the same
calls made one by one: after every replay, observations, masks, rewards, terminals and the
arena states are bit-identical to the eager sequence rsb_set_actions_device, rsb_step,
rsb_build_obs, rsb_build_rewards_terminals, rsb_reset_done(seed + k).  The reset seed
advancing on the device is what keeps replays from resetting every finished arena the same
way, so the test drives goals (balls flying at a goal) and checks that arenas reset."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    assert torch.cuda.is_available()
    return torch


def _make(pkg, meshes_dir, n, cull):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    b = rsb.Batch(lib, n, team_size=3, meshes_path=meshes_dir, rewards=rsb.default_rewards(lib))
    b.set_action_lut(rsb.default_action_lut(lib))
    b.set_cull_mode(cull)
    return b


def _goal_scene(b, seed):
    """Random-state start; in every third arena the ball flies at a goal from 600 uu out."""
    balls = b.get_balls()
    rng = np.random.default_rng(seed)
    for a in range(0, b.num_arenas, 3):
        sgn = 1.0 if rng.random() < 0.5 else -1.0
        balls["pos"]["x"][a] = rng.uniform(-500, 500)
        balls["pos"]["y"][a] = sgn * 4500.0
        balls["pos"]["z"][a] = 250.0
        balls["vel"]["x"][a], balls["vel"]["y"][a], balls["vel"]["z"][a] = 0.0, sgn * 3000.0, 0.0
        for c in "xyz":
            balls["ang_vel"][c][a] = 0.0
    return balls


@pytest.mark.parametrize("cull", ["exact", "voxel"])
def test_graph_replays_match_eager_steps(pkg, meshes_dir, cull):
    torch = _torch()
    rsb = pkg.rsb
    mode = {"exact": rsb.RSB_CULL_EXACT, "voxel": rsb.RSB_CULL_VOXEL}[cull]
    n, tick_skip, steps, seed = 1536, 8, 24, 0xA11CE
    g, e = _make(pkg, meshes_dir, n, mode), _make(pkg, meshes_dir, n, mode)
    for b in (g, e):
        b.reset_all(41, rsb.RSB_RESET_RANDOM_STATE)
    balls = _goal_scene(g, 3)
    for b in (g, e):
        b.set_balls(balls)
    acts = torch.zeros(g.num_cars, dtype=torch.int32, device="cuda")
    g.env_graph_capture(acts.data_ptr(), tick_skip, rsb.RSB_RESET_RANDOM_STATE, seed)
    rng = np.random.default_rng(11)
    resets = 0
    for k in range(steps):
        a = rng.integers(0, 90, g.num_cars).astype(np.int32)
        acts.copy_(torch.from_numpy(a))
        torch.cuda.synchronize()
        g.env_graph_launch()
        e.set_actions_device(acts.data_ptr(), e.num_cars)
        e.step(tick_skip)
        e.build_obs()
        e.build_rewards_terminals(tick_skip)
        e.reset_done(seed + k, rsb.RSB_RESET_RANDOM_STATE)
        g.sync()
        e.sync()
        tg, te = g.copy_terminals(), e.copy_terminals()
        assert (tg == te).all(), f"step {k}: terminals differ"
        resets += int(tg.sum())
        assert g.copy_obs().tobytes() == e.copy_obs().tobytes(), f"step {k}: observations differ"
        assert (g.copy_masks() == e.copy_masks()).all(), f"step {k}: masks differ"
        assert g.copy_rewards().tobytes() == e.copy_rewards().tobytes(), f"step {k}: rewards differ"
        assert g.get_cars().tobytes() == e.get_cars().tobytes(), f"step {k}: cars differ"
        assert g.get_balls().tobytes() == e.get_balls().tobytes(), f"step {k}: balls differ"
    assert resets > 0, "no arena finished, so the advancing seed went untested"
    sg, se = g.stats(), e.stats()
    assert sg["ticks_simulated"] == se["ticks_simulated"]
    g.close()
    e.close()


def test_graph_capture_errors(pkg, meshes_dir):
    torch = _torch()
    rsb = pkg.rsb
    lib = pkg.engine_library()
    b = rsb.Batch(lib, 64, team_size=1, meshes_path=meshes_dir)
    acts = torch.zeros(b.num_cars, dtype=torch.int32, device="cuda")
    with pytest.raises(rsb.RsbError):
        b.env_graph_launch()  # nothing captured
    with pytest.raises(rsb.RsbError):
        b.env_graph_capture(acts.data_ptr(), 8, rsb.RSB_RESET_KICKOFF, 1)  # no action table, no rewards
    b.set_action_lut(rsb.default_action_lut(lib))
    with pytest.raises(rsb.RsbError):
        b.env_graph_capture(acts.data_ptr(), 8, rsb.RSB_RESET_KICKOFF, 1)  # no reward configuration
    with pytest.raises(rsb.RsbError):
        b.env_graph_capture(acts.data_ptr(), 0, rsb.RSB_RESET_KICKOFF, 1)
    b.close()
