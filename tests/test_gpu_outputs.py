"""rsb_copy_outputs and page-locked host buffers: the four outputs in one call equal the
four single copies, in registered (pinned) arrays reused across steps."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_copy_outputs_into_pinned_buffers(pkg, meshes_dir):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    b = rsb.Batch(lib, 96, team_sizes=np.array([1, 2, 3] * 32, np.int32), meshes_path=meshes_dir,
                  rewards=rsb.default_rewards(lib))
    b.reset_all(3, rsb.RSB_RESET_RANDOM_STATE)
    b.set_action_lut(rsb.default_action_lut(lib))
    outs = b.pinned_outputs()
    acts = b.pin(np.random.default_rng(0).integers(0, rsb.RSB_NUM_ACTIONS, (2, b.num_cars)).astype(np.int32))
    for k in range(2):
        b.set_actions(acts[k])
        b.step(8)
        b.build_obs()
        b.build_rewards_terminals(8)
        b.copy_outputs(outs)
        assert np.array_equal(outs["obs"], b.copy_obs())
        assert np.array_equal(outs["masks"], b.copy_masks())
        assert np.array_equal(outs["rewards"], b.copy_rewards())
        assert np.array_equal(outs["terminals"], b.copy_terminals())
    b.close()
