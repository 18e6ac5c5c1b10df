"""rsb_set_actions_host_static against rsb_set_actions_host: the same actions staged
through the library's static device array give the same simulation, on two calls in a
row; oversize requests are refused with a clear error."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(pkg, meshes_dir, n, team_size):
    rsb = pkg.rsb
    lut = rsb.default_action_lut(pkg.engine_library())
    a = rsb.Batch(pkg.engine_library(), n, team_size=team_size, meshes_path=meshes_dir)
    b = rsb.Batch(pkg.engine_library(), n, team_size=team_size, meshes_path=meshes_dir)
    for x in (a, b):
        x.set_action_lut(lut)
    return a, b


def test_static_actions_match_allocating_path_twice(pkg, meshes_dir):
    a, b = _pair(pkg, meshes_dir, 64, 3)
    rng = np.random.default_rng(11)
    for _ in range(2):
        idx = rng.integers(0, pkg.rsb.RSB_NUM_ACTIONS, a.num_cars).astype(np.int32)
        a.set_actions(idx)
        b.set_actions_static(idx)
        a.step(8)
        b.step(8)
        assert a.get_cars().tobytes() == b.get_cars().tobytes()
        assert a.get_balls().tobytes() == b.get_balls().tobytes()


def test_static_actions_allocate_no_device_memory(pkg, meshes_dir):
    """After the first call on the device (which looks up the array's address), further calls
    leave the device's free memory unchanged."""
    import gc

    import torch

    a, b = _pair(pkg, meshes_dir, 4096, 3)
    a.close()
    gc.collect()  # batches of earlier tests release their device memory before the window
    rng = np.random.default_rng(12)
    idx = rng.integers(0, pkg.rsb.RSB_NUM_ACTIONS, b.num_cars).astype(np.int32)
    b.set_actions_static(idx)
    b.sync()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        b.set_actions_static(rng.integers(0, pkg.rsb.RSB_NUM_ACTIONS, b.num_cars).astype(np.int32))
    b.sync()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"


def test_static_actions_reject_oversize(pkg, meshes_dir):
    rsb = pkg.rsb
    a, _ = _pair(pkg, meshes_dir, 2, 1)
    too_many = np.zeros(rsb.RSB_STATIC_ACTIONS_MAX + 1, np.int32)
    with pytest.raises(rsb.RsbError) as e:
        a.set_actions_static(too_many)
    assert e.value.code == -1
    assert "RSB_STATIC_ACTIONS_MAX" in str(e.value)
