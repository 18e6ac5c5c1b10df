"""The reset curriculum (rsb_set_reset_curriculum + RSB_RESET_CURRICULUM), the reference
batch's SetResetCurriculum / ResetArena (RocketSimCudaApi.cuh:203-442), pinned statistically:
each arena takes one of kickoff / fuzzed kickoff / aerial / ball chase with the given weights,
and each mode's placements stay inside the reference's ranges."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import vec

pytestmark = pytest.mark.gpu


SPOTS = np.array([[-2048, -2560], [2048, -2560], [-256, -3840], [256, -3840], [0, -4608]], np.float64)
SPOTS = np.concatenate([SPOTS, -SPOTS])


def _near_spot(xy):
    return np.abs(xy[:, None, :] - SPOTS[None]).max(axis=2).min(axis=1)


def _classify(b, c, off):
    """Mode of every arena from its reset state: 0 kickoff, 1 fuzzed, 2 aerial, 3 chase."""
    n = len(b)
    bp, bv = vec(b, "pos"), vec(b, "vel")
    cp = vec(c, "pos")
    mode = np.full(n, -1)
    for a in range(n):
        s = slice(off[a], off[a + 1])
        ground = c["is_on_ground"][s].astype(bool)
        at_spots = _near_spot(cp[s, :2]).max() <= 40.01
        if np.allclose(bp[a], [0, 0, 93.15]) and not bv[a].any():
            mode[a] = 0
        elif (abs(bp[a, 2] - 93.15) < 1e-3 and abs(bp[a, 0]) <= 180 and abs(bp[a, 1]) <= 220 and at_spots
              and (np.abs(bv[a]) <= [90, 90, 35]).all()):
            mode[a] = 1
        elif 420 <= bp[a, 2] <= 780:
            mode[a] = 2
        elif abs(bp[a, 2] - 93.15) < 1e-3 and ground.all():
            mode[a] = 3
    return mode


def test_curriculum_mix_and_ranges(pkg, meshes_dir):
    rsb = pkg.rsb
    n = 4096
    eng = rsb.Batch(pkg.engine_library(), n, team_size=2, meshes_path=meshes_dir)
    eng.set_reset_curriculum(1.0, 1.0, 1.0, 1.0)
    eng.reset_all(0xC0FFEE, rsb.RSB_RESET_CURRICULUM)
    b, c = eng.get_balls(), eng.get_cars()
    off = eng.car_offset
    mode = _classify(b, c, off)
    assert (mode >= 0).all(), f"{int((mode < 0).sum())} arenas match no mode"
    frac = np.bincount(mode, minlength=4) / n
    assert np.abs(frac - 0.25).max() < 0.04, frac
    bp, bv = vec(b, "pos"), vec(b, "vel")
    cp, cv = vec(c, "pos"), vec(c, "vel")
    owner = np.repeat(np.arange(n), np.diff(off))
    # fuzzed: ball velocity within (90, 90, 35); cars within 40 uu of a kickoff spot
    f = mode == 1
    assert (np.abs(bv[f]) <= [90, 90, 35]).all()
    assert _near_spot(cp[f[owner], :2]).max() <= 40.01
    # aerial: exactly one airborne car per arena, below and near the ball, moving up
    ae = mode == 2
    air = ~c["is_on_ground"].astype(bool)
    per = np.bincount(owner, weights=air, minlength=n)
    assert (per[ae] == 1).all()
    sel = ae[owner] & air
    assert (cv[sel, 2] >= 80).all() and (cv[sel, 2] <= 200.01).all()
    horiz = np.linalg.norm(cp[sel, :2] - bp[owner[sel], :2], axis=1)
    assert (horiz >= 179.9).all() and (horiz <= 340.1).all()
    assert (c["boost"][sel] >= 55).all()
    # chase: cars on the ground 450-1850 uu from the ball (less where clamped to the field),
    # facing it, at most 600 uu/s toward it, boost 30-100
    ch = mode == 3
    assert (np.abs(bv[ch]) <= [500, 500, 80]).all()
    sel = ch[owner]
    dist = np.linalg.norm(cp[sel, :2] - bp[owner[sel], :2], axis=1)
    assert dist.max() <= 1850.01
    fwd = vec(c["rot"], "forward")[sel]
    to = bp[owner[sel], :2] - cp[sel, :2]
    to /= np.linalg.norm(to, axis=1, keepdims=True)
    assert (np.sum(fwd[:, :2] * to, axis=1) > 0.999).all()
    assert (np.linalg.norm(cv[sel], axis=1) <= 600.01).all()
    assert (c["boost"][sel] >= 30).all() and (c["boost"][sel] <= 100).all()


def test_curriculum_weights(pkg, meshes_dir):
    rsb = pkg.rsb
    n = 512
    eng = rsb.Batch(pkg.engine_library(), n, team_size=1, meshes_path=meshes_dir)
    for w, want in (((0, 0, 0, 1), 3), ((0, 0, 1, 0), 2), ((-1.0, float("nan"), 0, 0), 0), ((0, 2e6, 0, 0), 0)):
        eng.set_reset_curriculum(*w)
        eng.reset_all(5, rsb.RSB_RESET_CURRICULUM)
        mode = _classify(eng.get_balls(), eng.get_cars(), eng.car_offset)
        assert (mode == want).all(), (w, np.bincount(mode + 1))
