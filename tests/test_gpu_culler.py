"""The learned culler's CUDA kernels against the CPU restatement in oracle/culler_ref.py,
its training and margin calibration, and the culled step against the exact step.

  * exact point-to-mesh distances: within 0.05 uu (+1e-5 relative) of float64;
  * MLP estimates and the loss gradient of the fused forward/backward training kernel:
    within 1e-4 / 1e-3 relative of float64 with the same BF16 weights;
  * a trained culler has zero held-out misses, and the learned step reproduces the exact
    step bit for bit while the audit counts no missed contact.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import culler_ref as cr  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tris(meshes_dir):
    return cr.load_mesh_triangles(meshes_dir)


def _batch(pkg, meshes_dir, n=64, team_size=3, cull=0, **kw):
    return pkg.rsb.Batch(pkg.engine_library(), n, team_size=team_size, meshes_path=meshes_dir, cull_mode=cull, **kw)


def _random_points(rng, n):
    return np.stack([rng.uniform(-4300, 4300, n), rng.uniform(-6100, 6100, n), rng.uniform(-100, 2150, n)], 1)


def test_mesh_distance_matches_cpu(pkg, meshes_dir, tris):
    assert len(tris) == 8020
    b = _batch(pkg, meshes_dir)
    rng = np.random.default_rng(1)
    pts = _random_points(rng, 384).astype(np.float32)
    # also points right on and next to the walls, ramps and goals
    near = tris[rng.integers(0, len(tris), 128)].mean(axis=1) + rng.normal(0, 30, (128, 3))
    pts = np.concatenate([pts, near.astype(np.float32)])
    got = b.culler_distance(pts)
    ref = cr.point_triangle_distance(pts.astype(np.float64), tris)
    assert np.all(np.abs(got - ref) <= 0.05 + 1e-5 * ref), np.abs(got - ref).max()


def _random_weights(rng):
    w = np.zeros(cr.NPARAM, np.float32)
    w[cr.P_W1:cr.P_B1] = rng.uniform(-1, 1, 192) * np.sqrt(6 / 3)
    w[cr.P_B1:cr.P_W2] = rng.uniform(-0.1, 0.1, 64)
    w[cr.P_W2:cr.P_B2] = rng.uniform(-1, 1, 4096) * np.sqrt(6 / 64)
    w[cr.P_B2:cr.P_W3] = rng.uniform(-0.1, 0.1, 64)
    w[cr.P_W3:cr.P_B3] = rng.uniform(-1, 1, 64) * np.sqrt(6 / 64)
    w[cr.P_B3] = 0.3
    return w


def test_predict_and_gradients_match_cpu(pkg, meshes_dir):
    b = _batch(pkg, meshes_dir)
    rng = np.random.default_rng(2)
    w = _random_weights(rng)
    b.culler_set(w, 0.0)
    wb = cr.bf16(w)
    pts = _random_points(rng, 3000).astype(np.float32)
    target = rng.uniform(0, 2500, len(pts)).astype(np.float32)
    pred = b.culler_predict(pts)
    y, _ = cr.forward(wb, pts)
    assert np.allclose(pred, y * cr.OUT, rtol=1e-4, atol=1e-2)
    g, loss = b.culler_gradients(pts, target, over_weight=4.0)
    ref_loss, ref_g = cr.loss_and_grad(wb, pts, target, 4.0)
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss) + 1e-7
    for lo, hi in ((cr.P_W1, cr.P_B1), (cr.P_B1, cr.P_W2), (cr.P_W2, cr.P_B2), (cr.P_B2, cr.P_W3),
                   (cr.P_W3, cr.P_B3), (cr.P_B3, cr.NPARAM)):
        scale = np.abs(ref_g[lo:hi]).max()
        assert np.allclose(g[lo:hi], ref_g[lo:hi], rtol=1e-3, atol=1e-4 * scale), (lo, hi)


@pytest.fixture(scope="module")
def trained(pkg, meshes_dir):
    """A culler trained on logged centres of random-state and high-contact rollouts."""
    rsb = pkg.rsb
    b = _batch(pkg, meshes_dir, n=4096, team_size=3)
    b.set_action_lut(rsb.default_action_lut(b.lib))
    rng = np.random.default_rng(3)
    for k in range(12):
        b.reset_all(100 + k, rsb.RSB_RESET_RANDOM_STATE if k % 3 else rsb.RSB_RESET_HIGH_CONTACT)
        for _ in range(4):
            b.set_actions(rng.integers(0, 90, b.num_cars).astype(np.int32))
            b.step(8)
            b.culler_log()
    rep = b.culler_train(rsb.culler_config(train_points=600_000, heldout_points=150_000, epochs=12))
    w, margin = b.culler_get()
    return rep, w, margin


def test_training_calibrates_zero_misses(pkg, meshes_dir, trained):
    rep, w, margin = trained
    assert rep["logged_points"] > 0 and rep["steps"] > 0
    assert rep["heldout_misses"] == 0
    assert 0 < rep["margin"] < 1000 and rep["heldout_mae"] < 300, rep
    # on fresh points the calibrated bound still holds almost everywhere
    b = _batch(pkg, meshes_dir)
    b.culler_set(w, margin)
    rng = np.random.default_rng(4)
    pts = _random_points(rng, 20000).astype(np.float32)
    d = b.culler_distance(pts)
    bound = b.culler_predict(pts) - margin
    assert (bound > d).mean() < 1e-3


def test_learned_step_matches_exact(pkg, meshes_dir, trained):
    rsb = pkg.rsb
    _, w, margin = trained
    n = 2048
    runs = {}
    for mode in (rsb.RSB_CULL_EXACT, rsb.RSB_CULL_LEARNED, rsb.RSB_CULL_LEARNED_AUDIT):
        b = _batch(pkg, meshes_dir, n=n, team_size=3, cull=mode)
        b.set_action_lut(rsb.default_action_lut(b.lib))
        if mode != rsb.RSB_CULL_EXACT:
            b.culler_set(w, margin)
        b.reset_all(7, rsb.RSB_RESET_RANDOM_STATE)
        b.reset_arenas(np.arange(0, n, 4, dtype=np.int32), 8, rsb.RSB_RESET_HIGH_CONTACT)
        rng = np.random.default_rng(5)
        for _ in range(8):
            b.set_actions(rng.integers(0, 90, b.num_cars).astype(np.int32))
            b.step(8)
        runs[mode] = (b.get_cars().tobytes(), b.get_balls().tobytes(), b.stats())
    ex, le, au = runs[rsb.RSB_CULL_EXACT], runs[rsb.RSB_CULL_LEARNED], runs[rsb.RSB_CULL_LEARNED_AUDIT]
    assert au[2]["missed_contacts"] == 0 and au[2]["arenas_reverted"] == 0
    assert le[2]["culled_queries"] > 0
    assert le[2]["narrowphase_queries"] < ex[2]["narrowphase_queries"]
    assert le[0] == ex[0] and le[1] == ex[1]
    assert au[0] == ex[0] and au[1] == ex[1]


def _culled_runs(pkg, meshes_dir, modes, w=None, margin=None, n=2048):
    """The same seeded rollout (random-state starts, a quarter of the arenas high-contact) under
    each cull mode: final states and the library's counters."""
    rsb = pkg.rsb
    runs = {}
    for mode in modes:
        b = _batch(pkg, meshes_dir, n=n, team_size=3, cull=mode)
        b.set_action_lut(rsb.default_action_lut(b.lib))
        if mode in (rsb.RSB_CULL_LEARNED, rsb.RSB_CULL_LEARNED_AUDIT):
            b.culler_set(w, margin)
        b.reset_all(7, rsb.RSB_RESET_RANDOM_STATE)
        b.reset_arenas(np.arange(0, n, 4, dtype=np.int32), 8, rsb.RSB_RESET_HIGH_CONTACT)
        rng = np.random.default_rng(5)
        for _ in range(8):
            b.set_actions(rng.integers(0, 90, b.num_cars).astype(np.int32))
            b.step(8)
        runs[mode] = (b.get_cars().tobytes(), b.get_balls().tobytes(), b.stats())
    return runs


def test_voxel_bound_step_matches_exact(pkg, meshes_dir):
    """RSB_CULL_VOXEL skips the static tests of bodies its (exact) voxel distance bound clears:
    the step equals the exact step bit for bit, and under audit the skipped tests find nothing."""
    rsb = pkg.rsb
    runs = _culled_runs(pkg, meshes_dir, (rsb.RSB_CULL_EXACT, rsb.RSB_CULL_VOXEL, rsb.RSB_CULL_VOXEL_AUDIT))
    ex, vx, au = runs[rsb.RSB_CULL_EXACT], runs[rsb.RSB_CULL_VOXEL], runs[rsb.RSB_CULL_VOXEL_AUDIT]
    assert vx[2]["culled_queries"] > 0
    assert au[2]["missed_contacts"] == 0 and au[2]["arenas_reverted"] == 0
    assert vx[0] == ex[0] and vx[1] == ex[1]
    assert au[0] == ex[0] and au[1] == ex[1]


def test_learned_bound_against_voxel_bound(pkg, meshes_dir, trained):
    """What the trained network adds over the bound that needs no training, on one rollout:
    the share of static tests each skips (printed).  The voxel bound is exact but coarse (64 uu
    voxels, less their diagonal); the network's estimate is finer but gives up its calibrated
    margin everywhere.  Both skip some tests and leave the results bit-identical."""
    rsb = pkg.rsb
    _, w, margin = trained
    runs = _culled_runs(pkg, meshes_dir, (rsb.RSB_CULL_LEARNED, rsb.RSB_CULL_VOXEL), w, margin)
    le, vx = runs[rsb.RSB_CULL_LEARNED][2], runs[rsb.RSB_CULL_VOXEL][2]
    share = lambda s: s["culled_queries"] / max(1, s["culled_queries"] + s["narrowphase_queries"])
    print(f"CULL learned skips {share(le):.4f} of static tests, voxel {share(vx):.4f}, margin {margin:.1f} uu")
    assert runs[rsb.RSB_CULL_LEARNED][0] == runs[rsb.RSB_CULL_VOXEL][0]
    assert share(le) > 0 and share(vx) > 0
