"""The CPU restatement of the culler's arithmetic (oracle/culler_ref.py) on cases with known
answers, so that the GPU checks against it rest on a checked base.  CPU only."""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import culler_ref as cr  # noqa: E402


def test_point_triangle_distance_known_cases():
    tri = np.array([[[0, 0, 0], [10, 0, 0], [0, 10, 0]]], np.float64)
    cases = [((2, 2, 5), 5.0), ((-3, -4, 0), 5.0), ((5, -2, 0), 2.0), ((20, 0, 0), 10.0), ((6, 6, 0), np.sqrt(2.0))]
    for p, d in cases:
        assert abs(cr.point_triangle_distance(np.array([p], np.float64), tri)[0] - d) < 1e-12


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(0, 0.3, cr.NPARAM)
    pts = np.stack([rng.uniform(-4000, 4000, 64), rng.uniform(-5000, 5000, 64), rng.uniform(0, 2000, 64)], 1)
    t = rng.uniform(0, 2000, 64)
    _, g = cr.loss_and_grad(w, pts, t, 4.0)
    for k in rng.integers(0, cr.NPARAM, 40):
        e = np.zeros(cr.NPARAM)
        e[k] = 1e-6
        fd = (cr.loss_and_grad(w + e, pts, t, 4.0)[0] - cr.loss_and_grad(w - e, pts, t, 4.0)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-5 + 1e-4 * abs(g[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159], np.float32)
    r = cr.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125) and abs(r[3] + 3.140625) < 1e-6


def test_mesh_triangles(meshes_dir):
    t = cr.load_mesh_triangles(meshes_dir)
    assert t.shape == (8020, 3, 3)
    assert np.abs(t[..., 0]).max() < 4200 and np.abs(t[..., 1]).max() < 6100


def test_voxel_bound_is_a_lower_bound(pkg, meshes_dir):
    """The voxel distance field behind RSB_CULL_VOXEL (built on the host from the mesh
    occupancy grid) never exceeds the exact float64 distance to the arena meshes, and is
    informative away from them."""
    import ctypes as C

    from host_util import build_host_engine

    rsb = pkg.rsb
    lib = rsb.load_library(build_host_engine())
    fn = lib.rsb_host_voxel_bound
    fn.restype = C.c_int32
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    b = rsb.Batch(lib, 1, team_size=1, meshes_path=meshes_dir, threads=1)
    tris = cr.load_mesh_triangles(meshes_dir)
    rng = np.random.default_rng(9)
    n = 3000
    pts = np.stack([rng.uniform(-4400, 4400, n), rng.uniform(-6300, 6300, n), rng.uniform(-200, 2300, n)], 1)
    near = tris[rng.integers(0, len(tris), 1000)].mean(axis=1) + rng.normal(0, 150, (1000, 3))
    pts = np.concatenate([pts, near]).astype(np.float32)
    out = np.zeros(len(pts), np.float32)
    assert fn(b._h, pts.ctypes.data, len(pts), out.ctypes.data) == 0
    exact = cr.point_triangle_distance(pts.astype(np.float64), tris)
    assert (out <= exact + 1e-3).all(), f"bound above the exact distance by {float((out - exact).max()):.3g} uu"
    far = exact > 400
    assert far.any() and np.median(out[far] / exact[far]) > 0.5
