"""ORACLE — test infrastructure only.

CPU restatement, in float64 numpy, of the learned culler's arithmetic: the exact distance
from points to the soccar arena meshes, and the 3 -> 64 -> 64 -> 1 MLP's forward pass,
weighted squared loss and parameter gradients.  The tests use it as the checker of the
library's CUDA kernels (meshDistanceKernel, mlpTrainKernel, mlpPredictKernel).  The culler
has no counterpart in the reference; the meshes are the reference's soccar collision meshes
(soccar/mesh_*.cmf, the files RocketSim::Init loads).  Nothing in the product imports this.
"""
from __future__ import annotations

import glob
import os
import struct

import numpy as np

H = 64
P_W1, P_B1, P_W2, P_B2, P_W3, P_B3 = 0, 192, 256, 256 + 4096, 256 + 4096 + 64, 256 + 4096 + 128
NPARAM = P_B3 + 1
SCALE = np.array([1 / 4096, 1 / 5120, 1 / 2048], np.float64)
OUT = 1000.0
BT_TO_UU = 50.0


def bf16(x):
    """Round float32 values to BF16 (round to nearest even), returned as float32."""
    f = np.ascontiguousarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[P_W1:P_B1].reshape(H, 3), w[P_B1:P_W2], w[P_W2:P_B2].reshape(H, H), w[P_B2:P_W3], w[P_W3:P_B3],
            w[P_B3])


def forward(w, pts):
    """MLP estimate in km for points in uu (weights used as given)."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(pts, np.float64) * SCALE
    h1 = np.maximum(0.0, x @ W1.T + b1)
    z2 = h1 @ W2.T + b2
    y = np.maximum(0.0, z2) @ W3 + b3
    return y, (x, h1, z2)


def loss_and_grad(w, pts, target_uu, over_weight):
    """Mean over the points of w_i (y_i - t_i)^2 (km), w_i = over_weight where y_i > t_i,
    and its gradient with respect to the flat parameter vector."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    y, (x, h1, z2) = forward(w, pts)
    t = np.asarray(target_uu, np.float64) / OUT
    d = y - t
    wt = np.where(d > 0, over_weight, 1.0)
    n = len(y)
    loss = float(np.sum(wt * d * d) / n)
    g = 2.0 * wt * d / n
    h2 = np.maximum(0.0, z2)
    grad = np.zeros(NPARAM)
    grad[P_W3:P_B3] = g @ h2
    grad[P_B3] = g.sum()
    d2 = (g[:, None] * W3[None, :]) * (z2 > 0)
    grad[P_W2:P_B2] = (d2.T @ h1).ravel()
    grad[P_B2:P_W3] = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    grad[P_W1:P_B1] = (d1.T @ x).ravel()
    grad[P_B1:P_W2] = d1.sum(0)
    return loss, grad


def load_mesh_triangles(meshes_dir):
    """All soccar mesh triangles as an (n, 3, 3) array in uu, mesh_0 .. mesh_15 in order."""
    tris = []
    files = sorted(glob.glob(os.path.join(meshes_dir, "soccar", "mesh_*.cmf")),
                   key=lambda f: int(os.path.basename(f)[5:-4]))
    for f in files:
        d = open(f, "rb").read()
        nt, nv = struct.unpack_from("<ii", d, 0)
        idx = np.frombuffer(d, np.int32, 3 * nt, 8).reshape(nt, 3)
        v = np.frombuffer(d, np.float32, 3 * nv, 8 + 12 * nt).reshape(nv, 3).astype(np.float64) * BT_TO_UU
        tris.append(v[idx])
    return np.concatenate(tris)


def point_triangle_distance(pts, tris):
    """Exact Euclidean distance from each point to the nearest triangle (float64).

    For every (point, triangle) pair: the distance to the triangle's plane when the point
    projects inside the triangle, else the smallest distance to its three edge segments."""
    pts = np.asarray(pts, np.float64)
    a, b, c = tris[:, 0], tris[:, 1], tris[:, 2]
    n = np.cross(b - a, c - a)
    nn = np.linalg.norm(n, axis=1)
    ok = nn > 0
    n_unit = np.zeros_like(n)
    n_unit[ok] = n[ok] / nn[ok, None]
    out = np.empty(len(pts))
    for i0 in range(0, len(pts), 256):
        p = pts[i0:i0 + 256, None, :]                      # (P, 1, 3)
        # plane projection and inside test by edge orientation
        dist_plane = np.einsum("ptk,tk->pt", p - a[None], n_unit)
        q = p - dist_plane[..., None] * n_unit[None]
        s0 = np.einsum("ptk,tk->pt", np.cross(b - a, q - a[None]), n)
        s1 = np.einsum("ptk,tk->pt", np.cross(c - b, q - b[None]), n)
        s2 = np.einsum("ptk,tk->pt", np.cross(a - c, q - c[None]), n)
        inside = (s0 >= 0) & (s1 >= 0) & (s2 >= 0) & ok[None]

        def seg(u, v):
            uv = v - u
            t = np.clip(np.einsum("ptk,tk->pt", p - u[None], uv) / np.maximum(np.einsum("tk,tk->t", uv, uv), 1e-300),
                        0.0, 1.0)
            c_ = u[None] + t[..., None] * uv[None]
            return np.linalg.norm(p - c_, axis=-1)

        edge = np.minimum(np.minimum(seg(a, b), seg(b, c)), seg(c, a))
        d = np.where(inside, np.abs(dist_plane), edge)
        out[i0:i0 + 256] = d.min(axis=1)
    return out
