// Wheel ray casts against the static arena (btCollisionWorld::rayTest through the RocketSim
// broadphase, btCollisionWorld.cpp:877-966, btRSBroadphase.cpp:325-356).
//
// The suspension-grid shortcut is compiled out of the reference build (RS_NO_SUSPCOLGRID,
// Framework.h:111), so every wheel ray is a full ray test against the objects registered
// in the broadphase cell of the ray start: arena meshes (btTriangleRaycastCallback over the
// BVH, btRaycastCallback.cpp:31-108), the static planes (two large triangles,
// btStaticPlaneShape::processAllTriangles), and dynamic bodies.
//
// ALTERED SOURCE: this file is not the original Bullet code.  It restates the algorithms of
// the Bullet 3.24 files named above (as patched in RocketSim) for a CUDA device and a host
// build, with its own data layout, naming and control flow; the original's notice follows.
//
// Bullet Continuous Collision Detection and Physics Library
// Copyright (c) 2003-2006 Erwin Coumans  https://bulletphysics.org
//
// This software is provided 'as-is', without any express or implied warranty.
// In no event will the authors be held liable for any damages arising from the use of this software.
// Permission is granted to anyone to use this software for any purpose,
// including commercial applications, and to alter it and redistribute it freely,
// subject to the following restrictions:
//
// 1. The origin of this software must not be misrepresented; you must not claim that you wrote the original software. If you use this software in a product, an acknowledgment in the product documentation would be appreciated but is not required.
// 2. Altered source versions must be plainly marked as such, and must not be misrepresented as being the original software.
// 3. This notice may not be removed or altered from any source distribution.
#pragma once
#include "arena_static.h"

namespace rsb {

struct RayHit {
    float fraction;   // closest hit fraction so far (btCollisionWorld::RayResultCallback)
    int obj;          // collision object id, -1 none
    V3 normal;        // m_hitNormalWorld
};

// btTriangleRaycastCallback::processTriangle (no flags); updates hit on a closer hit.
RSB_HD void rayTriangle(const V3* t, V3 from, V3 to, int obj, RayHit& hit, float& cbFraction) {
    V3 v10 = t[1] - t[0];
    V3 v20 = t[2] - t[0];
    V3 n = cross(v10, v20);
    float dist = dot(t[0], n);
    float da = dot(n, from) - dist;
    float db = dot(n, to) - dist;
    if (da * db >= 0.f) return;
    float proj = da - db;
    float distance = da / proj;
    if (distance < cbFraction) {
        float edgeTol = length2(n) * -0.0001f;
        V3 point = from * (1.f - distance) + to * distance;
        V3 v0p = t[0] - point, v1p = t[1] - point;
        if (dot(cross(v0p, v1p), n) >= edgeTol) {
            V3 v2p = t[2] - point;
            if (dot(cross(v1p, v2p), n) >= edgeTol) {
                if (dot(cross(v2p, v0p), n) >= edgeTol) {
                    n = normalized(n);
                    V3 rn = (da <= 0.f) ? -n : n;
                    hit.fraction = distance;
                    hit.obj = obj;
                    hit.normal = rn;
                    cbFraction = distance;
                }
            }
        }
    }
}

RSB_HD void rayVsMesh(const ArenaStatic& S, int mesh, V3 from, V3 to, RayHit& hit) {
    float cbf = hit.fraction;
    bvhQueryRay(S, mesh, from, to, [&](int tri) {
        V3 v[3];
        triVerts(S, mesh, tri, v);
        rayTriangle(v, from, to, mesh, hit, cbf);
        return true;
    });
}

// The closest hit over the meshes in `meshes` (bit m = mesh m), exactly as rayVsMesh called
// for those meshes in ascending order would report it, found from the voxel triangle lists
// instead of the BVH walks: the lists of the voxels around the segment hold every triangle
// the segment can touch, a triangle is tested only if its BVH leaf passes the two tests the
// walk applies to it (a leaf that passes them has ancestors that pass them), and the
// candidates are taken in (mesh, leaf) order, the order of the walks.  Returns false, with
// `hit` untouched, when the segment leaves the grid or has more candidates than fit.
constexpr int kRayCandidates = 48;

// The candidates (keys mesh << 22 | leaf << 10 | triangle) of the voxels around the segment,
// sorted and without duplicates; false when the segment leaves the grid or more than
// kRayCandidates candidates are found.
RSB_HD bool rayVoxGather(const ArenaStatic& S, uint32_t meshes, V3 src, V3 dst, float tol, uint32_t* cand, int& nc) {
    nc = 0;
    const V3 mn = vmin(src, dst) - V3{tol, tol, tol}, mx = vmax(src, dst) + V3{tol, tol, tol};
    const float f = S.occInvCell;
    const int x0 = (int)floorf((mn.x - S.occMin.x) * f), x1 = (int)floorf((mx.x - S.occMin.x) * f);
    const int y0 = (int)floorf((mn.y - S.occMin.y) * f), y1 = (int)floorf((mx.y - S.occMin.y) * f);
    const int z0 = (int)floorf((mn.z - S.occMin.z) * f), z1 = (int)floorf((mx.z - S.occMin.z) * f);
    if (!(x0 >= 0 && y0 >= 0 && z0 >= 0 && x1 < S.occX && y1 < S.occY && z1 < S.occZ)) return false;
    for (int x = x0; x <= x1; x++)
        for (int y = y0; y <= y1; y++)
            for (int z = z0; z <= z1; z++) {
                const int v = (x * S.occY + y) * S.occZ + z;
                for (uint32_t i = S.voxOff[v], e = S.voxOff[v + 1]; i < e; i++) {
                    const uint32_t key = S.voxList[i];
                    if (!((meshes >> (key >> 22)) & 1u)) continue;
                    // sorted insert without duplicates
                    int p = nc;
                    while (p > 0 && cand[p - 1] > key) p--;
                    if (p > 0 && cand[p - 1] == key) continue;
                    if (nc == kRayCandidates) return false;
                    for (int q = nc; q > p; q--) cand[q] = cand[q - 1];
                    cand[p] = key;
                    nc++;
                }
            }
    return true;
}

// The ray set-up of bvhQueryRay for one segment.
struct RaySetup {
    V3 src, dst, inv, rmn, rmx;
    unsigned sign[3];
    float lambdaMax;
};
RSB_HD RaySetup raySetup(V3 src, V3 dst) {
    RaySetup r;
    r.src = src;
    r.dst = dst;
    const V3 rayDir = safeNormalized(dst - src);
    r.lambdaMax = dot(rayDir, dst - src);
    r.inv.x = rayDir.x == 0.f ? kLargeFloat : 1.f / rayDir.x;
    r.inv.y = rayDir.y == 0.f ? kLargeFloat : 1.f / rayDir.y;
    r.inv.z = rayDir.z == 0.f ? kLargeFloat : 1.f / rayDir.z;
    r.sign[0] = r.inv.x < 0.f;
    r.sign[1] = r.inv.y < 0.f;
    r.sign[2] = r.inv.z < 0.f;
    r.rmn = vmin(src, dst);
    r.rmx = vmax(src, dst);
    return r;
}

// The voxel-list query, candidate after candidate (the reference's visiting order).
RSB_HD bool rayVsMeshesVoxSerial(const ArenaStatic& S, uint32_t meshes, V3 src, V3 dst, float tol, RayHit& hit,
                                 uint32_t* cand) {
    int nc;
    if (!rayVoxGather(S, meshes, src, dst, tol, cand, nc)) return false;
    const RaySetup R = raySetup(src, dst);
    int cur = -1;
    uint16_t qmn[3], qmx[3];
    float cbf = hit.fraction;
    for (int c = 0; c < nc; c++) {
        const int m = (int)(cand[c] >> 22), leaf = (int)((cand[c] >> 10) & 0xFFFu), tri = (int)(cand[c] & 0x3FFu);
        const MeshDesc& md = S.meshes[m];
        if (m != cur) {
            if (hit.fraction == 0.f) break;  // castRay tests no further object after an exact hit
            cur = m;
            bvhQuantizeClamp(md, R.rmn, 0, qmn);
            bvhQuantizeClamp(md, R.rmx, 1, qmx);
            cbf = hit.fraction;
        }
        const BvhNode& nd = S.nodes[md.nodeOff + leaf];
        if (!qOverlap(qmn, qmx, nd.qmin, nd.qmax)) continue;
        V3 bounds[2];
        bounds[0] = bvhUnquantize(md, nd.qmin);
        bounds[1] = bvhUnquantize(md, nd.qmax);
        float param = 1.f;
        if (!rayAabb2(src, R.inv, R.sign, bounds, param, 0.f, R.lambdaMax)) continue;
        V3 v[3];
        triVerts(S, m, tri, v);
        rayTriangle(v, src, dst, m, hit, cbf);
    }
    return true;
}

RSB_HD bool rayVsMeshesVox(const ArenaStatic& S, uint32_t meshes, V3 src, V3 dst, float tol, RayHit& hit) {
    uint32_t cand[kRayCandidates];
    return rayVsMeshesVoxSerial(S, meshes, src, dst, tol, hit, cand);
}

RSB_HD void rayVsPlane(const ArenaStatic& S, int plane, V3 fromW, V3 toW, RayHit& hit) {
    V3 origin = S.planeOrigin[plane - MAX_MESHES];
    V3 n = S.planeNormal[plane - MAX_MESHES];
    {
        // a segment that stays on one side of the plane, farther than any rounding of the
        // two triangles below from it, crosses neither of them
        const float tol = 1e-3f;
        const float sa = dot(n, fromW - origin), sb = dot(n, toW - origin);
        if ((sa > tol && sb > tol) || (sa < -tol && sb < -tol)) return;
    }
    // world -> plane-object transform (identity basis): translate by -origin
    Xf inv = xfInverse(Xf{m3identity(), origin});
    V3 from = xfPoint(inv, fromW), to = xfPoint(inv, toW);
    V3 amn = vmin(from, to), amx = vmax(from, to);
    V3 he = (amx - amn) * 0.5f;
    float radius = length(he);
    V3 center = (amx + amn) * 0.5f;
    V3 t0, t1;
    planeSpace1(n, t0, t1);
    V3 pc = center - n * (dot(n, center) - 0.f);
    V3 tri[3];
    float cbf = hit.fraction;
    tri[0] = (pc + t0 * radius) + t1 * radius;
    tri[1] = (pc + t0 * radius) - t1 * radius;
    tri[2] = (pc - t0 * radius) - t1 * radius;
    rayTriangle(tri, from, to, plane, hit, cbf);
    tri[0] = (pc - t0 * radius) - t1 * radius;
    tri[1] = (pc - t0 * radius) + t1 * radius;
    tri[2] = (pc + t0 * radius) + t1 * radius;
    rayTriangle(tri, from, to, plane, hit, cbf);
}

}  // namespace rsb
