// Wheel ray casts against the static arena (btCollisionWorld::rayTest through the RocketSim
// broadphase, btCollisionWorld.cpp:877-966, btRSBroadphase.cpp:325-356).
//
// The suspension-grid shortcut is compiled out of the reference build (RS_NO_SUSPCOLGRID,
// Framework.h:111), so every wheel ray is a full ray test against the objects registered
// in the broadphase cell of the ray start: arena meshes (btTriangleRaycastCallback over the
// BVH, btRaycastCallback.cpp:31-108), the static planes (two large triangles,
// btStaticPlaneShape::processAllTriangles), and dynamic bodies.
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
