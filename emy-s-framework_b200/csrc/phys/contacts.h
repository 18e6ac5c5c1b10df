// Contact generation shared by all narrowphase routines: manifold point insertion,
// RocketSim's contact-added callback rules and Bullet's internal-edge normal fix-up.
//
//   addContact ........... btManifoldResult::addContactPoint (btManifoldResult.cpp:107-200)
//                          with btPersistentManifold::getCacheEntry returning -1
//                          (btPersistentManifold.cpp:191-195: new points never merge)
//   sortCachedPoints ..... btPersistentManifold::sortCachedPoints (.cpp:90-160)
//   refreshContactPoints . btPersistentManifold::refreshContactPoints (.cpp:262-320)
//   adjustInternalEdge ... btAdjustInternalEdgeContacts (btInternalEdgeUtility.cpp:420-798)
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
#include "world_types.h"

namespace rsb {

struct World;  // forward

// Transform and material of an object id (statics are at fixed transforms).
struct ObjRef {
    Xf xf;
    float friction, restitution;
    bool isStatic;
};

RSB_HD void mpInit(MPoint& p) {
    p.localA = p.localB = p.posA = p.posB = p.normal = v3zero();
    p.dist = p.fric = p.rest = 0.f;
    p.index1 = -1;
    p.special = 0;
}

// closestAxis4 of (res0..res3): index of the first largest absolute value
RSB_HD int closestAxis4(float a, float b, float c, float d) {
    float v[4] = {fabsf(a), fabsf(b), fabsf(c), fabsf(d)};
    int idx = -1;
    float mx = -kLargeFloat;
    for (int i = 0; i < 4; i++)
        if (v[i] > mx) { idx = i; mx = v[i]; }
    return idx;
}

RSB_HD int sortCachedPoints(const Manifold& m, const MPoint& pt) {
    int maxPenIdx = -1;
    float maxPen = pt.dist;
    for (int i = 0; i < 4; i++)
        if (m.pt[i].dist < maxPen) { maxPenIdx = i; maxPen = m.pt[i].dist; }
    float r0 = 0.f, r1 = 0.f, r2 = 0.f, r3 = 0.f;
    if (maxPenIdx != 0) r0 = length2(cross(pt.localA - m.pt[1].localA, m.pt[3].localA - m.pt[2].localA));
    if (maxPenIdx != 1) r1 = length2(cross(pt.localA - m.pt[0].localA, m.pt[3].localA - m.pt[2].localA));
    if (maxPenIdx != 2) r2 = length2(cross(pt.localA - m.pt[0].localA, m.pt[3].localA - m.pt[1].localA));
    if (maxPenIdx != 3) r3 = length2(cross(pt.localA - m.pt[0].localA, m.pt[2].localA - m.pt[1].localA));
    return closestAxis4(r0, r1, r2, r3);
}

// Inserts a contact into manifold m.  res0/res1 are the btManifoldResult's bodies (the
// pair order); the manifold's own body order decides the swap, as in the reference.
// Returns the point slot, or -1 when the point is beyond the breaking threshold.
RSB_HD int addContact(Manifold& m, BlockPool& pool, int res0, const ObjRef& r0, int res1, const ObjRef& r1,
                      V3 normalOnB, V3 pointInWorld, float depth) {
    if (depth > m.cbt) return -1;
    if (!m.pt) {
        if (pool.n >= MAX_BLOCKS) {
            *pool.status |= 2u;  // row/contact pool overflow: contact dropped
            return -1;
        }
        m.pt = pool.pts + MAX_POINTS * pool.n++;
    }
    bool swapped = m.o0 != res0;
    V3 pointA = pointInWorld + normalOnB * depth;
    MPoint np;
    mpInit(np);
    if (swapped) {
        np.localA = xfInvPoint(r1.xf, pointA);
        np.localB = xfInvPoint(r0.xf, pointInWorld);
    } else {
        np.localA = xfInvPoint(r0.xf, pointA);
        np.localB = xfInvPoint(r1.xf, pointInWorld);
    }
    np.normal = normalOnB;
    np.dist = depth;
    np.posA = pointA;
    np.posB = pointInWorld;
    // gCalculateCombinedFriction / Restitution (btManifoldResult.cpp:58-80)
    if (r0.isStatic || r1.isStatic) {
        np.fric = r0.friction < r1.friction ? r0.friction : r1.friction;
        np.rest = r0.restitution > r1.restitution ? r0.restitution : r1.restitution;
    } else {
        np.fric = r0.friction * r1.friction;
        np.rest = r0.restitution * r1.restitution;
    }
    int idx;
    if (m.n == MAX_POINTS) {
        idx = sortCachedPoints(m, np);
        if (idx < 0) idx = 0;
    } else {
        idx = m.n++;
    }
    m.pt[idx] = np;
    return idx;
}

RSB_HD void removeContactPoint(Manifold& m, int i) {
    int last = m.n - 1;
    if (i != last) m.pt[i] = m.pt[last];
    m.n--;
}

RSB_HD void refreshContactPoints(Manifold& m, const Xf& trA, const Xf& trB) {
    for (int i = m.n - 1; i >= 0; i--) {
        MPoint& p = m.pt[i];
        p.posA = xfPoint(trA, p.localA);
        p.posB = xfPoint(trB, p.localB);
        p.dist = dot(p.posA - p.posB, p.normal);
    }
    for (int i = m.n - 1; i >= 0; i--) {
        MPoint& p = m.pt[i];
        if (!(p.dist <= m.cbt)) {
            removeContactPoint(m, i);
        } else {
            V3 proj = p.posA - p.normal * p.dist;
            V3 diff = p.posB - proj;
            float d2 = dot(diff, diff);
            if (d2 > m.cbt * m.cbt) removeContactPoint(m, i);
        }
    }
}

// ---------------------------------------------------------------- internal edges

RSB_HD void nearestPointInLineSegment(V3 point, V3 l0, V3 l1, V3& nearest) {
    V3 d = l1 - l0;
    if (fuzzyZero(d)) {
        nearest = l0;
    } else {
        float delta = dot(point - l0, d) / dot(d, d);
        if (delta < 0) delta = 0;
        else if (delta > 1) delta = 1;
        nearest = l0 + d * delta;
    }
}

RSB_HD float edgeAngle(V3 edgeA, V3 normalA, V3 normalB) {
    return rsAtan2f(dot(normalB, edgeA), dot(normalB, normalA));
}

RSB_HD bool clampNormal(V3 edge, V3 triNormalOrg, V3 localNormal, float corrected, V3& clamped) {
    V3 triNormal = triNormalOrg;
    V3 edgeCross = normalized(cross(edge, triNormal));
    float cur = edgeAngle(edgeCross, triNormal, localNormal);
    if (corrected < 0) {
        if (cur < corrected) {
            float diff = corrected - cur;
            clamped = m3fromQuat(qaxisAngle(edge, diff)) * localNormal;
            return true;
        }
    }
    if (corrected >= 0) {
        if (cur > corrected) {
            float diff = corrected - cur;
            clamped = m3fromQuat(qaxisAngle(edge, diff)) * localNormal;
            return true;
        }
    }
    return false;
}

// The mesh's collision object is at the identity transform, so mesh-local and world
// coordinates coincide (the reference's basis products with the identity are exact).
RSB_HD void adjustInternalEdge(MPoint& cp, const V3* v, const TriEdgeInfo& info) {
    if (!(info.flags & TRI_INFO_PRESENT)) return;
    const float kMaxEdgeAngle = kTwoPi, kConvexEps = 0.f, kEdgeDist = 0.1f;
    const float frontFacing = 1.f;  // normalAdjustFlags == 0
    V3 v0 = v[0], v1 = v[1], v2 = v[2];
    V3 triNormal = normalized(cross(v1 - v0, v2 - v0));
    V3 nearest;
    nearestPointInLineSegment(cp.localB, v0, v1, nearest);
    V3 contact = cp.localB;
    bool isNearEdge = false;
    int numConcave = 0;
    V3 localNormal = normalized(cp.normal);
    int best = -1;
    float bestDist = kLargeFloat;
    if (fabsf(info.a01) < kMaxEdgeAngle) {
        V3 nr;
        nearestPointInLineSegment(cp.localB, v0, v1, nr);
        float len = length(contact - nr);
        if (len < bestDist) { best = 0; bestDist = len; }
    }
    if (fabsf(info.a12) < kMaxEdgeAngle) {
        V3 nr;
        nearestPointInLineSegment(cp.localB, v1, v2, nr);
        float len = length(contact - nr);
        if (len < bestDist) { best = 1; bestDist = len; }
    }
    if (fabsf(info.a20) < kMaxEdgeAngle) {
        V3 nr;
        nearestPointInLineSegment(cp.localB, v2, v0, nr);
        float len = length(contact - nr);
        if (len < bestDist) { best = 2; bestDist = len; }
    }
    // edge v0-v1 (uses the outer `localNormal`, normalised)
    if (fabsf(info.a01) < kMaxEdgeAngle) {
        float len = length(contact - nearest);
        if (len < kEdgeDist && best == 0) {
            V3 edge = v0 - v1;
            isNearEdge = true;
            if (info.a01 == 0.f) {
                numConcave++;
            } else {
                bool isConvex = (info.flags & TRI_INFO_V0V1_CONVEX) != 0;
                float swapFactor = isConvex ? 1.f : -1.f;
                V3 nA = triNormal * swapFactor;
                V3 cnB = quatRotate(qaxisAngle(edge, info.a01), triNormal);
                if (info.flags & TRI_INFO_V0V1_SWAP_NORMALB) cnB *= -1.f;
                V3 nB = cnB * swapFactor;
                float ndA = dot(localNormal, nA), ndB = dot(localNormal, nB);
                bool back = (ndA < kConvexEps) && (ndB < kConvexEps);
                if (back) {
                    numConcave++;
                } else {
                    V3 clamped;
                    if (clampNormal(edge, triNormal * swapFactor, localNormal, info.a01, clamped)) {
                        if (dot(clamped, triNormal * frontFacing) > 0) {
                            cp.normal = clamped;
                            cp.posB = cp.posA - cp.normal * cp.dist;
                            cp.localB = cp.posB;
                        }
                    }
                }
            }
        }
    }
    nearestPointInLineSegment(contact, v1, v2, nearest);
    if (fabsf(info.a12) < kMaxEdgeAngle) {
        float len = length(contact - nearest);
        if (len < kEdgeDist && best == 1) {
            isNearEdge = true;
            V3 edge = v1 - v2;
            if (info.a12 == 0.f) {
                numConcave++;
            } else {
                bool isConvex = (info.flags & TRI_INFO_V1V2_CONVEX) != 0;
                float swapFactor = isConvex ? 1.f : -1.f;
                V3 nA = triNormal * swapFactor;
                V3 cnB = quatRotate(qaxisAngle(edge, info.a12), triNormal);
                if (info.flags & TRI_INFO_V1V2_SWAP_NORMALB) cnB *= -1.f;
                V3 nB = cnB * swapFactor;
                float ndA = dot(localNormal, nA), ndB = dot(localNormal, nB);
                bool back = (ndA < kConvexEps) && (ndB < kConvexEps);
                if (back) {
                    numConcave++;
                } else {
                    V3 ln = cp.normal;  // recomputed without normalisation, as the reference does
                    V3 clamped;
                    if (clampNormal(edge, triNormal * swapFactor, ln, info.a12, clamped)) {
                        if (dot(clamped, triNormal * frontFacing) > 0) {
                            cp.normal = clamped;
                            cp.posB = cp.posA - cp.normal * cp.dist;
                            cp.localB = cp.posB;
                        }
                    }
                }
            }
        }
    }
    nearestPointInLineSegment(contact, v2, v0, nearest);
    if (fabsf(info.a20) < kMaxEdgeAngle) {
        float len = length(contact - nearest);
        if (len < kEdgeDist && best == 2) {
            isNearEdge = true;
            V3 edge = v2 - v0;
            if (info.a20 == 0.f) {
                numConcave++;
            } else {
                bool isConvex = (info.flags & TRI_INFO_V2V0_CONVEX) != 0;
                float swapFactor = isConvex ? 1.f : -1.f;
                V3 nA = triNormal * swapFactor;
                V3 cnB = quatRotate(qaxisAngle(edge, info.a20), triNormal);
                if (info.flags & TRI_INFO_V2V0_SWAP_NORMALB) cnB *= -1.f;
                V3 nB = cnB * swapFactor;
                float ndA = dot(localNormal, nA), ndB = dot(localNormal, nB);
                bool back = (ndA < kConvexEps) && (ndB < kConvexEps);
                if (back) {
                    numConcave++;
                } else {
                    V3 ln = cp.normal;
                    V3 clamped;
                    if (clampNormal(edge, triNormal * swapFactor, ln, info.a20, clamped)) {
                        if (dot(clamped, triNormal * frontFacing) > 0) {
                            cp.normal = clamped;
                            cp.posB = cp.posA - cp.normal * cp.dist;
                            cp.localB = cp.posB;
                        }
                    }
                }
            }
        }
    }
    if (isNearEdge && numConcave > 0) {
        V3 newNormal = triNormal * frontFacing;
        float d = dot(newNormal, localNormal);
        if (d < 0) return;
        cp.normal = newNormal;
        cp.posB = cp.posA - cp.normal * cp.dist;
        cp.localB = cp.posB;
    }
}

}  // namespace rsb
