// One physics tick of one arena: broadphase, narrowphase, islands, solve, integrate.
//
// Restates btDiscreteDynamicsWorld::stepSimulation / internalSingleStepSimulation
// (btDiscreteDynamicsWorld.cpp:320-437) as RocketSim drives it, including
//   - btRSBroadphase pair generation (btRSBroadphase.cpp:377-460): every pair is removed
//     and re-added each tick, so collision algorithms and manifolds are fresh per tick
//     and manifolds are created in pair order;
//   - btCollisionDispatcher::defaultNearCallback / needsCollision (btCollisionDispatcher.cpp:130-300);
//   - btSimulationIslandManager with STATIC_SIMULATION_ISLAND_OPTIMIZATION and
//     USE_PATH_COMPRESSION (btSimulationIslandManager.cpp, btUnionFind.h), including
//     the unstable quickSort of btAlignedObjectArray that fixes manifold order;
//   - integrateTransforms / updateActivationState.
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
#include "contacts.h"
#include "solver.h"
#include "ray.h"
#include "gjk.h"
#include "boxbox.h"

namespace rsb {

// Dynamic bodies in ascending (registration stamp, body index) order with their
// broadphase cells.  btRSBroadphase visits the proxies of a cell in registration order;
// registrations change only in updateBodyAabb, so the order is rebuilt after it (for the
// pair search) and before the car pre-ticks (for the wheel rays), which lets both walk it
// once instead of searching for the next stamp body by body.
struct RegOrder {
    int n;
    int8_t body[MAX_BODIES];
    uint32_t stamp[MAX_BODIES];
    int16_t ci[MAX_BODIES], cj[MAX_BODIES], ck[MAX_BODIES];
};

struct World {
    const ArenaStatic* S;
    const WorldParams* P;
    int nb;                 // bodies: 0 = ball, 1.. = cars
    Body b[MAX_BODIES];
    int noRot[MAX_BODIES];
    uint32_t stampBase;     // registration stamps of this tick
    int np;
    int16_t po0[MAX_PAIRS], po1[MAX_PAIRS];
    int nm;
    Manifold m[MAX_MANIFOLDS];
    BlockPool pool;
    uint32_t status;
    // cars
    int nc;
    CarSim c[MAX_CARS];
    uint64_t tick;          // Arena::tickCount at the start of this tick
    V3 ballVelCache;        // Ball::_velocityImpulseCache
    EpaWork* epa;           // EPA scratch (faces and support vertices)
    // learned culling: bit b set = body b (0 ball, 1 + s car s) is clear of every static
    // shape for this launch, so its static tests (wheel rays against meshes and planes,
    // mesh / plane narrowphase) cannot find anything and are skipped; with cullAudit they
    // run anyway and whatever they find is counted as a miss
    uint32_t cull;
    int32_t cullAudit;
    mutable uint32_t nStatic, nCulled, nMissed;  // static tests run / skipped / skipped but hit
    mutable uint32_t cullMissed;                 // WS_CULL_MISS once a skipped test would have hit
    mutable uint32_t nRows;                      // solver rows (contact + friction) set up this launch
    RegOrder reg;
};

// world status bits (per-arena status word)
enum : uint32_t { WS_NONFINITE = 1u, WS_OVERFLOW = 2u, WS_CULL_MISS = 8u, WS_EPA_OVERFLOW = 16u };  // 4 is reserved (rsb.h)

// Index of the lowest set bit of a non-zero mask.
RSB_HD int lowestBit(uint32_t m) {
#if defined(__CUDA_ARCH__)
    return __ffs((int)m) - 1;
#else
    return __builtin_ctz(m);
#endif
}

// Number of set bits.
RSB_HD int bitCount(uint32_t m) {
#if defined(__CUDA_ARCH__)
    return __popc(m);
#else
    return __builtin_popcount(m);
#endif
}

// Tolerance of the exact occupancy reject around a mesh query box or ray segment (Bullet
// units).  A ray's convex cast against the ball or a car has no such reject: Bullet's
// subsimplex cast reports a hit when it runs out of iterations, which can lie well outside
// the shape's box (0.23 BT in one 3v3 rollout), and the reference keeps that hit.
constexpr float kOccTol = 2.f * kUuToBt;

// Bookkeeping of one static test of body b: returns true when the test must be skipped.
// (nCulled counts the tests the bound clears, also in audit mode where they still run.)
RSB_HD bool cullSkip(const World& W, int b) {
    if ((W.cull >> b) & 1u) {
        W.nCulled++;
        if (!W.cullAudit) return true;
    }
    W.nStatic++;
    return false;
}
RSB_HD void cullCheck(const World& W, int b, bool found) {
    if (found && ((W.cull >> b) & 1u)) {
        W.nMissed++;
        W.cullMissed = WS_CULL_MISS;
    }
}

// ------------------------------------------------------------------ objects

RSB_HD bool objIsStatic(int o) { return o < OBJ_BALL; }
RSB_HD bool objIsPlane(int o) { return o >= MAX_MESHES && o < NUM_STATICS; }

RSB_HD ObjRef objRef(const World& W, int o) {
    ObjRef r;
    if (o < MAX_MESHES) {
        r.xf = xfIdentity();
        r.friction = STATIC_FRICTION;
        r.restitution = STATIC_RESTITUTION;
        r.isStatic = true;
    } else if (o < NUM_STATICS) {
        r.xf = Xf{m3identity(), W.S->planeOrigin[o - MAX_MESHES]};
        r.friction = STATIC_FRICTION;
        r.restitution = STATIC_RESTITUTION;
        r.isStatic = true;
    } else {
        const Body& b = W.b[o - OBJ_BALL];
        r.xf = b.xf;
        r.friction = b.friction;
        r.restitution = b.restitution;
        r.isStatic = false;
    }
    return r;
}

RSB_HD bool objActive(const World& W, int o) {
    if (objIsStatic(o)) return false;  // static objects are ISLAND_SLEEPING
    int a = W.b[o - OBJ_BALL].act;
    return a != ACT_SLEEPING && a != ACT_DISABLE_SIM;
}

// ------------------------------------------------------------------ AABBs / broadphase

RSB_HD void ballAabb(const WorldParams& P, const Xf& xf, V3& mn, V3& mx) {
    V3 e{P.ballAabbExt, P.ballAabbExt, P.ballAabbExt};
    mn = xf.o - e;
    mx = xf.o + e;
}

// Car hitbox: a btCompoundShape holding one btBoxShape at the hitbox offset
RSB_HD Xf carChildXf(const CarParams& C, const Xf& carXf) { return xfMul(carXf, Xf{m3identity(), C.childOff}); }
// btCompoundShape::getAabb
RSB_HD void carCompoundAabb(const CarParams& C, const Xf& xf, V3& mn, V3& mx) { transformAabb(C.cmpMin, C.cmpMax, 0.f, xf, mn, mx); }
// btBoxShape::getAabb of the child at its world transform
RSB_HD void carBoxAabb(const CarParams& C, const Xf& childXf, V3& mn, V3& mx) {
    transformAabbHalf(C.boxHe, C.boxMargin, childXf, mn, mx);
}
RSB_HD ConvexShape carBoxShape(const CarParams& C) { return makeBox(C.boxHe, C.boxMargin); }

RSB_HD void bodyShapeAabb(const World& W, int bi, const Xf& xf, V3& mn, V3& mx) {
    if (bi == 0) ballAabb(*W.P, xf, mn, mx);
    else carCompoundAabb(W.P->car, xf, mn, mx);
}

RSB_HD void bpCellIndices(const BpGrid& g, V3 pos, int& i, int& j, int& k) {
    V3 f = bdiv(pos - g.minPos, g.cellSize);
    auto toInt = [](float x) -> int {
        if (!(x > -2147483648.f && x < 2147483648.f)) return (int)0x80000000;
        return (int)x;
    };
    i = imin_(imax_(toInt(f.x), 0), g.cellsX - 1);
    j = imin_(imax_(toInt(f.y), 0), g.cellsY - 1);
    k = imin_(imax_(toInt(f.z), 0), g.cellsZ - 1);
}

// btCollisionWorld::updateSingleAabb + btRSBroadphase::setAabb (dynamic proxies)
RSB_HD void updateBodyAabb(World& W, int bi) {
    Body& b = W.b[bi];
    V3 mn, mx, mn2, mx2;
    bodyShapeAabb(W, bi, b.xf, mn, mx);
    V3 thr{0.02f, 0.02f, 0.02f};
    mn = mn - thr;
    mx = mx + thr;
    bodyShapeAabb(W, bi, b.ixf, mn2, mx2);
    mn2 = mn2 - thr;
    mx2 = mx2 + thr;
    mn = vmin(mn, mn2);
    mx = vmax(mx, mx2);
    if (!(length2(mx - mn) < 1e12f)) {
        b.act = ACT_DISABLE_SIM;
        W.status |= 1u;
        return;
    }
    b.bpMin = mn;
    b.bpMax = mx;
    const BpGrid& g = W.S->bp;
    int i, j, k;
    bpCellIndices(g, mn, i, j, k);
    int cell = i * g.cellsY * g.cellsZ + j * g.cellsZ + k;
    if (cell != b.cell) {
        b.cell = cell;
        if (W.nb > 1) {  // numDynProxies > 1
            b.ci = i;
            b.cj = j;
            b.ck = k;
            b.regStamp = W.stampBase + (uint32_t)bi;
        }
    }
}

RSB_HD bool findPair(const World& W, int a, int b) {
    for (int p = 0; p < W.np; p++)
        if (W.po0[p] == a && W.po1[p] == b) return true;
    return false;
}

RSB_HD void addPair(World& W, int a, int b) {
    int lo = a < b ? a : b, hi = a < b ? b : a;
    if (findPair(W, lo, hi)) return;
    if (W.np >= MAX_PAIRS) { W.status |= 2u; return; }
    W.po0[W.np] = (int16_t)lo;
    W.po1[W.np] = (int16_t)hi;
    W.np++;
}

RSB_HD bool inRegNeighbourhood(const Body& b, int ci, int cj, int ck) {
    return ci >= b.ci - 1 && ci <= b.ci + 1 && cj >= b.cj - 1 && cj <= b.cj + 1 && ck >= b.ck - 1 && ck <= b.ck + 1;
}

RSB_HD void buildRegOrder(World& W) {
    RegOrder& R = W.reg;
    R.n = 0;
    for (int e = 0; e < W.nb; e++) {
        const Body& b = W.b[e];
        // insertion keeps equal stamps in body-index order
        int r = R.n++;
        while (r > 0 && R.stamp[r - 1] > b.regStamp) {
            R.body[r] = R.body[r - 1];
            R.stamp[r] = R.stamp[r - 1];
            R.ci[r] = R.ci[r - 1];
            R.cj[r] = R.cj[r - 1];
            R.ck[r] = R.ck[r - 1];
            r--;
        }
        R.body[r] = (int8_t)e;
        R.stamp[r] = b.regStamp;
        R.ci[r] = (int16_t)b.ci;
        R.cj[r] = (int16_t)b.cj;
        R.ck[r] = (int16_t)b.ck;
    }
}

RSB_HD bool regNear(const RegOrder& R, int r, int ci, int cj, int ck) {
    return ci >= R.ci[r] - 1 && ci <= R.ci[r] + 1 && cj >= R.cj[r] - 1 && cj <= R.cj[r] + 1 && ck >= R.ck[r] - 1 &&
           ck <= R.ck[r] + 1;
}

// btRSBroadphase::calculateOverlappingPairs
RSB_HD void computePairs(World& W) {
    W.np = 0;
    buildRegOrder(W);
    const ArenaStatic& S = *W.S;
    const BpGrid& g = S.bp;
    for (int bi = 0; bi < W.nb; bi++) {
        const Body& b = W.b[bi];
        int obj = OBJ_BALL + bi;
        uint32_t mask = S.bpCells[b.cell];
        for (int s = 0; s < NUM_STATICS; s++) {
            if (!(mask & (1u << s))) continue;
            V3 smn, smx;
            if (s < MAX_MESHES) { smn = S.meshes[s].bpMin; smx = S.meshes[s].bpMax; }
            else { smn = S.planeBpMin[s - MAX_MESHES]; smx = S.planeBpMax[s - MAX_MESHES]; }
            if (aabbOverlap(b.bpMin, b.bpMax, smn, smx)) addPair(W, s, obj);
        }
        if (W.nb > 1) {
            int ci = b.cell / (g.cellsY * g.cellsZ);
            int cj = (b.cell / g.cellsZ) % g.cellsY;
            int ck = b.cell % g.cellsZ;
            const RegOrder& R = W.reg;
            int inCell = 0;
            for (int r = 0; r < R.n; r++) inCell += regNear(R, r, ci, cj, ck) ? 1 : 0;
            if (inCell > 1) {
                // visit the other dynamic proxies of this cell in registration order (a
                // proxy whose stamp equals the one just visited is passed over)
                uint32_t last = 0;
                bool first = true;
                for (int r = 0; r < R.n; r++) {
                    if (!regNear(R, r, ci, cj, ck)) continue;
                    if (!first && R.stamp[r] <= last) continue;
                    first = false;
                    last = R.stamp[r];
                    const int pick = R.body[r];
                    if (pick == bi) continue;
                    if (aabbOverlap(b.bpMin, b.bpMax, W.b[pick].bpMin, W.b[pick].bpMax))
                        addPair(W, obj, OBJ_BALL + pick);
                }
            }
        }
    }
}

// ------------------------------------------------------------------ narrowphase: ball

// Sphere support point (btSphereShape::localGetSupportingVertex)
RSB_HD V3 sphereSupport(V3 vec, float margin) {
    V3 vn;
    if (length2(vec) < kEpsilon * kEpsilon) vn = normalized(V3{-1.f, -1.f, -1.f});
    else vn = normalized(vec);
    return vn * margin;
}

// SphereTriangleDetector::collide (SphereTriangleDetector.cpp:120-230, VirxEC variants)
RSB_HD bool pointInTriangleBary(const V3* v, V3 p) {
    V3 u = v[1] - v[0], w2 = v[2] - v[0];
    V3 n = cross(u, w2);
    float nLenSq = dot(n, n);
    V3 w = p - v[0];
    float gamma = dot(cross(u, w), n) / nLenSq;
    float beta = dot(cross(w, w2), n) / nLenSq;
    float alpha = 1 - gamma - beta;
    return (0 <= alpha) && (alpha <= 1) && (0 <= beta) && (beta <= 1) && (0 <= gamma) && (gamma <= 1);
}

RSB_HD V3 closestPointTriangle(V3 p, V3 a, V3 b, V3 c) {
    V3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) return a;
    V3 bp = p - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.f && d4 <= d3) return b;
    V3 cp = p - c;
    float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.f && d5 <= d6) return c;
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        float v = d1 / (d1 - d3);
        return a + ab * v;
    }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        float v = d2 / (d2 - d6);
        return a + ac * v;
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        float v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return b + (c - b) * v;
    }
    float denom = 1.f / (va + vb + vc);
    float v = vb * denom, w = vc * denom;
    return (a + ab * v) + ac * w;
}

RSB_HD bool sphereTriCollide(const V3* v, V3 center, float radius, float cbt, V3& point, V3& rnormal, float& depth) {
    float rwt = radius + cbt;
    V3 normal = cross(v[1] - v[0], v[2] - v[0]);
    float l2 = length2(normal);
    bool has = false;
    V3 contactPoint;
    if (l2 >= kEpsilon * kEpsilon) {
        normal = bdiv(normal, fsqrt(l2));
        V3 p1c = center - v[0];
        float dfp = dot(p1c, normal);
        if (dfp < 0.f) {
            dfp *= -1.f;
            normal *= -1.f;
        }
        if (dfp < rwt) {
            if (pointInTriangleBary(v, center)) {
                has = true;
                contactPoint = center - normal * dfp;
            } else {
                float minD2 = rwt * rwt;
                V3 ne = closestPointTriangle(center, v[0], v[1], v[2]);
                float d2 = length2(center - ne);
                if (d2 < minD2) {
                    has = true;
                    contactPoint = ne;
                }
            }
        }
    }
    if (has) {
        V3 c2c = center - contactPoint;
        float d2 = length2(c2c);
        if (d2 < rwt * rwt) {
            if (d2 > kEpsilon) {
                float d = fsqrt(d2);
                rnormal = normalized(c2c);
                point = contactPoint;
                depth = -(radius - d);
            } else {
                rnormal = normal;
                point = contactPoint;
                depth = -radius;
            }
            return true;
        }
    }
    return false;
}

// Ball vs one arena mesh: btConvexConcaveCollisionAlgorithm (swapped: the pair is
// (mesh, ball)) -> per triangle early-out + btSphereTriangleCollisionAlgorithm.
RSB_HD void collideBallMesh(World& W, int mesh, Manifold& man) {
    const WorldParams& P = *W.P;
    const Body& ball = W.b[0];
    ObjRef rMesh = objRef(W, mesh), rBall = objRef(W, OBJ_BALL);
    bool found = false;
    if (!cullSkip(W, 0)) {
    V3 amn, amx;
    ballAabb(P, ball.xf, amn, amx);  // convexInTriangleSpace == ball transform (mesh at identity)
    M3 invB = inverse(ball.xf.b);
    // no triangle of this mesh near the query box: the walk below could not report one
    if ((occMask(*W.S, amn - V3{kOccTol, kOccTol, kOccTol}, amx + V3{kOccTol, kOccTol, kOccTol}) >> mesh) & 1u)
    bvhQueryAabb(*W.S, mesh, amn, amx, [&](int tri) {
        V3 v[3];
        triVerts(*W.S, mesh, tri, v);
        if (!triAabbOverlap(v, amn, amx)) return true;
        // convex-concave early out (btConvexConcaveCollisionAlgorithm.cpp:100-137)
        V3 tn = normalized(cross(v[1] - v[0], v[2] - v[0]));
        float thr = man.cbt + 0.f;
        for (int side = 0; side < 2; side++) {
            V3 lp = sphereSupport(invB * tn, P.ballMargin);
            V3 wp = xfPoint(ball.xf, lp);
            float dist = dot(tn, v[0]) - dot(tn, wp);
            if (dist > thr) return true;
            tn *= -1.f;
        }
        V3 point, normal;
        float depth;
        if (sphereTriCollide(v, ball.xf.o, P.ballRadius, man.cbt, point, normal, depth)) {
            found = true;
            int idx = addContact(man, W.pool, mesh, rMesh, OBJ_BALL, rBall, normal, point, depth);
            if (idx >= 0) {
                MPoint& cp = man.pt[idx];
                cp.index1 = tri;
                cp.special = 1;  // ball + world (Arena.cpp:264-271)
                adjustInternalEdge(cp, v, W.S->triInfo[W.S->meshes[mesh].triOff + tri]);
            }
        }
        return true;
    });
    }
    cullCheck(W, 0, found);
    if (man.n) refreshContactPoints(man, rBall.xf, rMesh.xf);
}

// Ball vs static plane: btConvexPlaneCollisionAlgorithm (swapped pair (plane, ball))
RSB_HD void collideBallPlane(World& W, int plane, Manifold& man) {
    const WorldParams& P = *W.P;
    ObjRef rPlane = objRef(W, plane), rBall = objRef(W, OBJ_BALL);
    V3 pn = W.S->planeNormal[plane - MAX_MESHES];
    float pc = 0.f;
    Xf planeInConvex = xfMul(xfInverse(rBall.xf), rPlane.xf);
    Xf convexInPlane = xfMul(xfInverse(rPlane.xf), rBall.xf);
    if (!cullSkip(W, 0)) {
        V3 vtx = sphereSupport(planeInConvex.b * (-pn), P.ballMargin);
        V3 vip = xfPoint(convexInPlane, vtx);
        float distance = dot(pn, vip) - pc;
        if (distance < man.cbt + 0.f) {
            cullCheck(W, 0, true);
            V3 proj = vip - pn * distance;
            V3 world = xfPoint(rPlane.xf, proj);
            V3 nb = rPlane.xf.b * pn;
            int idx = addContact(man, W.pool, plane, rPlane, OBJ_BALL, rBall, nb, world, distance);
            if (idx >= 0) man.pt[idx].special = 1;
        }
    }
    if (man.n) refreshContactPoints(man, rBall.xf, rPlane.xf);
}

// ------------------------------------------------------------------ contact callbacks

RSB_HD bool carResponds(const World& W, int ci) { return !W.b[1 + ci].noResp; }

// Arena::_BtCallback_OnCarWorldCollision (Arena.cpp:420-427)
RSB_HD void onCarWorld(World& W, int ci, MPoint& cp) {
    CarSim& c = W.c[ci];
    c.flags |= CF_WORLD_CONTACT;
    c.worldContactNormal = cp.normal;
    cp.fric = W.P->car.worldFriction;
    cp.rest = W.P->car.worldRestitution;
}

// Arena::_BtCallback_OnCarBallCollision (Arena.cpp:278-332)
RSB_HD void onCarBall(World& W, int ci, MPoint& cp, bool ballIsBodyA) {
    const CarParams& C = W.P->car;
    CarSim& c = W.c[ci];
    const Body& cb = W.b[1 + ci];
    const Body& bb = W.b[0];
    V3 carPos = cb.xf.o * kBtToUu, carVel = cb.lin * kBtToUu;
    V3 ballPos = bb.xf.o * kBtToUu, ballVel = bb.lin * kBtToUu;
    cp.fric = CARBALL_COLLISION_FRICTION;
    cp.rest = CARBALL_COLLISION_RESTITUTION;
    c.flags |= CF_BALL_HIT_VALID;
    c.ballHitRelPos = (ballIsBodyA ? cp.localA : cp.localB) * kBtToUu;
    c.ballHitTick = W.tick;
    c.ballHitBallPos = ballPos;
    c.ballHitExtraVel = v3zero();
    if ((W.tick > c.ballHitExtraTick + 1) || (c.ballHitExtraTick > W.tick)) c.ballHitExtraTick = W.tick;
    else return;
    V3 carForward = c.rotMat.col(0);
    V3 relPos = ballPos - carPos;
    V3 relVel = ballVel - carVel;
    float relSpeed = fmin_(length(relVel), BALL_CAR_EXTRA_IMPULSE_MAXDELTAVEL_UU);
    if (relSpeed > 0) {
        V3 hitDir = safeNormalized(relPos * V3{1, 1, BALL_CAR_EXTRA_IMPULSE_Z_SCALE});
        V3 fwdAdj = (carForward * dot(hitDir, carForward)) * (1 - BALL_CAR_EXTRA_IMPULSE_FORWARD_SCALE);
        hitDir = safeNormalized(hitDir - fwdAdj);
        V3 addedVel = ((hitDir * relSpeed) * curveOut(crvBallCarExtra(), relSpeed)) * C.ballHitExtraScale;
        c.ballHitExtraVel = addedVel;
        W.ballVelCache = W.ballVelCache + addedVel * kUuToBt;
    }
}

// Arena::_BtCallback_OnCarCarCollision (Arena.cpp:334-418); car1 is the manifold's body 0
RSB_HD void onCarCar(World& W, int car1, int car2, MPoint& cp) {
    const CarParams& C = W.P->car;
    cp.fric = CARCAR_COLLISION_FRICTION;
    cp.rest = CARCAR_COLLISION_RESTITUTION;
    for (int i = 0; i < 2; i++) {
        bool isSwapped = (i == 1);
        if (isSwapped) { int t = car1; car1 = car2; car2 = t; }
        CarSim& s1 = W.c[car1];
        CarSim& s2 = W.c[car2];
        if ((s1.flags & CF_DEMOED) || (s2.flags & CF_DEMOED)) return;
        if ((s1.carContactOtherId == s2.id) && (s1.carContactCooldown > 0)) continue;
        V3 pos1 = W.b[1 + car1].xf.o * kBtToUu, vel1 = W.b[1 + car1].lin * kBtToUu;
        V3 pos2 = W.b[1 + car2].xf.o * kBtToUu, vel2 = W.b[1 + car2].lin * kBtToUu;
        V3 deltaPos = pos2 - pos1;
        if (dot(vel1, deltaPos) > 0) {
            V3 velDir = rsNormalized(vel1);
            V3 dirToOther = rsNormalized(deltaPos);
            float speedTowards = dot(vel1, dirToOther);
            float otherAway = dot(vel2, velDir);
            if (speedTowards > otherAway) {
                V3 localPoint = isSwapped ? cp.localB : cp.localA;
                bool hitWithBumper = (localPoint.x * kBtToUu) > BUMP_MIN_FORWARD_DIST;
                if (hitWithBumper) {
                    bool isDemo;
                    if (C.demoMode == 1) isDemo = true;
                    else if (C.demoMode == 2) isDemo = false;
                    else isDemo = (s1.flags & CF_SUPERSONIC) != 0;
                    if (isDemo && !C.teamDemos) isDemo = s1.team != s2.team;
                    if (isDemo) {
                        s2.flags |= CF_DEMOED;
                        s2.demoRespawnTimer = C.respawnDelay;
                    } else {
                        bool groundHit = (s2.flags & CF_ON_GROUND) != 0;
                        float baseScale = curveOut(groundHit ? crvBumpGround() : crvBumpAir(), speedTowards);
                        V3 hitUpDir = groundHit ? s2.rotMat.col(2) : V3{0, 0, 1};
                        V3 bump = velDir * baseScale + (hitUpDir * curveOut(crvBumpUp(), speedTowards)) * C.bumpForceScale;
                        s2.velCache = s2.velCache + bump * kUuToBt;
                    }
                    s1.carContactOtherId = s2.id;
                    s1.carContactCooldown = C.bumpCooldown;
                }
            }
        }
    }
}

// ------------------------------------------------------------------ narrowphase: cars

// Manifold bookkeeping of btCollisionDispatcher: getNewManifold appends, releaseManifold
// swaps the released manifold with the last one (btCollisionDispatcher.cpp:70-130).
RSB_HD int newManifold(World& W, int o0, int o1, float cbt) {
    if (W.nm >= MAX_MANIFOLDS) {
        W.status |= WS_OVERFLOW;
        return -1;
    }
    Manifold& m = W.m[W.nm];
    m.o0 = o0;
    m.o1 = o1;
    m.cbt = cbt;
    m.n = 0;
    m.pt = nullptr;
    return W.nm++;
}
RSB_HD void releaseManifold(World& W, int idx) {
    if (idx < 0) return;
    int last = W.nm - 1;
    if (idx != last) W.m[idx] = W.m[last];
    W.nm--;
}

RSB_HD float sq(float x) { return x * x; }

// True when some separating axis (the triangle normal, the box axes, or a box axis crossed
// with a triangle edge) puts the triangle more than `limit` away from the box of implicit
// half extents `he` at `x`.  The gap along an axis bounds the distance between the two
// from below, so GJK could not report a contact for such a triangle.
RSB_HD bool boxTriFar(const Xf& x, V3 he, const V3* v, float limit) {
    const V3 a0 = x.b.col(0), a1 = x.b.col(1), a2 = x.b.col(2);
    const V3 p0 = v[0] - x.o, p1 = v[1] - x.o, p2 = v[2] - x.o;
    auto sep = [&](V3 L) -> bool {
        const float l2 = dot(L, L);
        if (l2 < 1e-12f) return false;
        const float r = fabsf(dot(a0, L)) * he.x + fabsf(dot(a1, L)) * he.y + fabsf(dot(a2, L)) * he.z;
        const float t0 = dot(p0, L), t1 = dot(p1, L), t2 = dot(p2, L);
        const float gap = fmaxf(fmin_(t0, fmin_(t1, t2)) - r, -r - fmax_(t0, fmax_(t1, t2)));
        return gap > limit * sqrtf(l2);
    };
    const V3 e0 = p1 - p0, e1 = p2 - p1, e2 = p0 - p2;
    if (sep(cross(e0, e1)) || sep(a0) || sep(a1) || sep(a2)) return true;
    const V3 ax[3] = {a0, a1, a2}, ed[3] = {e0, e1, e2};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (sep(cross(ax[i], ed[j]))) return true;
    return false;
}

// Car box vs one arena mesh: the compound's child algorithm is btConvexConcaveCollisionAlgorithm
// (btConvexConcaveCollisionAlgorithm.cpp:60-250), each overlapping triangle through
// btConvexConvexAlgorithm's GJK (btConvexConvexAlgorithm.cpp:268-590).
RSB_HD void collideBoxMesh(World& W, int mesh, int ci, const Xf& childXf, Manifold& man) {
    const CarParams& C = W.P->car;
    int carObj = OBJ_CAR0 + ci;
    ObjRef rMesh = objRef(W, mesh), rCar = objRef(W, carObj);
    ConvexShape box = carBoxShape(C);
    V3 amn, amx;
    carBoxAabb(C, childXf, amn, amx);
    M3 invB = inverse(childXf.b);
    float maxDist2 = sq((C.boxMargin + 0.f) + man.cbt);
    bool responds = carResponds(W, ci);
    bool found = false;
    if (!cullSkip(W, 1 + ci) &&
        ((occMask(*W.S, amn - V3{kOccTol, kOccTol, kOccTol}, amx + V3{kOccTol, kOccTol, kOccTol}) >> mesh) & 1u)) {
    bvhQueryAabb(*W.S, mesh, amn, amx, [&](int tri) {
        V3 v[3];
        triVerts(*W.S, mesh, tri, v);
        if (!triAabbOverlap(v, amn, amx)) return true;
        V3 tn = normalized(cross(v[1] - v[0], v[2] - v[0]));
        for (int side = 0; side < 2; side++) {
            V3 lp = supportVirtual(box, invB * tn);
            V3 wp = xfPoint(childXf, lp);
            float dist = dot(tn, v[0]) - dot(tn, wp);
            if (dist > man.cbt + 0.f) return true;
            tn *= -1.f;
        }
        // separated well beyond the contact distance: GJK would find no contact
        if (boxTriFar(childXf, box.he, v, (C.boxMargin + 0.f) + man.cbt + 0.02f)) return true;
        ConvexShape triS = makeTri(v, 0.f);
        GjkOut g = gjkPairDetector(W.epa, box, childXf, triS, xfIdentity(), maxDist2);
        if (g.overflow) W.status |= WS_EPA_OVERFLOW;
        if (g.has) {
            found = true;
            int idx = addContact(man, W.pool, mesh, rMesh, carObj, rCar, g.normal, g.point, g.dist);
            if (idx >= 0 && responds) {
                MPoint& cp = man.pt[idx];
                cp.index1 = tri;
                onCarWorld(W, ci, cp);
                adjustInternalEdge(cp, v, W.S->triInfo[W.S->meshes[mesh].triOff + tri]);
            }
        }
        return true;
    });
    }
    cullCheck(W, 1 + ci, found);
    if (man.n) refreshContactPoints(man, rCar.xf, rMesh.xf);
}

// Car box vs a static plane: btConvexPlaneCollisionAlgorithm owning its manifold
RSB_HD void collideBoxPlane(World& W, int plane, int ci, const Xf& childXf, Manifold& man) {
    const CarParams& C = W.P->car;
    int carObj = OBJ_CAR0 + ci;
    ObjRef rPlane = objRef(W, plane), rCar = objRef(W, carObj);
    ConvexShape box = carBoxShape(C);
    V3 pn = W.S->planeNormal[plane - MAX_MESHES];
    Xf planeInConvex = xfMul(xfInverse(childXf), rPlane.xf);
    Xf convexInPlane = xfMul(xfInverse(rPlane.xf), childXf);
    if (!cullSkip(W, 1 + ci)) {
        V3 vtx = supportVirtual(box, planeInConvex.b * (-pn));
        V3 vip = xfPoint(convexInPlane, vtx);
        float distance = dot(pn, vip) - 0.f;
        if (distance < man.cbt + 0.f) {
            cullCheck(W, 1 + ci, true);
            V3 proj = vip - pn * distance;
            V3 world = xfPoint(rPlane.xf, proj);
            V3 nb = rPlane.xf.b * pn;
            int idx = addContact(man, W.pool, plane, rPlane, carObj, rCar, nb, world, distance);
            if (idx >= 0 && carResponds(W, ci)) onCarWorld(W, ci, man.pt[idx]);
        }
    }
    if (man.n) refreshContactPoints(man, rCar.xf, rPlane.xf);
}

// (static, car) pair: swapped btCompoundCollisionAlgorithm (btCompoundCollisionAlgorithm.cpp:120-330).
// The child algorithm is built with the pair's algorithm, so its manifold exists before
// processing; it is destroyed again when the child's AABB misses the static shape's AABB.
RSB_HD void collideCarStatic(World& W, int s, int ci) {
    const CarParams& C = W.P->car;
    int mi = newManifold(W, OBJ_CAR0 + ci, s, C.cbt);
    if (mi < 0) return;
    Xf childXf = carChildXf(C, W.b[1 + ci].xf);
    V3 bmn, bmx, omn, omx;
    carBoxAabb(C, childXf, bmn, bmx);
    if (s < MAX_MESHES) { omn = W.S->meshes[s].shapeMin; omx = W.S->meshes[s].shapeMax; }
    else { omn = W.S->planeShapeMin[s - MAX_MESHES]; omx = W.S->planeShapeMax[s - MAX_MESHES]; }
    bool overlap = aabbOverlap(bmn, bmx, omn, omx);
    if (overlap) {
        if (s < MAX_MESHES) collideBoxMesh(W, s, ci, childXf, W.m[mi]);
        else collideBoxPlane(W, s, ci, childXf, W.m[mi]);
    } else {
        releaseManifold(W, mi);
    }
}

// (ball, car) pair: swapped compound over a btConvexConvexAlgorithm that creates its
// manifold on first use
RSB_HD void collideCarBall(World& W, int ci) {
    const WorldParams& P = *W.P;
    const CarParams& C = P.car;
    int carObj = OBJ_CAR0 + ci;
    Xf childXf = carChildXf(C, W.b[1 + ci].xf);
    V3 bmn, bmx, smn, smx;
    carBoxAabb(C, childXf, bmn, bmx);
    ballAabb(P, W.b[0].xf, smn, smx);
    if (!aabbOverlap(bmn, bmx, smn, smx)) return;
    int mi = newManifold(W, carObj, OBJ_BALL, fmin_(C.cbt, P.ballCbt));
    if (mi < 0) return;
    Manifold& man = W.m[mi];
    ObjRef rBall = objRef(W, OBJ_BALL), rCar = objRef(W, carObj);
    ConvexShape box = carBoxShape(C), sph = makeSphere(P.ballRadius);
    float maxDist2 = sq((C.boxMargin + P.ballMargin) + man.cbt);
    GjkOut g = gjkPairDetector(W.epa, box, childXf, sph, W.b[0].xf, maxDist2);
    if (g.overflow) W.status |= WS_EPA_OVERFLOW;
    if (g.has) {
        int idx = addContact(man, W.pool, OBJ_BALL, rBall, carObj, rCar, g.normal, g.point, g.dist);
        if (idx >= 0 && carResponds(W, ci)) onCarBall(W, ci, man.pt[idx], false);
    }
    if (man.n) refreshContactPoints(man, rCar.xf, rBall.xf);
}

// (car a, car b), a < b: btCompoundCompoundCollisionAlgorithm without child trees falls back to
// the compound algorithm (car a's box vs car b's compound), whose child is a swapped compound
// (car b's box vs car a's box) over btBoxBoxCollisionAlgorithm.  The box-box manifold is built
// with the pair's algorithm, with car b as its body 0.
RSB_HD void collideCarCar(World& W, int ca, int cb) {
    const CarParams& C = W.P->car;
    int objA = OBJ_CAR0 + ca, objB = OBJ_CAR0 + cb;
    int mi = newManifold(W, objB, objA, C.cbt);
    if (mi < 0) return;
    Xf xa = carChildXf(C, W.b[1 + ca].xf), xb = carChildXf(C, W.b[1 + cb].xf);
    V3 aMn, aMx, cMn, cMx, bMn, bMx;
    carBoxAabb(C, xa, aMn, aMx);
    carCompoundAabb(C, W.b[1 + cb].xf, cMn, cMx);
    bool outer = aabbOverlap(aMn, aMx, cMn, cMx);
    bool inner = false;
    if (outer) {
        carBoxAabb(C, xb, bMn, bMx);
        inner = aabbOverlap(bMn, bMx, aMn, aMx);
        if (inner) {
            Manifold& man = W.m[mi];
            ObjRef rA = objRef(W, objA), rB = objRef(W, objB);
            BoxContacts bc;
            boxBoxContacts(xb, C.boxHeM, xa, C.boxHeM, bc);
            bool responds = carResponds(W, ca) && carResponds(W, cb);
            for (int k = 0; k < bc.n; k++) {
                int idx = addContact(man, W.pool, objA, rA, objB, rB, bc.c[k].normalOnB, bc.c[k].point, bc.c[k].depth);
                if (idx >= 0 && responds) onCarCar(W, cb, ca, man.pt[idx]);
            }
            if (man.n) refreshContactPoints(man, rB.xf, rA.xf);
        }
    }
    if (!(outer && inner)) releaseManifold(W, mi);
}

// ------------------------------------------------------------------ dispatch

// btCollisionDispatcher::dispatchAllCollisionPairs in pair order
RSB_HD void dispatchPairs(World& W) {
    W.nm = 0;
    W.pool.n = 0;
    W.pool.status = &W.status;
    for (int p = 0; p < W.np; p++) {
        int o0 = W.po0[p], o1 = W.po1[p];
        if (!objActive(W, o0) && !objActive(W, o1)) continue;  // needsCollision
        if (o1 == OBJ_BALL) {
            int mi = newManifold(W, OBJ_BALL, o0, W.P->ballCbt);
            if (mi < 0) continue;
            if (o0 < MAX_MESHES) collideBallMesh(W, o0, W.m[mi]);
            else collideBallPlane(W, o0, W.m[mi]);
        } else if (objIsStatic(o0)) {
            collideCarStatic(W, o0, o1 - OBJ_CAR0);
        } else if (o0 == OBJ_BALL) {
            collideCarBall(W, o1 - OBJ_CAR0);
        } else {
            collideCarCar(W, o0 - OBJ_CAR0, o1 - OBJ_CAR0);
        }
    }
}

// ------------------------------------------------------------------ wheel ray casts

// Registration order before the car pre-ticks (for the wheel rays).
RSB_HD void buildRayOrder(World& W) { buildRegOrder(W); }

// btDefaultVehicleRaycaster::castRay (btDefaultVehicleRaycaster.cpp:32-53) over
// btCollisionWorld::rayTest with ClosestRayResultCallback ignoring the casting chassis.
// The broadphase hands over every object registered in the cell of the ray start
// (btRSBroadphase::rayTest, btRSBroadphase.cpp:325-356): statics in registration order,
// then dynamic bodies in registration order; objects are tested without AABB culling.
// Returns the object hit, or -1 (also when the closest object has no contact response).
RSB_HD int castRay(const World& W, V3 from, V3 to, int ignoreObj, V3& hitPoint, V3& hitNormal, float& hitFrac) {
    const ArenaStatic& S = *W.S;
    const WorldParams& P = *W.P;
    RayHit hit;
    hit.fraction = 1.f;
    hit.obj = -1;
    hit.normal = v3zero();
    const int rayBody = ignoreObj - OBJ_BALL;  // the casting car's body
    // meshes with a triangle near the segment: no other mesh can be hit
    const V3 tolv{kOccTol, kOccTol, kOccTol};
    const uint32_t meshNear = occMask(S, vmin(from, to) - tolv, vmax(from, to) + tolv);
    // the culling state is read once and the test counts kept in registers
    const bool culled = (W.cull >> rayBody) & 1u, audit = W.cullAudit != 0;
    uint32_t nRun = 0, nSkip = 0;
    bool missed = false;
    auto testObj = [&](int o) {
        if (hit.fraction == 0.f) return;
        if (o == ignoreObj) return;
        if (o < MAX_MESHES && !((meshNear >> o) & 1u)) return;
        if (o < NUM_STATICS) {
            if (culled) {
                nSkip++;
                if (!audit) return;
                // audit: would this static have been hit at all?
                RayHit probe;
                probe.fraction = 1.f;
                probe.obj = -1;
                probe.normal = v3zero();
                if (o < MAX_MESHES) rayVsMesh(S, o, from, to, probe);
                else rayVsPlane(S, o, from, to, probe);
                missed |= probe.obj >= 0;
            }
            nRun++;
            if (o < MAX_MESHES) rayVsMesh(S, o, from, to, hit);
            else rayVsPlane(S, o, from, to, hit);
        } else {
            int bi = o - OBJ_BALL;
            const Body& b = W.b[bi];
            ConvexShape sh;
            Xf x;
            if (bi == 0) {
                sh = makeSphere(P.ballRadius);
                x = b.xf;
            } else {
                sh = carBoxShape(P.car);
                x = carChildXf(P.car, b.xf);
            }
            float frac;
            V3 n;
            if (subsimplexCast(from, to, sh, x, frac, n)) {
                if (length2(n) > 0.0001f && frac < hit.fraction) {
                    hit.fraction = frac;
                    hit.obj = o;
                    hit.normal = normalized(n);
                }
            }
        }
    };
    const BpGrid& g = S.bp;
    float cs2 = g.cellSize * g.cellSize;
    if (dist2(from, to) < cs2) {
        int i, j, k;
        bpCellIndices(g, from, i, j, k);
        int cell = i * g.cellsY * g.cellsZ + j * g.cellsZ + k;
        // the statics registered in the cell, in ascending order: meshes (0..15) first, from
        // the voxel triangle lists when they cover the segment, then the planes
        uint32_t mask = S.bpCells[cell];
        const uint32_t meshes = mask & meshNear & ((1u << MAX_MESHES) - 1u);
        if (meshes && !culled && hit.fraction != 0.f && rayVsMeshesVox(S, meshes, from, to, kOccTol, hit)) {
            nRun += (uint32_t)bitCount(meshes);
            mask &= ~((1u << MAX_MESHES) - 1u);
        }
        for (; mask; mask &= mask - 1u) testObj(lowestBit(mask));
        // dynamic proxies of the cell in registration order (W.reg is built before the
        // car pre-ticks; see RegOrder)
        const RegOrder& R = W.reg;
        uint32_t last = 0;
        bool first = true;
        for (int r = 0; r < R.n; r++) {
            if (!regNear(R, r, i, j, k)) continue;
            if (!first && R.stamp[r] <= last) continue;
            first = false;
            last = R.stamp[r];
            testObj(OBJ_BALL + R.body[r]);
        }
    } else {
        for (int o = 0; o < OBJ_BALL + W.nb; o++) testObj(o);
    }
    W.nStatic += nRun;
    W.nCulled += nSkip;
    if (missed) {
        W.nMissed++;
        W.cullMissed = WS_CULL_MISS;
    }
    if (hit.obj < 0) return -1;
    if (!objIsStatic(hit.obj) && W.b[hit.obj - OBJ_BALL].noResp) return -1;
    float s = 1.f - hit.fraction;
    hitPoint = from * s + to * hit.fraction;
    hitNormal = normalized(hit.normal);
    hitFrac = hit.fraction;
    return hit.obj;
}

// ------------------------------------------------------------------ islands

// btUnionFind with path compression
struct UnionFind {
    int id[MAX_BODIES];
    int sz[MAX_BODIES];
    int n;
    RSB_HD void reset(int k) { n = k; for (int i = 0; i < k; i++) { id[i] = i; sz[i] = 1; } }
    RSB_HD int find(int x) {
        while (x != id[x]) {
            id[x] = id[id[x]];
            x = id[x];
        }
        return x;
    }
    RSB_HD void unite(int p, int q) {
        int i = find(p), j = find(q);
        if (i == j) return;
        id[i] = j;
        sz[j] += sz[i];
    }
};

// btAlignedObjectArray::quickSortInternal on (key, value) pairs, ascending by key.  The
// ranges waiting on the explicit stack are disjoint and hold at least two elements each, so
// sorting at most MAX_MANIFOLDS elements never needs more than MAX_MANIFOLDS / 2 of them;
// should a range not fit, the sort sets WS_OVERFLOW in `status` instead of skipping it
// silently.
constexpr int kSortStack = 2 * (MAX_MANIFOLDS / 2);
RSB_HD void quickSortKV(int* key, int* val, int lo, int hi, uint32_t& status) {
    // explicit stack keeps the device code free of recursion
    int stack[kSortStack];
    int sp = 0;
    stack[sp++] = lo;
    stack[sp++] = hi;
    while (sp > 0) {
        int h = stack[--sp];
        int l = stack[--sp];
        int i = l, j = h;
        int xk = key[(l + h) / 2];
        do {
            while (key[i] < xk) i++;
            while (xk < key[j]) j--;
            if (i <= j) {
                int tk = key[i]; key[i] = key[j]; key[j] = tk;
                int tv = val[i]; val[i] = val[j]; val[j] = tv;
                i++;
                j--;
            }
        } while (i <= j);
        // the reference recurses on (lo, j) first, then (i, hi): push in reverse
        if (i < h) {
            if (sp + 2 <= kSortStack) { stack[sp++] = i; stack[sp++] = h; }
            else status |= WS_OVERFLOW;
        }
        if (l < j) {
            if (sp + 2 <= kSortStack) { stack[sp++] = l; stack[sp++] = j; }
            else status |= WS_OVERFLOW;
        }
    }
}

// btSimulationIslandManager + InplaceSolverIslandCallback + btSequentialImpulseConstraintSolver
RSB_HD void solveIslands(World& W) {
    const float dt = W.P->dt;
    UnionFind uf;
    uf.reset(W.nb);
    for (int i = 0; i < W.nb; i++) W.b[i].islandTag = i;
    // findUnions over the overlapping pairs (dynamic, contact-responding objects only)
    for (int p = 0; p < W.np; p++) {
        int o0 = W.po0[p], o1 = W.po1[p];
        if (objIsStatic(o0) || objIsStatic(o1)) continue;
        const Body& b0 = W.b[o0 - OBJ_BALL];
        const Body& b1 = W.b[o1 - OBJ_BALL];
        if (b0.noResp || b1.noResp) continue;
        uf.unite(b0.islandTag, b1.islandTag);
    }
    for (int i = 0; i < W.nb; i++) W.b[i].islandTag = uf.find(i);

    // sortIslands: element (m_id = find(i), m_sz = collision object index)
    int eid[MAX_BODIES], eobj[MAX_BODIES];
    for (int i = 0; i < W.nb; i++) { eid[i] = uf.find(i); eobj[i] = i; }
    if (W.nb > 1) quickSortKV(eid, eobj, 0, W.nb - 1, W.status);

    // buildIslands: sleeping bookkeeping
    for (int s = 0; s < W.nb;) {
        int island = eid[s];
        int e = s + 1;
        while (e < W.nb && eid[e] == island) e++;
        bool allSleeping = true;
        for (int k = s; k < e; k++) {
            const Body& b = W.b[eobj[k]];
            if (b.islandTag == island && (b.act == ACT_ACTIVE || b.act == ACT_DISABLE_DEACT)) { allSleeping = false; break; }
        }
        for (int k = s; k < e; k++) {
            Body& b = W.b[eobj[k]];
            if (b.islandTag != island) continue;
            if (allSleeping) {
                if (b.act != ACT_DISABLE_DEACT && b.act != ACT_DISABLE_SIM) b.act = ACT_SLEEPING;
            } else if (b.act == ACT_SLEEPING) {
                b.act = ACT_WANTS_DEACT;
            }
        }
        s = e;
    }

    // island manifolds in dispatcher order, then unstable quickSort by island id
    int mkey[MAX_MANIFOLDS], midx[MAX_MANIFOLDS];
    int nim = 0;
    for (int i = 0; i < W.nm; i++) {
        const Manifold& m = W.m[i];
        bool s0 = objIsStatic(m.o0) || W.b[m.o0 - OBJ_BALL].act == ACT_SLEEPING;
        bool s1 = objIsStatic(m.o1) || W.b[m.o1 - OBJ_BALL].act == ACT_SLEEPING;
        if (s0 && s1) continue;
        bool resp0 = objIsStatic(m.o0) ? true : !W.b[m.o0 - OBJ_BALL].noResp;
        bool resp1 = objIsStatic(m.o1) ? true : !W.b[m.o1 - OBJ_BALL].noResp;
        if (!(resp0 && resp1)) continue;
        if (objIsStatic(m.o0) && objIsStatic(m.o1)) continue;
        int t0 = objIsStatic(m.o0) ? -1 : W.b[m.o0 - OBJ_BALL].islandTag;
        int t1 = objIsStatic(m.o1) ? -1 : W.b[m.o1 - OBJ_BALL].islandTag;
        mkey[nim] = t0 >= 0 ? t0 : t1;
        midx[nim] = i;
        nim++;
    }
    if (nim > 1) quickSortKV(mkey, midx, 0, nim - 1, W.status);

    // processIslands -> one batched solveGroup
    int bodyList[MAX_BODIES], nbl = 0;
    int manList[MAX_MANIFOLDS], nml = 0;
    int sm = 0;
    for (int s = 0; s < W.nb;) {
        int island = eid[s];
        int e = s;
        bool sleeping = true;
        int first = nbl;
        for (; e < W.nb && eid[e] == island; e++) {
            bodyList[nbl++] = eobj[e];
            if (W.b[eobj[e]].act != ACT_SLEEPING && W.b[eobj[e]].act != ACT_DISABLE_SIM) sleeping = false;
        }
        int cnt = 0, start = sm;
        if (sm < nim && mkey[sm] == island) {
            int em = sm + 1;
            while (em < nim && mkey[em] == island) em++;
            cnt = em - sm;
        }
        if (sleeping) {
            nbl = first;  // island not processed
        } else {
            for (int k = 0; k < cnt; k++) manList[nml++] = midx[start + k];
        }
        if (cnt) sm = start + cnt;
        s = e;
    }

    // ---- solveGroup
    Solver Sv;
    Sv.nsb = 0;
    Sv.fixedId = -1;
    Sv.nc = 0;
    Sv.nf = 0;
    for (int i = 0; i < W.nb; i++) W.b[i].solverId = -1;
    for (int k = 0; k < nbl; k++) solverBodyOf(Sv, W.b, OBJ_BALL + bodyList[k], dt);
    for (int k = 0; k < nml; k++) {
        Manifold& m = W.m[manList[k]];
        int sA = solverBodyOf(Sv, W.b, m.o0, dt);
        int sB = solverBodyOf(Sv, W.b, m.o1, dt);
        const Body* rb0 = objIsStatic(m.o0) ? nullptr : &W.b[m.o0 - OBJ_BALL];
        const Body* rb1 = objIsStatic(m.o1) ? nullptr : &W.b[m.o1 - OBJ_BALL];
        if (!rb0 && !rb1) continue;
        ObjRef r0 = objRef(W, m.o0), r1 = objRef(W, m.o1);
        for (int j = 0; j < m.n; j++) {
            MPoint& cp = m.pt[j];
            if (Sv.nc >= MAX_CONTACT_ROWS) { W.status |= 2u; break; }
            int row = Sv.nc++;
            SRow& r = Sv.c[row];
            V3 rel1 = cp.posA - r0.xf.o;
            V3 rel2 = cp.posB - r1.xf.o;
            setupContactRow(r, Sv, sA, sB, rb0, rb1, cp.normal, cp.dist, cp.fric, cp.rest, rel1, rel2, dt, cp.special);
            r.fIdx = (int16_t)Sv.nf;
            if (cp.special) {
                for (int side = 0; side < 2; side++) {
                    int o = side ? m.o1 : m.o0;
                    if (objIsStatic(o)) continue;
                    Body& sb = W.b[o - OBJ_BALL];
                    sb.spCount++;
                    sb.spFric = cp.fric;
                    sb.spRest = cp.rest;
                    sb.spNormal = sb.spNormal + cp.normal;
                    sb.spDist = sb.spDist + length(side ? rel2 : rel1);
                }
            }
            if (!addFrictionFor(Sv, row, sA, sB, rb0, rb1, cp.normal, cp.fric, rel1, rel2)) { W.status |= 2u; break; }
        }
    }
    // convertContactSpecial, per body in island order
    for (int k = 0; k < nbl; k++) {
        Body& b = W.b[bodyList[k]];
        if (b.spCount <= 0) continue;
        float distance = b.spDist / (float)b.spCount;
        V3 normal = bdiv(b.spNormal, (float)b.spCount);
        int sA = solverBodyOf(Sv, W.b, OBJ_BALL + bodyList[k], dt);
        if (Sv.fixedId < 0) {
            Sv.fixedId = Sv.nsb++;
            sbInitFixed(Sv.sb[Sv.fixedId]);
        }
        int sB = Sv.fixedId;
        if (Sv.nc < MAX_CONTACT_ROWS) {
            int row = Sv.nc++;
            SRow& r = Sv.c[row];
            V3 rel1 = normal * -distance;
            V3 rel2 = v3zero();
            setupContactRow(r, Sv, sA, sB, &b, nullptr, normal, distance, b.spFric, b.spRest, rel1, rel2, dt, 0);
            r.fIdx = (int16_t)Sv.nf;
            if (!addFrictionFor(Sv, row, sA, sB, &b, nullptr, normal, b.spFric, rel1, rel2)) W.status |= 2u;
        } else {
            W.status |= 2u;
        }
        b.spCount = 0;
        b.spFric = b.spRest = b.spDist = 0.f;
        b.spNormal = v3zero();
    }
    W.nRows += (uint32_t)(Sv.nc + Sv.nf);
    solverIterate(Sv);
    solverWriteBack(Sv, W.b, W.noRot, dt);
}

// ------------------------------------------------------------------ integration

RSB_HD void updateInertia(Body& b) { b.invIw = scaled(b.xf.b, b.invIl) * transpose(b.xf.b); }

RSB_HD void predictMotion(World& W) {
    const float dt = W.P->dt;
    for (int i = 0; i < W.nb; i++) {
        Body& b = W.b[i];
        // applyDamping (angular damping is 0: the factor pow(1, dt) is exactly 1)
        b.lin = b.lin * b.linDampFactor;
        b.ixf = W.noRot[i] ? integrateTransformNoRot(b.xf, b.lin, dt) : integrateTransform(b.xf, b.lin, b.ang, dt);
    }
}

RSB_HD void integrateBodies(World& W) {
    const float dt = W.P->dt;
    for (int i = 0; i < W.nb; i++) {
        Body& b = W.b[i];
        if (b.act == ACT_SLEEPING || b.act == ACT_DISABLE_SIM) continue;
        Xf pred = W.noRot[i] ? integrateTransformNoRot(b.xf, b.lin, dt) : integrateTransform(b.xf, b.lin, b.ang, dt);
        b.xf = pred;
        b.ixf = pred;
        updateInertia(b);
    }
}

// updateActivationState: with RocketSim resetting the activation of the ball and cars at
// the start of every tick, only the ISLAND_SLEEPING velocity zeroing has an effect.
RSB_HD void updateActivation(World& W) {
    for (int i = 0; i < W.nb; i++) {
        Body& b = W.b[i];
        if (b.act == ACT_SLEEPING) {
            b.lin = v3zero();
            b.ang = v3zero();
        }
    }
}

// stepSimulation(dt, 0, dt): gravity, one internal step, clearForces
RSB_HD void worldStep(World& W) {
    for (int i = 0; i < W.nb; i++) {
        Body& b = W.b[i];
        if (b.act != ACT_SLEEPING && b.act != ACT_DISABLE_SIM) b.force = b.force + b.grav;
    }
    predictMotion(W);
    for (int i = 0; i < W.nb; i++) updateBodyAabb(W, i);
    computePairs(W);
    dispatchPairs(W);
    solveIslands(W);
    integrateBodies(W);
    updateActivation(W);
    for (int i = 0; i < W.nb; i++) {
        W.b[i].force = v3zero();
        W.b[i].torque = v3zero();
    }
}

}  // namespace rsb
