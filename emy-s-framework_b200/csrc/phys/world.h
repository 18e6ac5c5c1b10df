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
#pragma once
#include "contacts.h"
#include "solver.h"

namespace rsb {

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
};

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

RSB_HD void bodyShapeAabb(const World& W, int bi, const Xf& xf, V3& mn, V3& mx) {
    if (bi == 0) ballAabb(*W.P, xf, mn, mx);
    else { mn = xf.o; mx = xf.o; }  // cars: filled in by the car module
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

// btRSBroadphase::calculateOverlappingPairs
RSB_HD void computePairs(World& W) {
    W.np = 0;
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
            int inCell = 0;
            for (int e = 0; e < W.nb; e++) inCell += inRegNeighbourhood(W.b[e], ci, cj, ck) ? 1 : 0;
            if (inCell > 1) {
                // visit the other dynamic proxies of this cell in registration order
                uint32_t last = 0;
                bool first = true;
                for (int it = 0; it < W.nb; it++) {
                    int pick = -1;
                    uint32_t best = 0xffffffffu;
                    for (int e = 0; e < W.nb; e++) {
                        if (!inRegNeighbourhood(W.b[e], ci, cj, ck)) continue;
                        uint32_t st = W.b[e].regStamp;
                        if ((first || st > last) && st < best) { best = st; pick = e; }
                    }
                    if (pick < 0) break;
                    first = false;
                    last = best;
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
    V3 amn, amx;
    ballAabb(P, ball.xf, amn, amx);  // convexInTriangleSpace == ball transform (mesh at identity)
    M3 invB = inverse(ball.xf.b);
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
    V3 vtx = sphereSupport(planeInConvex.b * (-pn), P.ballMargin);
    V3 vip = xfPoint(convexInPlane, vtx);
    float distance = dot(pn, vip) - pc;
    if (distance < man.cbt + 0.f) {
        V3 proj = vip - pn * distance;
        V3 world = xfPoint(rPlane.xf, proj);
        V3 nb = rPlane.xf.b * pn;
        int idx = addContact(man, W.pool, plane, rPlane, OBJ_BALL, rBall, nb, world, distance);
        if (idx >= 0) man.pt[idx].special = 1;
    }
    if (man.n) refreshContactPoints(man, rBall.xf, rPlane.xf);
}

// ------------------------------------------------------------------ dispatch

RSB_HD void dispatchPairs(World& W) {
    W.nm = 0;
    W.pool.n = 0;
    W.pool.status = &W.status;
    for (int p = 0; p < W.np; p++) {
        int o0 = W.po0[p], o1 = W.po1[p];
        if (!objActive(W, o0) && !objActive(W, o1)) continue;  // needsCollision
        if (o1 == OBJ_BALL && objIsStatic(o0)) {
            if (W.nm >= MAX_MANIFOLDS) { W.status |= 2u; continue; }
            Manifold& man = W.m[W.nm++];
            man.o0 = OBJ_BALL;
            man.o1 = o0;
            man.cbt = W.P->ballCbt;
            man.n = 0;
            man.pt = nullptr;
            if (o0 < MAX_MESHES) collideBallMesh(W, o0, man);
            else collideBallPlane(W, o0, man);
        }
        // car pairs are handled by the car narrowphase (added with the vehicle module)
    }
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

// btAlignedObjectArray::quickSortInternal on (key, value) pairs, ascending by key
RSB_HD void quickSortKV(int* key, int* val, int lo, int hi) {
    // explicit stack keeps the device code free of recursion
    int stack[64];
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
        if (i < h && sp + 2 <= 64) { stack[sp++] = i; stack[sp++] = h; }
        if (l < j && sp + 2 <= 64) { stack[sp++] = l; stack[sp++] = j; }
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
    if (W.nb > 1) quickSortKV(eid, eobj, 0, W.nb - 1);

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
    if (nim > 1) quickSortKV(mkey, midx, 0, nim - 1);

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
