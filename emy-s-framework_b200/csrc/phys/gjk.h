// Closest points and penetration between convex shapes.
//
//   VoronoiSimplex ..... btVoronoiSimplexSolver (btVoronoiSimplexSolver.cpp:34-577), with
//                        BT_USE_EQUAL_VERTEX_THRESHOLD (0.0001) and CATCH_DEGENERATE_TETRAHEDRON
//   gjkPairDetector .... btGjkPairDetector::getClosestPointsNonVirtual as RocketSim patches it
//                        (btGjkPairDetector.cpp:685-959): origins re-centred on their midpoint,
//                        margins added after the core GJK, EPA on penetration and the
//                        contact-normal direction fix from the shapes' AABB centres
//   epaPenetration ..... btGjkEpaPenetrationDepthSolver::calcPenDepth
//                        (btGjkEpaPenetrationDepthSolver.cpp:22-79) over gjkepa2_impl's GJK and
//                        EPA (btGjkEpa2.cpp:51-1030); faces and support vertices live in
//                        fixed arrays addressed by index, and EPA's recursive horizon walk
//                        runs on an explicit stack in the same visiting order
//   subsimplexCast ..... btSubsimplexConvexCast::calcTimeOfImpact (btSubSimplexConvexCast.cpp:31-147)
//
// ALTERED SOURCE: this file is not the original Bullet code.  It restates the algorithms of
// the Bullet 3.24 files named above (as patched in RocketSim) for a CUDA device and a host
// build, with its own data layout, naming and control flow; the original's notice follows.
//
// Bullet Continuous Collision Detection and Physics Library
// Copyright (c) 2003-2008 Erwin Coumans  https://bulletphysics.org
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
//
// GJK-EPA collision solver by Nathanael Presson, 2008
#pragma once
#include "shapes.h"

namespace rsb {

// ------------------------------------------------------------------ Voronoi simplex solver

struct SubSimplexResult {
    V3 closest;
    uint32_t used;  // bit i: vertex i used
    float bc[4];
    bool degenerate;
    RSB_HD void reset() {
        degenerate = false;
        bc[0] = bc[1] = bc[2] = bc[3] = 0.f;
        used = 0;
    }
    RSB_HD void setBC(float a, float b, float c, float d) { bc[0] = a; bc[1] = b; bc[2] = c; bc[3] = d; }
    RSB_HD bool isValid() const { return bc[0] >= 0.f && bc[1] >= 0.f && bc[2] >= 0.f && bc[3] >= 0.f; }
};

struct VoronoiSimplex {
    int n;
    V3 W[5], P[5], Q[5];
    V3 lastW;
    bool needsUpdate, cachedValid;
    V3 cP1, cP2, cV;
    SubSimplexResult bc;

    RSB_HD void reset() {
        cachedValid = false;
        n = 0;
        needsUpdate = true;
        lastW = V3{kLargeFloat, kLargeFloat, kLargeFloat};
        bc.reset();
    }
    RSB_HD void removeVertex(int i) {
        n--;
        W[i] = W[n];
        P[i] = P[n];
        Q[i] = Q[n];
    }
    RSB_HD void reduce(uint32_t used) {
        if (n >= 4 && !(used & 8)) removeVertex(3);
        if (n >= 3 && !(used & 4)) removeVertex(2);
        if (n >= 2 && !(used & 2)) removeVertex(1);
        if (n >= 1 && !(used & 1)) removeVertex(0);
    }
    RSB_HD void addVertex(V3 w, V3 p, V3 q) {
        lastW = w;
        needsUpdate = true;
        W[n] = w;
        P[n] = p;
        Q[n] = q;
        n++;
    }
    RSB_HD bool inSimplex(V3 w) const {
        bool found = false;
        for (int i = 0; i < n; i++)
            if (length2(w - W[i]) <= 0.0001f) { found = true; break; }
        if (w == lastW) return true;
        return found;
    }
    RSB_HD bool full() const { return n == 4; }

    static RSB_HD void closestPtTri(V3 p, V3 a, V3 b, V3 c, SubSimplexResult& r) {
        r.used = 0;
        V3 ab = b - a, ac = c - a, ap = p - a;
        float d1 = dot(ab, ap), d2 = dot(ac, ap);
        if (d1 <= 0.f && d2 <= 0.f) {
            r.closest = a; r.used = 1; r.setBC(1, 0, 0, 0);
            return;
        }
        V3 bp = p - b;
        float d3 = dot(ab, bp), d4 = dot(ac, bp);
        if (d3 >= 0.f && d4 <= d3) {
            r.closest = b; r.used = 2; r.setBC(0, 1, 0, 0);
            return;
        }
        float vc = d1 * d4 - d3 * d2;
        if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
            float v = d1 / (d1 - d3);
            r.closest = a + v * ab; r.used = 3; r.setBC(1 - v, v, 0, 0);
            return;
        }
        V3 cp = p - c;
        float d5 = dot(ab, cp), d6 = dot(ac, cp);
        if (d6 >= 0.f && d5 <= d6) {
            r.closest = c; r.used = 4; r.setBC(0, 0, 1, 0);
            return;
        }
        float vb = d5 * d2 - d1 * d6;
        if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
            float w = d2 / (d2 - d6);
            r.closest = a + w * ac; r.used = 5; r.setBC(1 - w, 0, w, 0);
            return;
        }
        float va = d3 * d6 - d5 * d4;
        if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
            float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
            r.closest = b + w * (c - b); r.used = 6; r.setBC(0, 1 - w, w, 0);
            return;
        }
        float denom = 1.f / (va + vb + vc);
        float v = vb * denom, w = vc * denom;
        r.closest = (a + ab * v) + ac * w;
        r.used = 7;
        r.setBC((1 - v) - w, v, w, 0);
    }

    static RSB_HD int outsidePlane(V3 p, V3 a, V3 b, V3 c, V3 d) {
        V3 nrm = cross(b - a, c - a);
        float sp = dot(p - a, nrm), sd = dot(d - a, nrm);
        if (sd * sd < (1e-4f * 1e-4f)) return -1;
        return sp * sd < 0.f;
    }

    static RSB_HD bool closestPtTetra(V3 p, V3 a, V3 b, V3 c, V3 d, SubSimplexResult& fin) {
        SubSimplexResult t;
        t.reset();
        fin.closest = p;
        fin.used = 15;
        int oABC = outsidePlane(p, a, b, c, d);
        int oACD = outsidePlane(p, a, c, d, b);
        int oADB = outsidePlane(p, a, d, b, c);
        int oBDC = outsidePlane(p, b, d, c, a);
        if (oABC < 0 || oACD < 0 || oADB < 0 || oBDC < 0) {
            fin.degenerate = true;
            return false;
        }
        if (!oABC && !oACD && !oADB && !oBDC) return false;
        float best = 3.402823466e+38f;
        if (oABC) {
            closestPtTri(p, a, b, c, t);
            V3 q = t.closest;
            float sq = dot(q - p, q - p);
            if (sq < best) {
                best = sq;
                fin.closest = q;
                fin.used = t.used & 7;
                fin.setBC(t.bc[0], t.bc[1], t.bc[2], 0);
            }
        }
        if (oACD) {
            closestPtTri(p, a, c, d, t);
            V3 q = t.closest;
            float sq = dot(q - p, q - p);
            if (sq < best) {
                best = sq;
                fin.closest = q;
                fin.used = (t.used & 1) | ((t.used & 2) ? 4u : 0u) | ((t.used & 4) ? 8u : 0u);
                fin.setBC(t.bc[0], 0, t.bc[1], t.bc[2]);
            }
        }
        if (oADB) {
            closestPtTri(p, a, d, b, t);
            V3 q = t.closest;
            float sq = dot(q - p, q - p);
            if (sq < best) {
                best = sq;
                fin.closest = q;
                fin.used = (t.used & 1) | ((t.used & 4) ? 2u : 0u) | ((t.used & 2) ? 8u : 0u);
                fin.setBC(t.bc[0], t.bc[2], 0, t.bc[1]);
            }
        }
        if (oBDC) {
            closestPtTri(p, b, d, c, t);
            V3 q = t.closest;
            float sq = dot(q - p, q - p);
            if (sq < best) {
                best = sq;
                fin.closest = q;
                fin.used = ((t.used & 1) ? 2u : 0u) | ((t.used & 4) ? 4u : 0u) | ((t.used & 2) ? 8u : 0u);
                fin.setBC(0, t.bc[0], t.bc[2], t.bc[1]);
            }
        }
        return true;
    }

    RSB_HD bool update() {
        if (!needsUpdate) return cachedValid;
        bc.reset();
        needsUpdate = false;
        switch (n) {
            case 0:
                cachedValid = false;
                break;
            case 1: {
                cP1 = P[0];
                cP2 = Q[0];
                cV = cP1 - cP2;
                bc.reset();
                bc.setBC(1, 0, 0, 0);
                cachedValid = bc.isValid();
                break;
            }
            case 2: {
                V3 from = W[0], to = W[1];
                V3 diff = v3zero() - from;
                V3 v = to - from;
                float t = dot(v, diff);
                if (t > 0) {
                    float dvv = dot(v, v);
                    if (t < dvv) {
                        t /= dvv;
                        bc.used |= 3;
                    } else {
                        t = 1;
                        bc.used |= 2;
                    }
                } else {
                    t = 0;
                    bc.used |= 1;
                }
                bc.setBC(1 - t, t, 0, 0);
                cP1 = P[0] + t * (P[1] - P[0]);
                cP2 = Q[0] + t * (Q[1] - Q[0]);
                cV = cP1 - cP2;
                reduce(bc.used);
                cachedValid = bc.isValid();
                break;
            }
            case 3: {
                closestPtTri(v3zero(), W[0], W[1], W[2], bc);
                cP1 = (P[0] * bc.bc[0] + P[1] * bc.bc[1]) + P[2] * bc.bc[2];
                cP2 = (Q[0] * bc.bc[0] + Q[1] * bc.bc[1]) + Q[2] * bc.bc[2];
                cV = cP1 - cP2;
                reduce(bc.used);
                cachedValid = bc.isValid();
                break;
            }
            case 4: {
                bool sep = closestPtTetra(v3zero(), W[0], W[1], W[2], W[3], bc);
                if (sep) {
                    cP1 = ((P[0] * bc.bc[0] + P[1] * bc.bc[1]) + P[2] * bc.bc[2]) + P[3] * bc.bc[3];
                    cP2 = ((Q[0] * bc.bc[0] + Q[1] * bc.bc[1]) + Q[2] * bc.bc[2]) + Q[3] * bc.bc[3];
                    cV = cP1 - cP2;
                    reduce(bc.used);
                } else {
                    if (bc.degenerate) {
                        cachedValid = false;
                    } else {
                        cachedValid = true;
                        cV = v3zero();
                    }
                    break;
                }
                cachedValid = bc.isValid();
                break;
            }
            default:
                cachedValid = false;
        }
        return cachedValid;
    }
    RSB_HD bool closest(V3& v) {
        bool ok = update();
        v = cV;
        return ok;
    }
    RSB_HD void computePoints(V3& p1, V3& p2) {
        update();
        p1 = cP1;
        p2 = cP2;
    }
};

// ------------------------------------------------------------------ gjkepa2 (EPA path)

constexpr int EPA_MAX_VERTICES = 128;
constexpr int EPA_MAX_FACES = EPA_MAX_VERTICES * 2;
constexpr int EPA_SV = 4 + EPA_MAX_VERTICES;  // GJK's four support vertices, then EPA's
constexpr int EPA_STACK = 256;

// MinkowskiDiff: shape 1 is evaluated in shape 0's frame; `margins` selects
// localGetSupportVertexNonVirtual (Penetration) or the margin-free variant (Distance).
struct MinkowskiDiff {
    const ConvexShape* s0;
    const ConvexShape* s1;
    M3 toShape1;
    Xf toShape0;
    bool margins;
    RSB_HD V3 ls(const ConvexShape& s, V3 d) const { return margins ? supportMarginN(s, d) : supportNoMargin(s, d); }
    RSB_HD V3 support0(V3 d) const { return ls(*s0, d); }
    RSB_HD V3 support1(V3 d) const { return xfPoint(toShape0, ls(*s1, toShape1 * d)); }
    RSB_HD V3 support(V3 d) const { return support0(d) - support1(-d); }
};

struct EpaSV {
    V3 d, w;
};
struct EpaFace {
    V3 n;
    float d;
    uint8_t c[3];   // support vertex indices
    uint8_t f[3];   // adjacent faces
    uint8_t e[3];   // matching edge in the adjacent face
    uint8_t pass;
    int16_t l[2];   // list links (-1 = none)
};

struct EpaWork {
    EpaSV sv[EPA_SV];
    EpaFace fc[EPA_MAX_FACES];
    int16_t stkF[EPA_STACK];
    uint8_t stkE[EPA_STACK], stkS[EPA_STACK];
};

struct EpaSimplex {
    uint8_t c[4];
    float p[4];
    uint32_t rank;
};

struct EpaSolver {
    EpaWork* wk;
    MinkowskiDiff shape;
    // GJK state
    V3 ray;
    float distance;
    EpaSimplex simplices[2];
    uint8_t freeIdx[4];
    uint32_t nfree;
    uint32_t current;
    int simplexSel;
    int gjkStatus;  // 0 valid, 1 inside, 2 failed
    // EPA state
    int epaStatus;
    EpaSimplex result;
    V3 normal;
    float depth;
    uint32_t nextsv;
    int16_t hullRoot, stockRoot;
    uint32_t hullCount, stockCount;
    bool overflow;

    RSB_HD EpaSimplex& simplex() { return simplices[simplexSel]; }

    RSB_HD void getsupport(V3 d, EpaSV& sv) const {
        sv.d = bdiv(d, length(d));
        sv.w = shape.support(sv.d);
    }
    RSB_HD void removevertice(EpaSimplex& s) { freeIdx[nfree++] = s.c[--s.rank]; }
    RSB_HD void appendvertice(EpaSimplex& s, V3 v) {
        s.p[s.rank] = 0;
        s.c[s.rank] = freeIdx[--nfree];
        getsupport(v, wk->sv[s.c[s.rank++]]);
    }
    static RSB_HD float det(V3 a, V3 b, V3 c) {
        return a.y * b.z * c.x + a.z * b.x * c.y - a.x * b.z * c.y - a.y * b.x * c.z + a.x * b.y * c.z - a.z * b.y * c.x;
    }
    static RSB_HD float projectorigin2(V3 a, V3 b, float* w, uint32_t& m) {
        V3 d = b - a;
        float l = length2(d);
        if (l > 0.f) {
            float t = l > 0 ? -dot(a, d) / l : 0;
            if (t >= 1) {
                w[0] = 0; w[1] = 1; m = 2;
                return length2(b);
            } else if (t <= 0) {
                w[0] = 1; w[1] = 0; m = 1;
                return length2(a);
            } else {
                w[1] = t;
                w[0] = 1 - t;
                m = 3;
                return length2(a + d * t);
            }
        }
        return -1;
    }
    static RSB_HD float projectorigin3(V3 a, V3 b, V3 c, float* w, uint32_t& m) {
        const uint32_t imd3[] = {1, 2, 0};
        const V3 vt[] = {a, b, c};
        const V3 dl[] = {a - b, b - c, c - a};
        V3 n = cross(dl[0], dl[1]);
        float l = length2(n);
        if (l > 0.f) {
            float mindist = -1;
            float subw[2] = {0.f, 0.f};
            uint32_t subm = 0;
            for (uint32_t i = 0; i < 3; ++i) {
                if (dot(vt[i], cross(dl[i], n)) > 0) {
                    uint32_t j = imd3[i];
                    float subd = projectorigin2(vt[i], vt[j], subw, subm);
                    if ((mindist < 0) || (subd < mindist)) {
                        mindist = subd;
                        m = ((subm & 1) ? 1u << i : 0u) + ((subm & 2) ? 1u << j : 0u);
                        w[i] = subw[0];
                        w[j] = subw[1];
                        w[imd3[j]] = 0;
                    }
                }
            }
            if (mindist < 0) {
                float d = dot(a, n);
                float s = fsqrt(l);
                V3 p = n * (d / l);
                mindist = length2(p);
                m = 7;
                w[0] = length(cross(dl[1], b - p)) / s;
                w[1] = length(cross(dl[2], c - p)) / s;
                w[2] = 1 - (w[0] + w[1]);
            }
            return mindist;
        }
        return -1;
    }
    static RSB_HD float projectorigin4(V3 a, V3 b, V3 c, V3 d, float* w, uint32_t& m) {
        const uint32_t imd3[] = {1, 2, 0};
        const V3 vt[] = {a, b, c, d};
        const V3 dl[] = {a - d, b - d, c - d};
        float vl = det(dl[0], dl[1], dl[2]);
        bool ng = (vl * dot(a, cross(b - c, a - b))) <= 0;
        if (ng && (fabsf(vl) > 0.f)) {
            float mindist = -1;
            float subw[3] = {0.f, 0.f, 0.f};
            uint32_t subm = 0;
            for (uint32_t i = 0; i < 3; ++i) {
                uint32_t j = imd3[i];
                float s = vl * dot(d, cross(dl[i], dl[j]));
                if (s > 0) {
                    float subd = projectorigin3(vt[i], vt[j], d, subw, subm);
                    if ((mindist < 0) || (subd < mindist)) {
                        mindist = subd;
                        m = ((subm & 1) ? 1u << i : 0u) + ((subm & 2) ? 1u << j : 0u) + ((subm & 4) ? 8u : 0u);
                        w[i] = subw[0];
                        w[j] = subw[1];
                        w[imd3[j]] = 0;
                        w[3] = subw[2];
                    }
                }
            }
            if (mindist < 0) {
                mindist = 0;
                m = 15;
                w[0] = det(c, b, d) / vl;
                w[1] = det(a, c, d) / vl;
                w[2] = det(b, a, d) / vl;
                w[3] = 1 - ((w[0] + w[1]) + w[2]);
            }
            return mindist;
        }
        return -1;
    }

    // GJK::Evaluate (btGjkEpa2.cpp:200-330)
    RSB_HD int gjkEvaluate(V3 guess) {
        uint32_t iterations = 0;
        float sqdist = 0, alpha = 0;
        V3 lastw[4];
        uint32_t clastw = 0;
        freeIdx[0] = 0; freeIdx[1] = 1; freeIdx[2] = 2; freeIdx[3] = 3;
        nfree = 4;
        current = 0;
        gjkStatus = 0;
        distance = 0;
        simplices[0].rank = 0;
        ray = guess;
        float sqrl = length2(ray);
        appendvertice(simplices[0], sqrl > 0 ? -ray : V3{1, 0, 0});
        simplices[0].p[0] = 1;
        ray = wk->sv[simplices[0].c[0]].w;
        sqdist = sqrl;
        lastw[0] = lastw[1] = lastw[2] = lastw[3] = ray;
        do {
            uint32_t next = 1 - current;
            EpaSimplex& cs = simplices[current];
            EpaSimplex& ns = simplices[next];
            float rl = length(ray);
            if (rl < 0.0001f) {
                gjkStatus = 1;
                break;
            }
            appendvertice(cs, -ray);
            V3 w = wk->sv[cs.c[cs.rank - 1]].w;
            bool found = false;
            for (uint32_t i = 0; i < 4; ++i)
                if (length2(w - lastw[i]) < 0.0001f) { found = true; break; }
            if (found) {
                removevertice(simplices[current]);
                break;
            } else {
                lastw[clastw = (clastw + 1) & 3] = w;
            }
            float omega = dot(ray, w) / rl;
            alpha = fmax_(omega, alpha);
            if (((rl - alpha) - (0.0001f * rl)) <= 0) {
                removevertice(simplices[current]);
                break;
            }
            float weights[4];
            uint32_t mask = 0;
            switch (cs.rank) {
                case 2: sqdist = projectorigin2(wk->sv[cs.c[0]].w, wk->sv[cs.c[1]].w, weights, mask); break;
                case 3: sqdist = projectorigin3(wk->sv[cs.c[0]].w, wk->sv[cs.c[1]].w, wk->sv[cs.c[2]].w, weights, mask); break;
                case 4:
                    sqdist = projectorigin4(wk->sv[cs.c[0]].w, wk->sv[cs.c[1]].w, wk->sv[cs.c[2]].w, wk->sv[cs.c[3]].w, weights, mask);
                    break;
            }
            if (sqdist >= 0) {
                ns.rank = 0;
                ray = v3zero();
                current = next;
                for (uint32_t i = 0, ni = cs.rank; i < ni; ++i) {
                    if (mask & (1u << i)) {
                        ns.c[ns.rank] = cs.c[i];
                        ns.p[ns.rank++] = weights[i];
                        ray += wk->sv[cs.c[i]].w * weights[i];
                    } else {
                        freeIdx[nfree++] = cs.c[i];
                    }
                }
                if (mask == 15) gjkStatus = 1;
            } else {
                removevertice(simplices[current]);
                break;
            }
            gjkStatus = ((++iterations) < 128u) ? gjkStatus : 2;
        } while (gjkStatus == 0);
        simplexSel = (int)current;
        if (gjkStatus == 0) distance = length(ray);
        else if (gjkStatus == 1) distance = 0;
        return gjkStatus;
    }

    // GJK::EncloseOrigin, recursion unrolled by rank (each level tries the same candidate
    // directions in the same order and undoes its append before the next try)
    RSB_HD bool encloseOrigin() {
        EpaSimplex& s = simplex();
        if (s.rank == 1) {
            for (int i = 0; i < 3; ++i) {
                V3 axis = v3zero();
                axis[i] = 1;
                for (int sg = 0; sg < 2; sg++) {
                    appendvertice(s, sg ? -axis : axis);
                    if (enclose2()) return true;
                    removevertice(s);
                }
            }
            return false;
        }
        if (s.rank == 2) return enclose2();
        if (s.rank == 3) return enclose3();
        if (s.rank == 4) return enclose4();
        return false;
    }
    RSB_HD bool enclose2() {
        EpaSimplex& s = simplex();
        V3 d = wk->sv[s.c[1]].w - wk->sv[s.c[0]].w;
        for (int i = 0; i < 3; ++i) {
            V3 axis = v3zero();
            axis[i] = 1;
            V3 p = cross(d, axis);
            if (length2(p) > 0) {
                for (int sg = 0; sg < 2; sg++) {
                    appendvertice(s, sg ? -p : p);
                    if (enclose3()) return true;
                    removevertice(s);
                }
            }
        }
        return false;
    }
    RSB_HD bool enclose3() {
        EpaSimplex& s = simplex();
        V3 n = cross(wk->sv[s.c[1]].w - wk->sv[s.c[0]].w, wk->sv[s.c[2]].w - wk->sv[s.c[0]].w);
        if (length2(n) > 0) {
            for (int sg = 0; sg < 2; sg++) {
                appendvertice(s, sg ? -n : n);
                if (enclose4()) return true;
                removevertice(s);
            }
        }
        return false;
    }
    RSB_HD bool enclose4() {
        EpaSimplex& s = simplex();
        return fabsf(det(wk->sv[s.c[0]].w - wk->sv[s.c[3]].w, wk->sv[s.c[1]].w - wk->sv[s.c[3]].w,
                         wk->sv[s.c[2]].w - wk->sv[s.c[3]].w)) > 0;
    }

    // ---- EPA lists
    RSB_HD void listAppend(bool hull, int16_t f) {
        int16_t& root = hull ? hullRoot : stockRoot;
        EpaFace& F = wk->fc[f];
        F.l[0] = -1;
        F.l[1] = root;
        if (root >= 0) wk->fc[root].l[0] = f;
        root = f;
        if (hull) hullCount++; else stockCount++;
    }
    RSB_HD void listRemove(bool hull, int16_t f) {
        int16_t& root = hull ? hullRoot : stockRoot;
        EpaFace& F = wk->fc[f];
        if (F.l[1] >= 0) wk->fc[F.l[1]].l[0] = F.l[0];
        if (F.l[0] >= 0) wk->fc[F.l[0]].l[1] = F.l[1];
        if (f == root) root = F.l[1];
        if (hull) hullCount--; else stockCount--;
    }
    RSB_HD void bind(int16_t fa, uint32_t ea, int16_t fb, uint32_t eb) {
        wk->fc[fa].e[ea] = (uint8_t)eb;
        wk->fc[fa].f[ea] = (uint8_t)fb;
        wk->fc[fb].e[eb] = (uint8_t)ea;
        wk->fc[fb].f[eb] = (uint8_t)fa;
    }
    RSB_HD bool getedgedist(const EpaFace& face, int ia, int ib, float& dist) const {
        V3 a = wk->sv[ia].w, b = wk->sv[ib].w;
        V3 ba = b - a;
        V3 nab = cross(ba, face.n);
        float adn = dot(a, nab);
        if (adn < 0) {
            float ba2 = length2(ba);
            float adba = dot(a, ba), bdba = dot(b, ba);
            if (adba > 0) dist = length(a);
            else if (bdba < 0) dist = length(b);
            else {
                float adb = dot(a, b);
                dist = fsqrt(fmax_((length2(a) * length2(b) - adb * adb) / ba2, 0.f));
            }
            return true;
        }
        return false;
    }
    RSB_HD int16_t newface(int ia, int ib, int ic, bool forced) {
        if (stockRoot >= 0) {
            int16_t f = stockRoot;
            listRemove(false, f);
            listAppend(true, f);
            EpaFace& F = wk->fc[f];
            F.pass = 0;
            F.c[0] = (uint8_t)ia;
            F.c[1] = (uint8_t)ib;
            F.c[2] = (uint8_t)ic;
            V3 a = wk->sv[ia].w, b = wk->sv[ib].w, c = wk->sv[ic].w;
            F.n = cross(b - a, c - a);
            float l = length(F.n);
            bool v = l > 0.0001f;
            if (v) {
                if (!(getedgedist(F, ia, ib, F.d) || getedgedist(F, ib, ic, F.d) || getedgedist(F, ic, ia, F.d)))
                    F.d = dot(a, F.n) / l;
                F.n = bdiv(F.n, l);
                if (forced || (F.d >= -0.00001f)) return f;
                epaStatus = 3;  // NonConvex
            } else {
                epaStatus = 2;  // Degenerated
            }
            listRemove(true, f);
            listAppend(false, f);
            return -1;
        }
        epaStatus = (stockRoot >= 0) ? 6 : 5;
        return -1;
    }
    RSB_HD int16_t findbest() const {
        int16_t minf = hullRoot;
        float mind = wk->fc[minf].d * wk->fc[minf].d;
        for (int16_t f = wk->fc[minf].l[1]; f >= 0; f = wk->fc[f].l[1]) {
            float sqd = wk->fc[f].d * wk->fc[f].d;
            if (sqd < mind) { minf = f; mind = sqd; }
        }
        return minf;
    }
    // EPA::expand (recursive in the reference), walked with an explicit frame stack
    RSB_HD bool expand(uint8_t pass, int wIdx, int16_t f0, uint8_t e0, int16_t& hcf, int16_t& hff, uint32_t& hnf) {
        const uint8_t i1m3[] = {1, 2, 0};
        const uint8_t i2m3[] = {2, 0, 1};
        int sp = 0;
        bool ret = false;
        wk->stkF[sp] = f0; wk->stkE[sp] = e0; wk->stkS[sp] = 0; sp++;
        while (sp > 0) {
            int top = sp - 1;
            int16_t f = wk->stkF[top];
            uint8_t e = wk->stkE[top];
            EpaFace& F = wk->fc[f];
            if (wk->stkS[top] == 0) {
                if (F.pass == pass) { ret = false; sp--; continue; }
                uint8_t e1 = i1m3[e];
                if ((dot(F.n, wk->sv[wIdx].w) - F.d) < -0.00001f) {
                    int16_t nf = newface(F.c[e1], F.c[e], wIdx, false);
                    if (nf >= 0) {
                        bind(nf, 0, f, e);
                        if (hcf >= 0) bind(hcf, 1, nf, 2);
                        else hff = nf;
                        hcf = nf;
                        ++hnf;
                        ret = true;
                    } else {
                        ret = false;
                    }
                    sp--;
                    continue;
                }
                F.pass = pass;
                wk->stkS[top] = 1;
                if (sp >= EPA_STACK) { overflow = true; return false; }
                wk->stkF[sp] = (int16_t)F.f[e1]; wk->stkE[sp] = F.e[e1]; wk->stkS[sp] = 0; sp++;
                continue;
            }
            if (wk->stkS[top] == 1) {
                if (!ret) { sp--; continue; }
                wk->stkS[top] = 2;
                uint8_t e2 = i2m3[e];
                if (sp >= EPA_STACK) { overflow = true; return false; }
                wk->stkF[sp] = (int16_t)F.f[e2]; wk->stkE[sp] = F.e[e2]; wk->stkS[sp] = 0; sp++;
                continue;
            }
            if (ret) {
                listRemove(true, f);
                listAppend(false, f);
            }
            sp--;
        }
        return ret;
    }

    // EPA::Evaluate (btGjkEpa2.cpp:640-770)
    RSB_HD int epaEvaluate(V3 guess) {
        EpaSimplex& s = simplex();
        if ((s.rank > 1) && encloseOrigin()) {
            while (hullRoot >= 0) {
                int16_t f = hullRoot;
                listRemove(true, f);
                listAppend(false, f);
            }
            epaStatus = 0;
            nextsv = 0;
            if (det(wk->sv[s.c[0]].w - wk->sv[s.c[3]].w, wk->sv[s.c[1]].w - wk->sv[s.c[3]].w,
                    wk->sv[s.c[2]].w - wk->sv[s.c[3]].w) < 0) {
                uint8_t tc = s.c[0]; s.c[0] = s.c[1]; s.c[1] = tc;
                float tp = s.p[0]; s.p[0] = s.p[1]; s.p[1] = tp;
            }
            int16_t tetra[4];
            tetra[0] = newface(s.c[0], s.c[1], s.c[2], true);
            tetra[1] = newface(s.c[1], s.c[0], s.c[3], true);
            tetra[2] = newface(s.c[2], s.c[1], s.c[3], true);
            tetra[3] = newface(s.c[0], s.c[2], s.c[3], true);
            if (hullCount == 4) {
                int16_t best = findbest();
                EpaFace outer = wk->fc[best];
                uint8_t pass = 0;
                uint32_t iterations = 0;
                bind(tetra[0], 0, tetra[1], 0);
                bind(tetra[0], 1, tetra[2], 0);
                bind(tetra[0], 2, tetra[3], 0);
                bind(tetra[1], 1, tetra[3], 2);
                bind(tetra[1], 2, tetra[2], 1);
                bind(tetra[2], 2, tetra[3], 1);
                epaStatus = 0;
                for (; iterations < 255u; ++iterations) {
                    if (nextsv < (uint32_t)EPA_MAX_VERTICES) {
                        int16_t hcf = -1, hff = -1;
                        uint32_t hnf = 0;
                        int wIdx = 4 + (int)nextsv++;
                        bool valid = true;
                        wk->fc[best].pass = (uint8_t)(++pass);
                        getsupport(wk->fc[best].n, wk->sv[wIdx]);
                        float wdist = dot(wk->fc[best].n, wk->sv[wIdx].w) - wk->fc[best].d;
                        if (wdist > 0.0001f) {
                            for (uint32_t j = 0; (j < 3) && valid; ++j)
                                valid &= expand(pass, wIdx, (int16_t)wk->fc[best].f[j], wk->fc[best].e[j], hcf, hff, hnf);
                            if (overflow) return 9;
                            if (valid && (hnf >= 3)) {
                                bind(hcf, 1, hff, 2);
                                listRemove(true, best);
                                listAppend(false, best);
                                best = findbest();
                                outer = wk->fc[best];
                            } else {
                                epaStatus = 4;  // InvalidHull
                                break;
                            }
                        } else {
                            epaStatus = 7;  // AccuraryReached
                            break;
                        }
                    } else {
                        epaStatus = 6;  // OutOfVertices
                        break;
                    }
                }
                V3 projection = outer.n * outer.d;
                normal = outer.n;
                depth = outer.d;
                result.rank = 3;
                result.c[0] = outer.c[0];
                result.c[1] = outer.c[1];
                result.c[2] = outer.c[2];
                V3 w0 = wk->sv[outer.c[0]].w, w1 = wk->sv[outer.c[1]].w, w2 = wk->sv[outer.c[2]].w;
                result.p[0] = length(cross(w1 - projection, w2 - projection));
                result.p[1] = length(cross(w2 - projection, w0 - projection));
                result.p[2] = length(cross(w0 - projection, w1 - projection));
                float sum = (result.p[0] + result.p[1]) + result.p[2];
                result.p[0] /= sum;
                result.p[1] /= sum;
                result.p[2] /= sum;
                return epaStatus;
            }
        }
        epaStatus = 8;  // FallBack
        normal = -guess;
        float nl = length(normal);
        if (nl > 0) normal = bdiv(normal, nl);
        else normal = V3{1, 0, 0};
        depth = 0;
        result.rank = 1;
        result.c[0] = s.c[0];
        result.p[0] = 1;
        return epaStatus;
    }

    // gjkepa2_impl::Initialize
    RSB_HD void init(EpaWork* w, const ConvexShape& a, const Xf& wa, const ConvexShape& b, const Xf& wb, bool margins) {
        wk = w;
        shape.s0 = &a;
        shape.s1 = &b;
        shape.toShape1 = transposeTimes(wb.b, wa.b);
        shape.toShape0 = xfInverseTimes(wa, wb);
        shape.margins = margins;
        overflow = false;
    }
    // EPA::Initialize: every face starts in the stock list
    RSB_HD void initEpa() {
        epaStatus = 9;
        normal = v3zero();
        depth = 0;
        nextsv = 0;
        hullRoot = stockRoot = -1;
        hullCount = stockCount = 0;
        for (int i = 0; i < EPA_MAX_FACES; ++i) listAppend(false, (int16_t)(EPA_MAX_FACES - i - 1));
    }
};

// btGjkEpaSolver2::Penetration (usemargins = true); witnesses in world space
RSB_HD bool gjkEpaPenetration(EpaWork* wk, const ConvexShape& a, const Xf& wa, const ConvexShape& b, const Xf& wb, V3 guess,
                              V3& wA, V3& wB, V3& nrm, bool& overflow) {
    EpaSolver S;
    S.init(wk, a, wa, b, wb, true);
    int gs = S.gjkEvaluate(-guess);
    overflow = false;
    if (gs == 1) {
        S.initEpa();
        int es = S.epaEvaluate(-guess);
        if (S.overflow) { overflow = true; return false; }
        if (es != 9) {
            V3 w0 = v3zero();
            for (uint32_t i = 0; i < S.result.rank; ++i) w0 += S.shape.support0(wk->sv[S.result.c[i]].d) * S.result.p[i];
            wA = xfPoint(wa, w0);
            wB = xfPoint(wa, w0 - S.normal * S.depth);
            nrm = -S.normal;
            return true;
        }
    }
    return false;
}

// btGjkEpaSolver2::Distance (margins off)
RSB_HD bool gjkEpaDistance(EpaWork* wk, const ConvexShape& a, const Xf& wa, const ConvexShape& b, const Xf& wb, V3 guess,
                           V3& wA, V3& wB, V3& nrm) {
    EpaSolver S;
    S.init(wk, a, wa, b, wb, false);
    int gs = S.gjkEvaluate(guess);
    if (gs == 0) {
        V3 w0 = v3zero(), w1 = v3zero();
        EpaSimplex& sx = S.simplex();
        for (uint32_t i = 0; i < sx.rank; ++i) {
            float p = sx.p[i];
            w0 += S.shape.support0(wk->sv[sx.c[i]].d) * p;
            w1 += S.shape.support1(-wk->sv[sx.c[i]].d) * p;
        }
        wA = xfPoint(wa, w0);
        wB = xfPoint(wa, w1);
        nrm = w0 - w1;
        float dist = length(nrm);
        nrm = bdiv(nrm, dist > 0.0001f ? dist : 1.f);
        return true;
    }
    return false;
}

// btGjkEpaPenetrationDepthSolver::calcPenDepth
RSB_HD bool calcPenDepth(EpaWork* wk, const ConvexShape& a, const Xf& ta, const ConvexShape& b, const Xf& tb, V3& v,
                         V3& wA, V3& wB, bool& overflow) {
    V3 guesses[9] = {safeNormalized(tb.o - ta.o), safeNormalized(ta.o - tb.o), V3{0, 0, 1}, V3{0, 1, 0}, V3{1, 0, 0},
                     V3{1, 1, 0}, V3{1, 1, 1}, V3{0, 1, 1}, V3{1, 0, 1}};
    overflow = false;
    for (int i = 0; i < 9; i++) {
        V3 g = guesses[i];
        V3 nrm;
        if (gjkEpaPenetration(wk, a, ta, b, tb, g, wA, wB, nrm, overflow)) {
            v = nrm;
            return true;
        }
        if (overflow) return false;
        if (gjkEpaDistance(wk, a, ta, b, tb, g, wA, wB, nrm)) {
            v = nrm;
            return false;
        }
    }
    wA = wB = v = v3zero();
    return false;
}

// ------------------------------------------------------------------ GJK pair detector

struct GjkOut {
    bool has;
    V3 normal;   // normal on B
    V3 point;    // point on B (world)
    float dist;
    bool overflow;
};

RSB_HD GjkOut gjkPairDetector(EpaWork* wk, const ConvexShape& A, const Xf& trA, const ConvexShape& B, const Xf& trB,
                              float maxDist2) {
    GjkOut out;
    out.has = false;
    out.overflow = false;
    float distance = 0.f;
    V3 normalInB = v3zero();
    V3 pointOnA = v3zero(), pointOnB = v3zero();
    Xf lA = trA, lB = trB;
    V3 positionOffset = (lA.o + lB.o) * 0.5f;
    lA.o = lA.o - positionOffset;
    lB.o = lB.o - positionOffset;
    float marginA = A.margin, marginB = B.margin;
    int curIter = 0;
    const int gGjkMaxIter = 1000;
    V3 axis = V3{0, 1, 0};
    bool isValid = false, checkSimplex = false;
    int degenerate = 0;
    VoronoiSimplex ss;
    float squaredDistance = kLargeFloat;
    float delta = 0.f;
    float margin = marginA + marginB;
    ss.reset();
    while (true) {
        V3 sepA = tmul(-axis, trA.b);
        V3 sepB = tmul(axis, trB.b);
        V3 pInA = supportNoMargin(A, sepA);
        V3 qInB = supportNoMargin(B, sepB);
        V3 pWorld = xfPoint(lA, pInA);
        V3 qWorld = xfPoint(lB, qInB);
        V3 w = pWorld - qWorld;
        delta = dot(axis, w);
        if ((delta > 0.f) && (delta * delta > squaredDistance * maxDist2)) {
            degenerate = 10;
            checkSimplex = true;
            break;
        }
        if (ss.inSimplex(w)) {
            degenerate = 1;
            checkSimplex = true;
            break;
        }
        float f0 = squaredDistance - delta;
        float f1 = squaredDistance * 1.0e-6f;
        if (f0 <= f1) {
            degenerate = (f0 <= 0.f) ? 2 : 11;
            checkSimplex = true;
            break;
        }
        ss.addVertex(w, pWorld, qWorld);
        V3 newAxis;
        if (!ss.closest(newAxis)) {
            degenerate = 3;
            checkSimplex = true;
            break;
        }
        if (length2(newAxis) < 1.0e-6f) {
            axis = newAxis;
            degenerate = 6;
            checkSimplex = true;
            break;
        }
        float prev = squaredDistance;
        squaredDistance = length2(newAxis);
        if (prev - squaredDistance <= kEpsilon * prev) {
            checkSimplex = true;
            degenerate = 12;
            break;
        }
        axis = newAxis;
        if (curIter++ > gGjkMaxIter) break;
        if (ss.full()) {
            degenerate = 13;
            break;
        }
    }
    if (checkSimplex) {
        ss.computePoints(pointOnA, pointOnB);
        normalInB = axis;
        float lenSqr = length2(axis);
        if (lenSqr < 0.0001f) degenerate = 5;
        if (lenSqr > kEpsilon * kEpsilon) {
            float rlen = 1.f / fsqrt(lenSqr);
            normalInB *= rlen;
            float s = fsqrt(squaredDistance);
            pointOnA -= axis * (marginA / s);
            pointOnB += axis * (marginB / s);
            distance = (1.f / rlen) - margin;
            isValid = true;
        }
    }
    bool catchDegenerate = degenerate && ((distance + margin) < 0.01f);
    if (!isValid || catchDegenerate) {
        V3 tA, tB;
        axis = v3zero();
        bool ovf = false;
        bool valid2 = calcPenDepth(wk, A, lA, B, lB, axis, tA, tB, ovf);
        if (ovf) {
            out.overflow = true;
            return out;
        }
        if (valid2) {
            V3 tn = tB - tA;
            float l2 = length2(tn);
            if (l2 <= kEpsilon * kEpsilon) {
                tn = axis;
                l2 = length2(axis);
            }
            if (l2 > kEpsilon * kEpsilon) {
                tn = bdiv(tn, fsqrt(l2));
                float d2 = -length(tA - tB);
                if (!isValid || (d2 < distance)) {
                    distance = d2;
                    pointOnA = tA;
                    pointOnB = tB;
                    normalInB = tn;
                    isValid = true;
                }
            }
        } else {
            if (length2(axis) > 0.f) {
                float d2 = length(tA - tB) - margin;
                if (!isValid || (d2 < distance)) {
                    distance = d2;
                    pointOnA = tA;
                    pointOnB = tB;
                    pointOnA -= axis * marginA;
                    pointOnB += axis * marginB;
                    normalInB = normalized(axis);
                    isValid = true;
                }
            }
        }
    }
    if (isValid && ((distance < 0) || (distance * distance < maxDist2))) {
        V3 mn, mx;
        shapeAabb(A, lA, mn, mx);
        V3 posA = (mx + mn) * 0.5f;
        shapeAabb(B, lB, mn, mx);
        V3 posB = (mn + mx) * 0.5f;
        V3 diff = posA - posB;
        if (dot(diff, normalInB) < 0.f) normalInB *= -1.f;
        out.has = true;
        out.normal = normalInB;
        out.point = pointOnB + positionOffset;
        out.dist = distance;
    }
    return out;
}

// ------------------------------------------------------------------ ray vs convex

// btSubsimplexConvexCast for a ray (point shape A moving from -> to) against a static convex
// B at transform tB.  Returns true with the hit fraction and the (unnormalised-then-
// normalised) hit normal when the ray enters B.
RSB_HD bool subsimplexCast(V3 from, V3 to, const ConvexShape& B, const Xf& tB, float& fraction, V3& normal) {
    VoronoiSimplex ss;
    ss.reset();
    V3 linVelA = to - from;
    V3 linVelB = tB.o - tB.o;
    float lambda = 0.f;
    Xf iA{m3identity(), from};
    Xf iB = tB;
    V3 r = linVelA - linVelB;
    V3 supA = xfPoint(Xf{m3identity(), from}, v3zero());
    V3 supB = xfPoint(tB, supportVirtual(B, tmul(r, tB.b)));
    V3 v = supA - supB;
    int maxIter = 32;
    V3 n = v3zero();
    float dist2 = length2(v);
    V3 w;
    while ((dist2 > 0.0001f) && maxIter--) {
        supA = xfPoint(iA, v3zero());
        supB = xfPoint(iB, supportVirtual(B, tmul(v, iB.b)));
        w = supA - supB;
        float VdotW = dot(v, w);
        if (lambda > 1.f) return false;
        if (VdotW > 0.f) {
            float VdotR = dot(v, r);
            if (VdotR >= -(kEpsilon * kEpsilon)) return false;
            lambda = lambda - VdotW / VdotR;
            float s = 1.f - lambda;
            iA.o = from * s + to * lambda;
            iB.o = tB.o * s + tB.o * lambda;
            w = supA - supB;
            n = v;
        }
        if (!ss.inSimplex(w)) ss.addVertex(w, supA, supB);
        if (ss.closest(v)) dist2 = length2(v);
        else dist2 = 0.f;
    }
    fraction = lambda;
    if (length2(n) >= kEpsilon * kEpsilon) normal = normalized(n);
    else normal = v3zero();
    if (dot(normal, r) >= -0.f) return false;
    return true;
}

}  // namespace rsb
