// Sequential-impulse contact solver (Bullet btSequentialImpulseConstraintSolver with the
// RocketSim changes), for one arena.
//
//   initSolverBody ............ btSequentialImpulseConstraintSolver.cpp:458-492
//   setupContactConstraint .... .cpp:795-983 (split impulse always on: threshold 1e30,
//                               erp2 = 0.8 set by Arena::Arena, Arena.cpp:485-488)
//   setupFrictionConstraint ... .cpp:517-607
//   convertContact(Inner) ..... .cpp:1003-1162, special-row aggregation .cpp:1048-1061
//   convertContactSpecial ..... .cpp:1164-1211 (one averaged ball-world row per body)
//   row kernels ............... the SSE2 variants (.cpp:149-340), selected by SOLVER_SIMD
//   iterations ................ .cpp:1601-1829 (10 split-impulse + 10 velocity iterations;
//                               special rows skipped in the velocity pass, .cpp:1730)
//   write-back ................ .cpp:1878-1904 and btSolverBody::writebackVelocityAndTransform
//
// Manifolds are rebuilt every tick (the RocketSim broadphase re-creates all pairs), so
// there is no warm-start impulse to carry between ticks.
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

struct SolverIn {
    float dt;
    int nBodies;
};

struct Solver {
    int nsb;
    SBody sb[MAX_BODIES + 1];
    int fixedId;
    int nc, nf;
    SRow c[MAX_CONTACT_ROWS];
    SRow f[MAX_FRICTION_ROWS];
};

constexpr float kErp2 = 0.8f, kSplitTurnErp = 0.1f, kRestVelThreshold = 0.2f;
constexpr int kNumIterations = 10;

RSB_HD void sbInitFixed(SBody& s) {
    s.xf = xfIdentity();
    s.invMassV = v3zero();
    s.lin = s.ang = s.extF = s.extT = s.dLin = s.dAng = s.push = s.turn = v3zero();
    s.body = -1;
}

RSB_HD void sbInitBody(SBody& s, const Body& b, int bi, float dt) {
    s.dLin = s.dAng = s.push = s.turn = v3zero();
    s.xf = b.xf;
    s.invMassV = V3{b.invMass, b.invMass, b.invMass};
    s.lin = b.lin;
    s.ang = b.ang;
    s.extF = (b.force * b.invMass) * dt;
    s.extT = tmul(b.torque, b.invIw) * dt;
    s.body = bi;
}

// getOrInitSolverBody for an object id: dynamic bodies map to their solver body,
// statics to the shared fixed body (created on first use).
RSB_HD int solverBodyOf(Solver& S, Body* bodies, int obj, float dt) {
    if (obj < OBJ_BALL) {
        if (S.fixedId < 0) {
            S.fixedId = S.nsb++;
            sbInitFixed(S.sb[S.fixedId]);
        }
        return S.fixedId;
    }
    Body& b = bodies[obj - OBJ_BALL];
    if (b.solverId >= 0) return b.solverId;
    int id = S.nsb++;
    sbInitBody(S.sb[id], b, obj - OBJ_BALL, dt);
    b.solverId = id;
    return id;
}

RSB_HD float restitutionCurve(float relVel, float restitution) {
    if (fabsf(relVel) < kRestVelThreshold) return 0.f;
    return restitution * -relVel;
}

// setupContactConstraint.  rb0/rb1 are null for the fixed body.
RSB_HD void setupContactRow(SRow& r, Solver& S, int sA, int sB, const Body* rb0, const Body* rb1,
                            V3 normal, float dist, float fric, float rest, V3 relPos1, V3 relPos2,
                            float dt, int special) {
    SBody& bodyA = S.sb[sA];
    SBody& bodyB = S.sb[sB];
    float invDt = 1.f / dt;
    float cfm = 0.f * invDt;
    V3 torqueAxis0 = cross(relPos1, normal);
    r.angA = rb0 ? rb0->invIw * torqueAxis0 : v3zero();
    V3 torqueAxis1 = cross(relPos2, normal);
    r.angB = rb1 ? rb1->invIw * (-torqueAxis1) : v3zero();
    float denom0 = 0.f, denom1 = 0.f;
    if (rb0) denom0 = rb0->invMass + dot(normal, cross(r.angA, relPos1));
    if (rb1) denom1 = rb1->invMass + dot(normal, cross(-r.angB, relPos2));
    r.jacInv = 1.f / (denom0 + denom1 + cfm);
    if (rb0) { r.n1 = normal; r.rc1 = torqueAxis0; } else { r.n1 = v3zero(); r.rc1 = v3zero(); }
    if (rb1) { r.n2 = -normal; r.rc2 = -torqueAxis1; } else { r.n2 = v3zero(); r.rc2 = v3zero(); }
    float penetration = dist + 0.f;
    V3 vel1 = rb0 ? rb0->lin + cross(rb0->ang, relPos1) : v3zero();
    V3 vel2 = rb1 ? rb1->lin + cross(rb1->ang, relPos2) : v3zero();
    float relVel = dot(normal, vel1 - vel2);
    r.friction = fric;
    float restitution = restitutionCurve(relVel, rest);
    if (restitution <= 0.f) restitution = 0.f;
    r.applied = 0.f;
    r.appliedPush = 0.f;
    V3 eFA = bodyA.body >= 0 ? bodyA.extF : v3zero();
    V3 eTA = bodyA.body >= 0 ? bodyA.extT : v3zero();
    V3 eFB = bodyB.body >= 0 ? bodyB.extF : v3zero();
    V3 eTB = bodyB.body >= 0 ? bodyB.extT : v3zero();
    float v1 = dot(r.n1, bodyA.lin + eFA) + dot(r.rc1, bodyA.ang + eTA);
    float v2 = dot(r.n2, bodyB.lin + eFB) + dot(r.rc2, bodyB.ang + eTB);
    float rel = v1 + v2;
    float velErr = restitution - rel;
    float posErr = (penetration > 0) ? 0.f : -penetration * kErp2 * invDt;
    r.rhsPen = posErr * r.jacInv;
    r.rhs = velErr * r.jacInv;
    r.cfm = cfm * r.jacInv;
    r.lo = 0.f;
    r.hi = 1e10f;
    r.special = (int16_t)special;
    r.bA = (int16_t)sA;
    r.bB = (int16_t)sB;
}

// setupFrictionConstraint.  b0/b1 are null for the fixed body.
RSB_HD void setupFrictionRow(SRow& r, Solver& S, int sA, int sB, const Body* b0, const Body* b1,
                             V3 axis, float fric, V3 relPos1, V3 relPos2) {
    SBody& sbA = S.sb[sA];
    SBody& sbB = S.sb[sB];
    r.bA = (int16_t)sA;
    r.bB = (int16_t)sB;
    r.friction = fric;
    r.applied = 0.f;
    r.appliedPush = 0.f;
    if (b0) {
        r.n1 = axis;
        V3 ft = cross(relPos1, r.n1);
        r.rc1 = ft;
        r.angA = b0->invIw * ft;
    } else {
        r.n1 = r.rc1 = r.angA = v3zero();
    }
    if (b1) {
        r.n2 = -axis;
        V3 ft = cross(relPos2, r.n2);
        r.rc2 = ft;
        r.angB = b1->invIw * ft;
    } else {
        r.n2 = r.rc2 = r.angB = v3zero();
    }
    float d0 = 0.f, d1 = 0.f;
    if (b0) d0 = b0->invMass + dot(axis, cross(r.angA, relPos1));
    if (b1) d1 = b1->invMass + dot(axis, cross(-r.angB, relPos2));
    r.jacInv = 1.f / (d0 + d1);
    float v1 = dot(r.n1, b0 ? sbA.lin + sbA.extF : v3zero()) + dot(r.rc1, b0 ? sbA.ang : v3zero());
    float v2 = dot(r.n2, b1 ? sbB.lin + sbB.extF : v3zero()) + dot(r.rc2, b1 ? sbB.ang : v3zero());
    float rel = v1 + v2;
    float velErr = 0.f - rel;
    float velImp = velErr * r.jacInv;
    r.rhs = 0.f + velImp;
    r.rhsPen = 0.f;
    r.cfm = 0.f;
    r.lo = -r.friction;
    r.hi = r.friction;
    r.special = 0;
}

RSB_HD void sbVelNoDelta(const SBody& s, V3 relPos, V3& v) {
    if (s.body >= 0) v = s.lin + s.extF + cross(s.ang + s.extT, relPos);
    else v = v3zero();
}

// convertContactInner (without rolling friction: every combined rolling friction is 0)
RSB_HD bool addFrictionFor(Solver& S, int contactRow, int sA, int sB, const Body* b0, const Body* b1,
                           V3 normal, float fric, V3 relPos1, V3 relPos2) {
    V3 vel1, vel2;
    sbVelNoDelta(S.sb[sA], relPos1, vel1);
    sbVelNoDelta(S.sb[sB], relPos2, vel2);
    V3 vel = vel1 - vel2;
    float relVel = dot(normal, vel);
    V3 lat1 = vel - normal * relVel;
    float latRel = length2(lat1);
    if (latRel > kEpsilon) {
        lat1 *= 1.f / fsqrt(latRel);
    } else {
        V3 lat2;
        planeSpace1(normal, lat1, lat2);
    }
    if (S.nf >= MAX_FRICTION_ROWS) return false;
    SRow& fr = S.f[S.nf];
    fr.fIdx = (int16_t)contactRow;
    setupFrictionRow(fr, S, sA, sB, b0, b1, lat1, fric, relPos1, relPos2);
    S.nf++;
    return true;
}

RSB_HD void applyImpulseDelta(SBody& s, V3 lin, V3 ang, float imp) {
    s.dLin = s.dLin + lin * imp;
    s.dAng = s.dAng + ang * imp;
}

// resolveSingleConstraintRowLowerLimit / Generic, SSE2 association
RSB_HD void solveRow(Solver& S, SRow& c, bool generic) {
    SBody& A = S.sb[c.bA];
    SBody& B = S.sb[c.bB];
    float applied0 = c.applied;
    float delta = c.rhs - c.applied * c.cfm;
    float d1 = dot_simd(c.n1, A.dLin) + dot_simd(c.rc1, A.dAng);
    float d2 = dot_simd(c.n2, B.dLin) + dot_simd(c.rc2, B.dAng);
    delta = delta - d1 * c.jacInv;
    delta = delta - d2 * c.jacInv;
    float sum = applied0 + delta;
    bool lowerLess = sum < c.lo;
    delta = lowerLess ? (c.lo - applied0) : delta;
    c.applied = lowerLess ? c.lo : sum;
    if (generic) {
        bool upperLess = sum < c.hi;
        delta = upperLess ? delta : (c.hi - applied0);
        c.applied = upperLess ? c.applied : c.hi;
    }
    if (A.body >= 0) applyImpulseDelta(A, c.n1 * A.invMassV, c.angA, delta);
    if (B.body >= 0) applyImpulseDelta(B, c.n2 * B.invMassV, c.angB, delta);
}

// resolveSplitPenetrationImpulse (SSE2); returns true when it changed anything
RSB_HD bool solveSplitRow(Solver& S, SRow& c) {
    if (c.rhsPen == 0.f) return false;
    SBody& A = S.sb[c.bA];
    SBody& B = S.sb[c.bB];
    float applied0 = c.appliedPush;
    float delta = c.rhsPen - c.appliedPush * c.cfm;
    float d1 = dot_simd(c.n1, A.push) + dot_simd(c.rc1, A.turn);
    float d2 = dot_simd(c.n2, B.push) + dot_simd(c.rc2, B.turn);
    delta = delta - d1 * c.jacInv;
    delta = delta - d2 * c.jacInv;
    float sum = applied0 + delta;
    bool lowerLess = sum < c.lo;
    delta = lowerLess ? (c.lo - applied0) : delta;
    c.appliedPush = lowerLess ? c.lo : sum;
    if (A.body >= 0) {
        A.push = A.push + (c.n1 * A.invMassV) * delta;
        A.turn = A.turn + c.angA * delta;
    }
    if (B.body >= 0) {
        B.push = B.push + (c.n2 * B.invMassV) * delta;
        B.turn = B.turn + c.angB * delta;
    }
    return delta != 0.f;
}

RSB_HD void solverIterate(Solver& S) {
    for (int it = 0; it < kNumIterations; it++) {
        bool any = false;
        for (int j = 0; j < S.nc; j++) any |= solveSplitRow(S, S.c[j]);
        if (!any || it >= kNumIterations - 1) break;
    }
    for (int it = 0; it < kNumIterations; it++) {
        for (int j = 0; j < S.nc; j++) {
            if (S.c[j].special) continue;
            solveRow(S, S.c[j], false);
        }
        for (int j = 0; j < S.nf; j++) {
            SRow& fr = S.f[j];
            float total = S.c[fr.fIdx].applied;
            if (total > 0.f) {
                fr.lo = -(fr.friction * total);
                fr.hi = fr.friction * total;
                solveRow(S, fr, true);
            }
        }
    }
}

// writeBackBodies with split-impulse position correction
RSB_HD void solverWriteBack(Solver& S, Body* bodies, const int* noRot, float dt) {
    for (int i = 0; i < S.nsb; i++) {
        SBody& s = S.sb[i];
        if (s.body < 0) continue;
        Body& b = bodies[s.body];
        s.lin = s.lin + s.dLin;
        s.ang = s.ang + s.dAng;
        if (s.push.x != 0.f || s.push.y != 0 || s.push.z != 0 || s.turn.x != 0.f || s.turn.y != 0 || s.turn.z != 0) {
            if (noRot[s.body]) s.xf = integrateTransformNoRot(s.xf, s.push, dt);
            else s.xf = integrateTransform(s.xf, s.push, s.turn * kSplitTurnErp, dt);
        }
        b.lin = s.lin + s.extF;
        b.ang = s.ang + s.extT;
        b.xf = s.xf;
        b.solverId = -1;
    }
}

}  // namespace rsb
