// Per-arena body of the step kernel: load the arena's records from the word planes,
// run the requested ticks, store the records back.  The kernel in rsb_engine.cu calls
// stepArena() once per arena.
#pragma once
#include "arena.h"

namespace rsb {

// Controls of one car as the C ABI passes them (rsb_controls, 24 bytes)
struct CtlRec {
    float v[5];
    uint8_t jump, boost, handbrake, pad_;
};

struct EngineView {
    ArenaStatic S;
    WorldParams P;
    int N;
    const int32_t* teamSize;
    const int32_t* carOffset;
    uint32_t* ball;
    uint32_t* car;
    uint32_t* pad;
    uint32_t* arena;
    const CtlRec* controls;
    uint32_t seed;
    const uint32_t* cull;          // per-arena body bits from the learned culler, or null
    int32_t cullAudit;             // run culled static tests anyway and count what they find
    unsigned long long* counters;  // [static tests run, tests culled, culled tests that hit, solver rows], or null
    unsigned int* work;            // next unclaimed arena of a persistent launch (zeroed before it)
};

RSB_HD void initBodyCommon(Body& b) {
    b.force = b.torque = v3zero();
    b.noResp = 0;
    b.act = ACT_ACTIVE;
    b.solverId = -1;
    b.spCount = 0;
    b.spFric = b.spRest = b.spDist = 0.f;
    b.spNormal = v3zero();
}

RSB_HD void ballBodyOf(const EngineView& D, const BallP& p, Body& b) {
    b.xf = xfFromP(p.pos, p.rot);
    b.lin = V3{p.lin[0], p.lin[1], p.lin[2]};
    b.ang = V3{p.ang[0], p.ang[1], p.ang[2]};
    initBodyCommon(b);
    b.invMass = D.P.ballInvMass;
    b.grav = D.P.ballGrav;
    b.invIl = D.P.ballInvInertia;
    b.linDampFactor = D.P.ballLinDampFactor;
    b.friction = D.P.ballFriction;
    b.restitution = D.P.ballRestitution;
    b.cell = p.cell;
    b.ci = p.ci;
    b.cj = p.cj;
    b.ck = p.ck;
    b.regStamp = p.regStamp;
    updateInertia(b);
    b.ixf = b.xf;
    b.bpMin = b.bpMax = b.xf.o;
}

RSB_HD void loadBall(const EngineView& D, int a, Body& b) {
    BallP p;
    loadPlanes(p, D.ball, a, D.N);
    ballBodyOf(D, p, b);
}

RSB_HD BallP ballRecordOf(const Body& b) {
    BallP p;
    xfToP(b.xf, p.pos, p.rot);
    p.lin[0] = b.lin.x; p.lin[1] = b.lin.y; p.lin[2] = b.lin.z;
    p.ang[0] = b.ang.x; p.ang[1] = b.ang.y; p.ang[2] = b.ang.z;
    p.cell = b.cell;
    p.ci = b.ci;
    p.cj = b.cj;
    p.ck = b.ck;
    p.regStamp = b.regStamp;
    return p;
}

RSB_HD void storeBall(const EngineView& D, int a, const Body& b) {
    BallP p = ballRecordOf(b);
    storePlanes(p, D.ball, a, D.N);
}

RSB_HD V3 v3of(const float* f) { return V3{f[0], f[1], f[2]}; }
RSB_HD void putV3(float* f, V3 v) { f[0] = v.x; f[1] = v.y; f[2] = v.z; }

RSB_HD void loadCar(const EngineView& D, int a, int s, Body& b, CarSim& c) {
    const CarParams& C = D.P.car;
    CarP p;
    loadPlanes(p, D.car, s * D.N + a, MAX_CARS * D.N);
    b.xf = xfFromP(p.pos, p.rot);
    b.lin = v3of(p.lin);
    b.ang = v3of(p.ang);
    initBodyCommon(b);
    b.noResp = (p.flags & CF_NO_RESPONSE) ? 1 : 0;
    b.invMass = C.invMass;
    b.grav = C.grav;
    b.invIl = C.invInertiaLocal;
    b.linDampFactor = 1.f;
    b.friction = CAR_COLLISION_FRICTION;
    b.restitution = CAR_COLLISION_RESTITUTION;
    b.cell = p.cell;
    b.ci = p.ci;
    b.cj = p.cj;
    b.ck = p.ck;
    b.regStamp = p.regStamp;
    updateInertia(b);
    b.ixf = b.xf;
    b.bpMin = b.bpMax = b.xf.o;

    c.boost = p.boost;
    c.timeSpentBoosting = p.timeSpentBoosting;
    c.jumpTime = p.jumpTime;
    c.flipTime = p.flipTime;
    c.airTime = p.airTime;
    c.airTimeSinceJump = p.airTimeSinceJump;
    c.supersonicTime = p.supersonicTime;
    c.handbrakeVal = p.handbrakeVal;
    c.autoFlipTimer = p.autoFlipTimer;
    c.autoFlipTorqueScale = p.autoFlipTorqueScale;
    c.demoRespawnTimer = p.demoRespawnTimer;
    c.carContactCooldown = p.carContactCooldown;
    c.flipRelTorque = v3of(p.flipRelTorque);
    c.worldContactNormal = v3of(p.worldContactNormal);
    c.carContactOtherId = p.carContactOtherId;
    c.flags = p.flags;
    c.ballHitTick = (uint64_t)p.ballHitTick[0] | ((uint64_t)p.ballHitTick[1] << 32);
    c.ballHitExtraTick = (uint64_t)p.ballHitExtraTick[0] | ((uint64_t)p.ballHitExtraTick[1] << 32);
    c.ballHitRelPos = v3of(p.ballHitRelPos);
    c.ballHitBallPos = v3of(p.ballHitBallPos);
    c.ballHitExtraVel = v3of(p.ballHitExtraVel);
    c.rotMat = m3(p.rotMat[0], p.rotMat[1], p.rotMat[2], p.rotMat[3], p.rotMat[4], p.rotMat[5], p.rotMat[6], p.rotMat[7], p.rotMat[8]);
    for (int k = 0; k < 5; k++) c.lastCtl[k] = p.lastCtl[k];
    c.lastCtlBits = p.lastCtlBits;
    c.steerAngle = p.steerAngle;
    c.engineForce = p.engineForce;
    c.brake = p.brake;
    for (int i = 0; i < 4; i++) {
        c.latF[i] = p.latFriction[i];
        c.longF[i] = p.longFriction[i];
        c.extraPush[i] = p.extraPushback[i];
    }
    c.velCache = v3zero();
    c.team = (p.flags & CF_TEAM_ORANGE) ? 1 : 0;
    c.id = (uint32_t)s + 1u;
    const CtlRec& ctl = D.controls[D.carOffset[a] + s];
    for (int k = 0; k < 5; k++) c.ctl[k] = ctl.v[k];
    c.ctlBits = (ctl.jump ? 1u : 0u) | (ctl.boost ? 2u : 0u) | (ctl.handbrake ? 4u : 0u);
}

RSB_HD void storeCar(const EngineView& D, int a, int s, const Body& b, const CarSim& c) {
    CarP p;
    xfToP(b.xf, p.pos, p.rot);
    putV3(p.lin, b.lin);
    putV3(p.ang, b.ang);
    p.cell = b.cell;
    p.ci = b.ci;
    p.cj = b.cj;
    p.ck = b.ck;
    p.regStamp = b.regStamp;
    p.boost = c.boost;
    p.timeSpentBoosting = c.timeSpentBoosting;
    p.jumpTime = c.jumpTime;
    p.flipTime = c.flipTime;
    p.airTime = c.airTime;
    p.airTimeSinceJump = c.airTimeSinceJump;
    p.supersonicTime = c.supersonicTime;
    p.handbrakeVal = c.handbrakeVal;
    p.autoFlipTimer = c.autoFlipTimer;
    p.autoFlipTorqueScale = c.autoFlipTorqueScale;
    p.demoRespawnTimer = c.demoRespawnTimer;
    p.carContactCooldown = c.carContactCooldown;
    putV3(p.flipRelTorque, c.flipRelTorque);
    putV3(p.worldContactNormal, c.worldContactNormal);
    p.carContactOtherId = c.carContactOtherId;
    p.flags = (c.flags & ~CF_NO_RESPONSE) | (b.noResp ? CF_NO_RESPONSE : 0u);
    p.ballHitTick[0] = (uint32_t)c.ballHitTick;
    p.ballHitTick[1] = (uint32_t)(c.ballHitTick >> 32);
    p.ballHitExtraTick[0] = (uint32_t)c.ballHitExtraTick;
    p.ballHitExtraTick[1] = (uint32_t)(c.ballHitExtraTick >> 32);
    putV3(p.ballHitRelPos, c.ballHitRelPos);
    putV3(p.ballHitBallPos, c.ballHitBallPos);
    putV3(p.ballHitExtraVel, c.ballHitExtraVel);
    for (int i = 0; i < 3; i++) {
        p.rotMat[3 * i + 0] = c.rotMat.r[i].x;
        p.rotMat[3 * i + 1] = c.rotMat.r[i].y;
        p.rotMat[3 * i + 2] = c.rotMat.r[i].z;
    }
    for (int k = 0; k < 5; k++) p.lastCtl[k] = c.lastCtl[k];
    p.lastCtlBits = c.lastCtlBits;
    p.steerAngle = c.steerAngle;
    p.engineForce = c.engineForce;
    p.brake = c.brake;
    for (int i = 0; i < 4; i++) {
        p.latFriction[i] = c.latF[i];
        p.longFriction[i] = c.longF[i];
        p.extraPushback[i] = c.extraPush[i];
    }
    storePlanes(p, D.car, s * D.N + a, MAX_CARS * D.N);
}

RSB_HD void stepArena(const EngineView& D, int a, int ticks, ArenaSim& A) {
    World& W = A.W;
    W.S = &D.S;
    W.P = &D.P;
    A.teamSize = D.teamSize[a];
    A.numCars = 2 * A.teamSize;
    W.nc = A.numCars;
    W.nb = 1 + A.numCars;
    W.status = 0;
    W.noRot[0] = 1;
    loadBall(D, a, W.b[0]);
    for (int s = 0; s < A.numCars; s++) {
        W.noRot[1 + s] = 0;
        loadCar(D, a, s, W.b[1 + s], W.c[s]);
    }
    for (int p = 0; p < NUM_PADS; p++) {
        PadP pp;
        loadPlanes(pp, D.pad, p * D.N + a, NUM_PADS * D.N);
        A.pads[p].cooldown = pp.cooldown;
        A.pads[p].isActive = pp.bits & 1u;
        A.pads[p].prevLocked = pp.bits >> 8;
        A.pads[p].curLocked = -1;
    }
    ArenaP ap;
    loadPlanes(ap, D.arena, a, D.N);
    A.tickCount = (uint64_t)ap.tick[0] | ((uint64_t)ap.tick[1] << 32);
    A.status = ap.status;
    A.goalTeam = ap.goalTeam;
    A.touchedMask = (uint32_t)ap.touchedMask;
    A.rngKey = mixHash(D.seed, (uint32_t)a, 0x5EEDu);
    W.cull = D.cull ? D.cull[a] : 0u;
    W.cullAudit = D.cullAudit;
    W.nStatic = W.nCulled = W.nMissed = 0;
    W.cullMissed = 0;
    W.nRows = 0;
    for (int t = 0; t < ticks; t++) arenaTick(A);
#if defined(__CUDA_ARCH__)
    if (D.counters) {
        atomicAdd(&D.counters[0], (unsigned long long)W.nStatic);
        atomicAdd(&D.counters[1], (unsigned long long)W.nCulled);
        if (W.nMissed) atomicAdd(&D.counters[2], (unsigned long long)W.nMissed);
        atomicAdd(&D.counters[3], (unsigned long long)W.nRows);
    }
#endif
    storeBall(D, a, W.b[0]);
    for (int s = 0; s < A.numCars; s++) storeCar(D, a, s, W.b[1 + s], W.c[s]);
    for (int p = 0; p < NUM_PADS; p++) {
        PadP pp;
        pp.cooldown = A.pads[p].cooldown;
        pp.bits = (A.pads[p].isActive & 1u) | (A.pads[p].prevLocked << 8);
        storePlanes(pp, D.pad, p * D.N + a, NUM_PADS * D.N);
    }
    ap.tick[0] = (uint32_t)A.tickCount;
    ap.tick[1] = (uint32_t)(A.tickCount >> 32);
    ap.episodeTicks += ticks;
    ap.status = A.status;
    ap.goalTeam = A.goalTeam;
    ap.touchedMask = (int32_t)A.touchedMask;
    ap.scored = ballScored(W, D.P.goalBaseY, D.P.ballRadiusUu) ? (W.b[0].xf.o.y > 0 ? 1 : 2) : 0;
    storePlanes(ap, D.arena, a, D.N);
}

}  // namespace rsb
