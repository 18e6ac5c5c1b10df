// Per-arena body of the step kernel: load the arena's records from the word planes,
// run the requested ticks, store the records back.  The kernel in rsb_engine.cu calls
// stepArena() once per thread.
#pragma once
#include "arena.h"

namespace rsb {

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
    const void* controls;
};

RSB_HD void loadBall(const EngineView& D, int a, Body& b) {
    BallP p;
    loadPlanes(p, D.ball, a, D.N);
    b.xf = xfFromP(p.pos, p.rot);
    b.lin = V3{p.lin[0], p.lin[1], p.lin[2]};
    b.ang = V3{p.ang[0], p.ang[1], p.ang[2]};
    b.force = b.torque = v3zero();
    b.invMass = D.P.ballInvMass;
    b.grav = D.P.ballGrav;
    b.invIl = D.P.ballInvInertia;
    b.linDampFactor = D.P.ballLinDampFactor;
    b.friction = D.P.ballFriction;
    b.restitution = D.P.ballRestitution;
    b.noResp = 0;
    b.act = ACT_ACTIVE;
    b.solverId = -1;
    b.spCount = 0;
    b.spFric = b.spRest = b.spDist = 0.f;
    b.spNormal = v3zero();
    b.cell = p.cell;
    b.ci = p.ci;
    b.cj = p.cj;
    b.ck = p.ck;
    b.regStamp = p.regStamp;
    updateInertia(b);
    b.ixf = b.xf;
    b.bpMin = b.bpMax = b.xf.o;
}

RSB_HD void storeBall(const EngineView& D, int a, const Body& b) {
    BallP p;
    xfToP(b.xf, p.pos, p.rot);
    p.lin[0] = b.lin.x; p.lin[1] = b.lin.y; p.lin[2] = b.lin.z;
    p.ang[0] = b.ang.x; p.ang[1] = b.ang.y; p.ang[2] = b.ang.z;
    p.cell = b.cell;
    p.ci = b.ci;
    p.cj = b.cj;
    p.ck = b.ck;
    p.regStamp = b.regStamp;
    storePlanes(p, D.ball, a, D.N);
}

RSB_HD void stepArena(const EngineView& D, int a, int ticks, ArenaSim& A) {
    A.W.S = &D.S;
    A.W.P = &D.P;
    A.teamSize = D.teamSize[a];
    A.numCars = 2 * A.teamSize;
    A.W.nb = 1;
    A.W.status = 0;
    A.W.noRot[0] = 1;
    loadBall(D, a, A.W.b[0]);
    ArenaP ap;
    loadPlanes(ap, D.arena, a, D.N);
    A.tickCount = (uint64_t)ap.tick[0] | ((uint64_t)ap.tick[1] << 32);
    A.status = ap.status;
    for (int t = 0; t < ticks; t++) arenaTick(A);
    storeBall(D, a, A.W.b[0]);
    ap.tick[0] = (uint32_t)A.tickCount;
    ap.tick[1] = (uint32_t)(A.tickCount >> 32);
    ap.episodeTicks += ticks;
    ap.status = A.status;
    if (ballScored(A.W, D.P.goalBaseY, D.P.ballRadiusUu) && ap.goalTeam < 0) ap.goalTeam = A.W.b[0].xf.o.y > 0 ? 0 : 1;
    storePlanes(ap, D.arena, a, D.N);
}

}  // namespace rsb
