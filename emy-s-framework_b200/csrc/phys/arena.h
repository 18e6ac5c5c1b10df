// Arena-level tick (RocketSim Arena::Step, Arena.cpp:716-812) around the Bullet world step:
// car pre-tick updates, boost pad timers, the world step, car post-tick updates with the
// boost pad pickups (BoostPad.cpp:37-105, BoostPadGrid.cpp:5-24), the ball's finish tick.
#pragma once
#include "state.h"
#include "car.h"

namespace rsb {

struct PadSim {
    float cooldown;
    uint32_t isActive;
    uint32_t prevLocked;   // car id, 0 none
    int32_t curLocked;     // car index locked this tick, -1 none
};

struct ArenaSim {
    World W;
    int numCars;
    int teamSize;
    uint64_t tickCount;
    int32_t status;
    int32_t goalTeam;
    uint32_t touchedMask;
    uint32_t rngKey;       // per-arena key of the demo respawn draws
    PadSim pads[NUM_PADS];
};

RSB_HD void ballFinishTick(World& W, V3 velCache) {
    Body& b = W.b[0];
    if (!isZero(velCache)) b.lin = b.lin + velCache;
    float ms = W.P->ballMaxSpeedBt;
    V3 v = b.lin, w = b.ang;
    if (length2(v) > ms * ms) v = normalized(v) * ms;
    if (length2(w) > BALL_MAX_ANG_SPEED * BALL_MAX_ANG_SPEED) w = normalized(w) * BALL_MAX_ANG_SPEED;
    b.lin = v;
    b.ang = w;
}

// Arena::IsBallScored for soccar (Arena.cpp:949-957): the ball centre past a goal line.
RSB_HD bool ballScored(const World& W, float goalBaseY, float ballRadiusUu) {
    float y = W.b[0].xf.o.y * kBtToUu;
    return fabsf(y) > (goalBaseY + ballRadiusUu);
}

// counter-based hash for the respawn location draws
RSB_HD uint32_t mixHash(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u ^ (c + 0x165667B1u) * 0xC2B2AE3Du;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    return h;
}

// BoostPad::_CheckCollide for one car
RSB_HD void padCheckCollide(ArenaSim& A, int p, int ci) {
    const World& W = A.W;
    const Body& cb = W.b[1 + ci];
    PadSim& pad = A.pads[p];
    bool big = p < NUM_BIG_PADS;
    PadLoc pl = padLoc(p);
    V3 posBT = V3{pl.x, pl.y, pl.z} * kUuToBt;
    V3 carPos = cb.xf.o;
    bool colliding = false;
    if (pad.prevLocked == W.c[ci].id) {
        V3 mn, mx;
        carCompoundAabb(W.P->car, cb.xf, mn, mx);
        float boxRad = (big ? PAD_BOX_RAD_BIG : PAD_BOX_RAD_SMALL) * kUuToBt;
        V3 boxMin = posBT - V3{boxRad, boxRad, 0};
        V3 boxMax = posBT + V3{boxRad, boxRad, PAD_BOX_HEIGHT * kUuToBt};
        colliding = (boxMax.x > mn.x && boxMax.y > mn.y && boxMax.z > mn.z) && (boxMin.x < mx.x && boxMin.y < mx.y && boxMin.z < mx.z);
    } else {
        float rad = (big ? PAD_CYL_RAD_BIG : PAD_CYL_RAD_SMALL) * kUuToBt;
        float dx = carPos.x - posBT.x, dy = carPos.y - posBT.y;
        if (dx * dx + dy * dy < rad * rad) colliding = fabsf(carPos.z - posBT.z) < PAD_CYL_HEIGHT * kUuToBt;
    }
    if (colliding) pad.curLocked = ci;
}

// BoostPadGrid::CheckCollision
RSB_HD void padGridCheck(ArenaSim& A, int ci) {
    const CarSim& c = A.W.c[ci];
    if ((c.flags & CF_DEMOED) || c.boost >= 100) return;
    V3 carPos = A.W.b[1 + ci].xf.o * kBtToUu;
    if (carPos.z > PAD_CYL_HEIGHT + 250.f) return;
    int ix = (int)(carPos.x / 1024.f + 4.f);
    int iy = (int)(carPos.y / 1024.f + 5.f);
    for (int i = imax_(ix - 1, 0); i <= imin_(ix + 1, 7); i++)
        for (int j = imax_(iy - 1, 0); j <= imin_(iy + 1, 9); j++) {
            int p = A.W.P->padGrid[i * 10 + j];
            if (p >= 0) padCheckCollide(A, p, ci);
        }
}

RSB_HD void arenaTick(ArenaSim& A) {
    World& W = A.W;
    const float dt = W.P->dt;
    const CarParams& C = W.P->car;
    W.tick = A.tickCount;
    // ball zero-velocity sleeping (Arena.cpp:721-727)
    {
        Body& b = W.b[0];
        b.act = (length2(b.lin) == 0.f && length2(b.ang) == 0.f) ? ACT_SLEEPING : ACT_ACTIVE;
    }
    bool ballOnly = W.nc == 0;
    // Arena::_cars is an unordered_set of car pointers: with each car in its own hash
    // bucket, libstdc++ iterates it in reverse insertion order
    buildRayOrder(W);  // the wheel rays walk the cell proxies in registration order
    for (int ci = W.nc - 1; ci >= 0; ci--) carPreTick(W, ci, mixHash(A.rngKey, (uint32_t)A.tickCount, (uint32_t)ci));
    if (!ballOnly) {
        for (int p = 0; p < NUM_PADS; p++) {
            PadSim& pad = A.pads[p];
            if (pad.cooldown > 0) pad.cooldown = fmax_(pad.cooldown - dt, 0);
            pad.isActive = pad.cooldown == 0;
            pad.curLocked = -1;
        }
    }
    W.stampBase = (uint32_t)((A.tickCount + 1) * 8u);
    W.ballVelCache = v3zero();
    worldStep(W);
    for (int ci = W.nc - 1; ci >= 0; ci--) {
        carPostTick(W, ci);
        padGridCheck(A, ci);
        if (W.c[ci].ballHitTick == A.tickCount) A.touchedMask |= 1u << ci;
    }
    if (!ballOnly) {
        for (int p = 0; p < NUM_PADS; p++) {
            PadSim& pad = A.pads[p];
            uint32_t locked = 0;
            if (pad.curLocked >= 0) {
                CarSim& c = W.c[pad.curLocked];
                locked = c.id;
                if (pad.isActive) {
                    float add = p < NUM_BIG_PADS ? PAD_BOOST_AMOUNT_BIG : PAD_BOOST_AMOUNT_SMALL;
                    c.boost = fmin_(c.boost + add, BOOST_MAX);
                    pad.isActive = 0;
                    pad.cooldown = p < NUM_BIG_PADS ? C.padCooldownBig : C.padCooldownSmall;
                }
            }
            pad.prevLocked = locked;
        }
    }
    ballFinishTick(W, W.ballVelCache);
    if (A.goalTeam < 0 && ballScored(W, W.P->goalBaseY, W.P->ballRadiusUu)) A.goalTeam = W.b[0].xf.o.y > 0 ? 0 : 1;
    A.tickCount++;
    A.status |= (int32_t)(W.status | W.cullMissed);
    W.status = 0;
}

}  // namespace rsb
