// Arena-level tick (RocketSim Arena::Step, Arena.cpp:716-812) around the Bullet world step.
#pragma once
#include "state.h"
#include "world.h"

namespace rsb {

struct ArenaSim {
    World W;
    int numCars;
    int teamSize;
    uint64_t tickCount;
    int32_t status;
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

RSB_HD void arenaTick(ArenaSim& A) {
    World& W = A.W;
    // ball zero-velocity sleeping (Arena.cpp:721-727)
    {
        Body& b = W.b[0];
        b.act = (length2(b.lin) == 0.f && length2(b.ang) == 0.f) ? ACT_SLEEPING : ACT_ACTIVE;
    }
    W.stampBase = (uint32_t)((A.tickCount + 1) * 8u);
    worldStep(W);
    ballFinishTick(W, v3zero());
    A.tickCount++;
    A.status |= (int32_t)W.status;
    W.status = 0;
}

}  // namespace rsb
