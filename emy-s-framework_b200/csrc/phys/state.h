// Persistent arena state as it lives in device memory between kernel launches.
//
// Every record is a sequence of 32-bit words.  Records are stored word-plane-major
// ("structure of arrays"): word w of arena a sits at planes[w * N + a], and car slot s
// of arena a at planes[(w * MAX_CARS + s) * N + a].  A kernel thread that owns arena a
// therefore reads and writes each word with a warp-coalesced access.
//
// Kinematics are kept in Bullet units (the reference's internal representation) so that
// a state carried across launches is bit-identical to one carried across ticks; the C ABI
// converts to Unreal units at the boundary, as RocketSim's Get/SetState do.
#pragma once
#include "world_types.h"

namespace rsb {

struct BallP {
    float pos[3];
    float rot[9];   // basis rows
    float lin[3];
    float ang[3];
    int32_t cell, ci, cj, ck;
    uint32_t regStamp;
};

struct CarP {
    float pos[3];
    float rot[9];
    float lin[3];
    float ang[3];
    int32_t cell, ci, cj, ck;
    uint32_t regStamp;
    // RocketSim CarState (Car.h:15-100)
    float boost, timeSpentBoosting, jumpTime, flipTime, airTime, airTimeSinceJump;
    float supersonicTime, handbrakeVal, autoFlipTimer, autoFlipTorqueScale;
    float demoRespawnTimer, carContactCooldown;
    float flipRelTorque[3];
    float worldContactNormal[3];
    uint32_t carContactOtherId;
    uint32_t flags;
    uint32_t ballHitTick[2];       // lo, hi
    uint32_t ballHitExtraTick[2];
    float ballHitRelPos[3], ballHitBallPos[3], ballHitExtraVel[3];
    float rotMat[9];               // CarState::rotMat (differs from rot only while demoed)
    // controls of the previous tick (CarState::lastControls)
    float lastCtl[5];
    uint32_t lastCtlBits;
    // btWheelInfoRL values carried from one tick to the next
    float steerAngle;              // front wheels (rear wheels never steer)
    float engineForce, brake;      // same on all four wheels
    float latFriction[4], longFriction[4], extraPushback[4];
};

struct PadP {
    float cooldown;
    uint32_t bits;   // isActive | prevLockedCarId << 8
};

struct ArenaP {
    uint32_t tick[2];     // tickCount lo, hi
    int32_t episodeTicks;
    int32_t status;
    int32_t goalTeam;     // -1, 0 blue scored, 1 orange scored (latched since the last reset)
    int32_t touchedMask;  // cars that touched the ball in the current env step
    float noTouchTimer;
    int32_t scored;       // ball past a goal line after the last tick (Arena::IsBallScored)
};

constexpr int W_BALL = sizeof(BallP) / 4;
constexpr int W_CAR = sizeof(CarP) / 4;
constexpr int W_PAD = sizeof(PadP) / 4;
constexpr int W_ARENA = sizeof(ArenaP) / 4;
static_assert(sizeof(BallP) % 4 == 0 && sizeof(CarP) % 4 == 0, "word records");

// Records are staged through a word array and memcpy: accessing a float record through
// a uint32_t pointer would break the aliasing rules the optimisers rely on.
template <class T>
RSB_HD void loadPlanes(T& rec, const uint32_t* planes, int idx, int stride) {
    uint32_t w[sizeof(T) / 4];
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 4); i++) w[i] = planes[(size_t)i * stride + idx];
    memcpy(&rec, w, sizeof(T));
}

template <class T>
RSB_HD void storePlanes(const T& rec, uint32_t* planes, int idx, int stride) {
    uint32_t w[sizeof(T) / 4];
    memcpy(w, &rec, sizeof(T));
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 4); i++) planes[(size_t)i * stride + idx] = w[i];
}

RSB_HD Xf xfFromP(const float* pos, const float* rot) {
    return Xf{m3(rot[0], rot[1], rot[2], rot[3], rot[4], rot[5], rot[6], rot[7], rot[8]), V3{pos[0], pos[1], pos[2]}};
}
RSB_HD void xfToP(const Xf& x, float* pos, float* rot) {
    pos[0] = x.o.x; pos[1] = x.o.y; pos[2] = x.o.z;
    for (int i = 0; i < 3; i++) {
        rot[3 * i + 0] = x.b.r[i].x;
        rot[3 * i + 1] = x.b.r[i].y;
        rot[3 * i + 2] = x.b.r[i].z;
    }
}

}  // namespace rsb
