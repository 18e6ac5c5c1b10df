// VantaObs v3.5 rows (366 floats per player) on the device, with the builder's per-arena and
// per-player state: boost-pad timers, demo timers and the "coyote" action timers.
//
// The row is the reference's (RocketSimCuda/src/VantaObsGpu.cuh:342-748, a transcription of
// RLGymCPP's VantaObs): ego 81, ball 29 (three ball-prediction slices at 1 / 2 / 3 s),
// goal context 16, team context 6, 2 teammates and 3 opponents of 39 each sorted by distance to
// the ball, a 5-slot validity mask, 34 boost pads.  Everything is in the player's canonical
// frame: the orange team's frame (InvertPhys), then mirrored in x when the player is on the
// negative-x side.  The float expressions follow the reference's order (three-term dot
// products, a vector divided by a length through one reciprocal, IEEE divisions by the
// normalisers), so that the rows are bit-identical on identical state.
//
// Two kernels per build, where the reference does the same two steps
// (RocketSimCudaObs.cuh:70-186):
//   vantaArenaKernel .. one thread per arena: pad availability and timers, demo timers, and
//                       each player's coyote timers (once per arena tick);
//   vantaRowKernel .... one thread per player: the row, staged a section at a time in shared
//                       memory and written by the warp into the packed [num_cars][366]
//                       buffer (rows in creation-slot order).
#pragma once
#include "env_kernels.cuh"

namespace rsb {

constexpr int VANTA_ROW = 366;
constexpr float VA_POS_STD = 2300.f, VA_VEL_STD = 2300.f, VA_BALL_VEL_STD = 6000.f, VA_ANG_STD = 5.5f;
constexpr float VA_DEMO_STD = 3.f, VA_GOAL_COEF = 1.f / 10240.f;
constexpr int CW_LASTCTL = (int)(offsetof(CarP, lastCtl) / 4), CW_LASTCTLBITS = (int)(offsetof(CarP, lastCtlBits) / 4);
constexpr int CW_HANDBRAKE = (int)(offsetof(CarP, handbrakeVal) / 4);

// Per-arena words (planes [word][N]): pad timers (RLGym pad order), availability bits,
// flags (bit 0: initialised), the arena tick of the last update (lo, hi).
constexpr int VA_TIMER = 0, VA_AVAIL = NUM_PADS, VA_FLAGS = NUM_PADS + 2, VA_TICK = NUM_PADS + 3;
constexpr int VA_WORDS = NUM_PADS + 5;
// Per-car words (planes [word][MAX_CARS][N]).
enum : int {
    VT_BOOST = 0, VT_BOOST_HOLD, VT_JUMP, VT_FLIP, VT_AIR, VT_HANDBRAKE, VT_DEMO,
    VT_FLIPDIR,              // 3 words
    VT_FLAGS = VT_FLIPDIR + 3,
    VT_TICK,                 // 2 words
    VT_WORDS = VT_TICK + 2
};
static_assert(VA_WORDS == VANTA_ARENA_WORDS && VT_WORDS == VANTA_CAR_WORDS, "builder state sizes");
enum : uint32_t {
    VF_JUMPING = 1, VF_JUMPED = 2, VF_DOUBLE = 4, VF_FLIPPED = 8, VF_ON_GROUND = 16, VF_WAS_DEMOED = 32,
    VF_INIT = 64, VF_PREV_JUMP = 128
};

// Pad tables in RLGym order: location (z 73 big / 70 small, as the reference's pad table),
// the engine's pad index, and the x-mirror permutation.
struct VantaTables {
    float x[NUM_PADS], y[NUM_PADS], z[NUM_PADS];
    uint8_t pad[NUM_PADS], mirror[NUM_PADS];
};

struct VantaView {
    uint32_t* arena;             // VA_WORDS planes
    uint32_t* car;               // VT_WORDS planes
    const rsb_ball_state* pred;  // [N][3] slices at 120 / 240 / 360 ticks, or null
    float* rows;                 // [num_cars][VANTA_ROW]
    float dt;                    // tickSkip / 120
    float deadzone;
    int onlyClosestOpp;
};

struct VV {
    float x, y, z;
};
RSB_D VV vv(float x, float y, float z) { return VV{x, y, z}; }
RSB_D VV vsub(VV a, VV b) { return VV{a.x - b.x, a.y - b.y, a.z - b.z}; }
RSB_D float vdot(VV a, VV b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RSB_D float vlen(VV a) { return sqrtf(vdot(a, a)); }
RSB_D VV vdiv(VV a, float s) {  // through one reciprocal, as the reference's Vec3 / float
    const float r = 1.f / s;
    return VV{a.x * r, a.y * r, a.z * r};
}
RSB_D VV vunit(VV a) {
    const float l = vlen(a);
    return l > 1e-6f ? vdiv(a, l) : VV{0.f, 0.f, 0.f};
}

// A body in a player's canonical frame.
struct VBody {
    VV pos, vel, ang, fwd, right, up;
};
RSB_D VBody canonical(VBody b, bool inv, bool mirror) {
    if (inv) {
        VV* v[6] = {&b.pos, &b.vel, &b.ang, &b.fwd, &b.right, &b.up};
        for (int k = 0; k < 6; k++) { v[k]->x = v[k]->x * -1.f; v[k]->y = v[k]->y * -1.f; }
    }
    if (mirror) {
        b.pos.x = -b.pos.x;
        b.vel.x = -b.vel.x;
        b.ang.y = -b.ang.y;
        b.ang.z = -b.ang.z;
        b.fwd.x = -b.fwd.x;
        b.right.x = -b.right.x;
        b.up.x = -b.up.x;
    }
    return b;
}
// world -> body frame of (fwd, right, up)
RSB_D VV toBody(const VBody& b, VV v) { return VV{vdot(b.fwd, v), vdot(b.right, v), vdot(b.up, v)}; }

RSB_D VBody carBody(const EnvView& E, int a, int s) {
    VBody b;
    b.pos = vv(carF(E, a, s, CW_POS) * kBtToUu, carF(E, a, s, CW_POS + 1) * kBtToUu, carF(E, a, s, CW_POS + 2) * kBtToUu);
    b.vel = vv(carF(E, a, s, CW_LIN) * kBtToUu, carF(E, a, s, CW_LIN + 1) * kBtToUu, carF(E, a, s, CW_LIN + 2) * kBtToUu);
    b.ang = vv(carF(E, a, s, CW_ANG), carF(E, a, s, CW_ANG + 1), carF(E, a, s, CW_ANG + 2));
    // CarState::rotMat rows forward, right, up are the basis columns
    b.fwd = vv(carF(E, a, s, CW_ROTMAT + 0), carF(E, a, s, CW_ROTMAT + 3), carF(E, a, s, CW_ROTMAT + 6));
    b.right = vv(carF(E, a, s, CW_ROTMAT + 1), carF(E, a, s, CW_ROTMAT + 4), carF(E, a, s, CW_ROTMAT + 7));
    b.up = vv(carF(E, a, s, CW_ROTMAT + 2), carF(E, a, s, CW_ROTMAT + 5), carF(E, a, s, CW_ROTMAT + 8));
    return b;
}

RSB_D uint32_t vaW(const VantaView& V, int N, int a, int w) { return V.arena[(size_t)w * N + a]; }
RSB_D uint32_t& vaRef(const VantaView& V, int N, int a, int w) { return V.arena[(size_t)w * N + a]; }
RSB_D uint32_t& vtRef(const VantaView& V, int N, int a, int s, int w) {
    return V.car[((size_t)w * MAX_CARS + s) * N + a];
}
RSB_D float vtF(const VantaView& V, int N, int a, int s, int w) {
    return __uint_as_float(V.car[((size_t)w * MAX_CARS + s) * N + a]);
}

// CarState::HasFlipOrJump (Car.cpp:285-289) and the two flip-reset flags of the row
RSB_D bool flipOrJump(uint32_t f, float airSinceJump) {
    return (f & CF_ON_GROUND) ||
           (!(f & CF_HAS_FLIPPED) && !(f & CF_HAS_DOUBLE_JUMPED) && airSinceJump < DOUBLEJUMP_MAX_DELAY);
}

// Nearest small-pad influence and small-pad density around a world position
// (VantaObsGpu.cuh:167-188).
RSB_D void smallPadStats(const VantaTables& T, uint32_t avail0, uint32_t avail1, VV p, float& maxInf,
                         float& density) {
    float m = 0.f, d = 0.f;
    for (int i = 0; i < NUM_PADS; i++) {
        const bool on = ((i < 32 ? avail0 >> i : avail1 >> (i - 32)) & 1u) != 0;
        if (T.z[i] < 72.f && on) {
            const float dist = vlen(vsub(vv(T.x[i], T.y[i], T.z[i]), p));
            const float inf = 1.f / (1.f + dist / 500.f);
            m = fmaxf(m, inf);
            if (dist < 2000.f) d += (1.f - dist / 2000.f);
        }
    }
    maxInf = m;
    density = d / 4.f;
}

// ------------------------------------------------------------------ per-arena update

// One thread per arena: VantaObs's UpdateBoostPads and UpdateDemoTimers
// (VantaObsGpu.cuh:190-246), then UpdateAdditionalTimers of every player
// (VantaObsGpu.cuh:248-339), each once per arena tick.
__global__ void vantaArenaKernel(EnvView E, VantaView V, VantaTables T) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = E.N;
    if (a >= N) return;
    const int M = 2 * E.teamSize[a];
    const uint64_t tick = (uint64_t)E.arena[(size_t)AW_TICK * N + a] |
                          ((uint64_t)E.arena[(size_t)(AW_TICK + 1) * N + a] << 32);
    const float dt = V.dt;
    uint32_t flags = vaW(V, N, a, VA_FLAGS);
    uint64_t last = (uint64_t)vaW(V, N, a, VA_TICK) | ((uint64_t)vaW(V, N, a, VA_TICK + 1) << 32);
    uint32_t avail[2] = {vaW(V, N, a, VA_AVAIL), vaW(V, N, a, VA_AVAIL + 1)};
    if (!(flags & 1u)) {
        for (int i = 0; i < NUM_PADS; i++) vaRef(V, N, a, VA_TIMER + i) = 0u;
        avail[0] = ~0u;
        avail[1] = 3u;
        flags |= 1u;
        last = ~0ull;
    }
    if (last != tick) {
        last = tick;
        for (int i = 0; i < NUM_PADS; i++) {
            const bool active = (E.pad[((size_t)NUM_PADS + T.pad[i]) * N + a] & 1u) != 0;
            uint32_t& w = avail[i >> 5];
            const uint32_t bit = 1u << (i & 31);
            const bool was = (w & bit) != 0;
            float t = __uint_as_float(vaW(V, N, a, VA_TIMER + i));
            if (active != was) {
                w = active ? (w | bit) : (w & ~bit);
                t = active ? 0.f : ((T.z[i] > 72.f) ? 10.f : 4.f);
            } else if (!was) {
                t = fmaxf(0.f, t - dt);
            }
            vaRef(V, N, a, VA_TIMER + i) = __float_as_uint(t);
        }
        // demo timers of every car
        for (int s = 0; s < M; s++) {
            const uint32_t cf = carW(E, a, s, CW_FLAGS);
            uint32_t vf = vtRef(V, N, a, s, VT_FLAGS);
            float demo = vtF(V, N, a, s, VT_DEMO);
            if (!(vf & VF_INIT)) {
                for (int w = 0; w < VT_WORDS; w++) vtRef(V, N, a, s, w) = 0u;
                vf = VF_INIT | ((cf & CF_ON_GROUND) ? VF_ON_GROUND : 0u);
                demo = 0.f;
                vtRef(V, N, a, s, VT_TICK) = ~0u;
                vtRef(V, N, a, s, VT_TICK + 1) = ~0u;
            }
            if (cf & CF_DEMOED) {
                if (!(vf & VF_WAS_DEMOED)) {
                    demo = 3.f;
                    vf |= VF_WAS_DEMOED;
                }
                demo = fmaxf(0.f, demo - dt);
            } else {
                demo = 0.f;
                vf &= ~VF_WAS_DEMOED;
            }
            vtRef(V, N, a, s, VT_DEMO) = __float_as_uint(demo);
            vtRef(V, N, a, s, VT_FLAGS) = vf;
        }
    }
    vaRef(V, N, a, VA_FLAGS) = flags;
    vaRef(V, N, a, VA_AVAIL) = avail[0];
    vaRef(V, N, a, VA_AVAIL + 1) = avail[1];
    vaRef(V, N, a, VA_TICK) = (uint32_t)last;
    vaRef(V, N, a, VA_TICK + 1) = (uint32_t)(last >> 32);

    // the players' coyote timers, driven by each car's previous action
    for (int s = 0; s < M; s++) {
        const uint32_t cf = carW(E, a, s, CW_FLAGS);
        uint32_t vf = vtRef(V, N, a, s, VT_FLAGS);
        if (!(vf & VF_INIT)) {
            for (int w = 0; w < VT_WORDS; w++) vtRef(V, N, a, s, w) = 0u;
            vf = VF_INIT | ((cf & CF_ON_GROUND) ? VF_ON_GROUND : 0u);
            vtRef(V, N, a, s, VT_TICK) = ~0u;
            vtRef(V, N, a, s, VT_TICK + 1) = ~0u;
        }
        const uint64_t pl = (uint64_t)vtRef(V, N, a, s, VT_TICK) | ((uint64_t)vtRef(V, N, a, s, VT_TICK + 1) << 32);
        if (pl == tick) {
            vtRef(V, N, a, s, VT_FLAGS) = vf;
            continue;
        }
        float boostT = vtF(V, N, a, s, VT_BOOST), holdT = vtF(V, N, a, s, VT_BOOST_HOLD);
        float jumpT = vtF(V, N, a, s, VT_JUMP), flipT = vtF(V, N, a, s, VT_FLIP), airT = vtF(V, N, a, s, VT_AIR);
        float hbT = vtF(V, N, a, s, VT_HANDBRAKE);
        VV flipDir = vv(vtF(V, N, a, s, VT_FLIPDIR), vtF(V, N, a, s, VT_FLIPDIR + 1), vtF(V, N, a, s, VT_FLIPDIR + 2));
        const uint32_t ctlBits = carW(E, a, s, CW_LASTCTLBITS);
        const float pPitch = carF(E, a, s, CW_LASTCTL + 2), pYaw = carF(E, a, s, CW_LASTCTL + 3);
        const float pRoll = carF(E, a, s, CW_LASTCTL + 4);
        const bool pJump = ctlBits & 1u, pBoost = ctlBits & 2u, pHandbrake = ctlBits & 4u;

        if (pBoost) boostT = fminf(boostT + dt * 120.f, 12.f);
        else if (boostT >= 12.f) boostT = 0.f;
        if (pBoost) holdT = fminf(holdT + dt * 120.f, 12.f);
        else holdT = fmaxf(holdT - 2.f * dt * 120.f, 0.f);

        bool jumping = vf & VF_JUMPING, jumped = vf & VF_JUMPED, dbl = vf & VF_DOUBLE, flipped = vf & VF_FLIPPED;
        bool onGround = vf & VF_ON_GROUND;
        if (onGround && !jumping) jumped = false;
        const bool jumpPrevReleased = !(vf & VF_PREV_JUMP);
        if (jumping) {
            jumping = jumpT < 3.f || (pJump && jumpT < 24.f);
        } else if (pJump && jumpPrevReleased && onGround) {
            jumping = true;
            jumpT = 0.f;
        }
        if (jumping) {
            jumped = true;
            jumpT = fminf(jumpT + dt * 120.f, 24.f);
        } else {
            jumpT = 0.f;
        }
        if (cf & CF_ON_GROUND) {
            jumping = jumped = dbl = flipped = false;
            airT = 0.f;
            flipT = 0.f;
            flipDir = vv(0.f, 0.f, 0.f);
            onGround = true;
        } else {
            airT = (jumped && !jumping) ? fminf(airT + dt * 120.f, 150.f) : 0.f;
            if (pJump && jumpPrevReleased && (!jumped || airT < 150.f)) {
                if (!dbl && !flipped) {
                    const float absMax = fmaxf(fmaxf(fabsf(pPitch), fabsf(pYaw)), fabsf(pRoll));
                    if (absMax >= V.deadzone) {
                        flipT = 0.f;
                        flipped = true;
                        float fx = pYaw;
                        if (fabsf(fx) < 1e-6f && fabsf(pRoll) >= V.deadzone) fx = pRoll;
                        const float fy = -pPitch;
                        const float n = sqrtf(fx * fx + fy * fy);
                        flipDir = n > 1e-6f ? vv(fx / n, fy / n, 0.f) : vv(0.f, 0.f, 0.f);
                    } else {
                        dbl = true;
                    }
                }
            }
            onGround = false;
        }
        if (flipped) flipT = fminf(flipT + dt * 120.f, 78.f);
        if (pHandbrake) hbT = fminf(hbT + 5.f * dt, 1.f);
        else hbT = fmaxf(hbT - 2.f * dt, 0.f);

        vf = (vf & (VF_INIT | VF_WAS_DEMOED)) | (jumping ? VF_JUMPING : 0u) | (jumped ? VF_JUMPED : 0u) |
             (dbl ? VF_DOUBLE : 0u) | (flipped ? VF_FLIPPED : 0u) | (onGround ? VF_ON_GROUND : 0u) |
             (pJump ? VF_PREV_JUMP : 0u);
        vtRef(V, N, a, s, VT_BOOST) = __float_as_uint(boostT);
        vtRef(V, N, a, s, VT_BOOST_HOLD) = __float_as_uint(holdT);
        vtRef(V, N, a, s, VT_JUMP) = __float_as_uint(jumpT);
        vtRef(V, N, a, s, VT_FLIP) = __float_as_uint(flipT);
        vtRef(V, N, a, s, VT_AIR) = __float_as_uint(airT);
        vtRef(V, N, a, s, VT_HANDBRAKE) = __float_as_uint(hbT);
        vtRef(V, N, a, s, VT_FLIPDIR) = __float_as_uint(flipDir.x);
        vtRef(V, N, a, s, VT_FLIPDIR + 1) = __float_as_uint(flipDir.y);
        vtRef(V, N, a, s, VT_FLIPDIR + 2) = __float_as_uint(flipDir.z);
        vtRef(V, N, a, s, VT_FLAGS) = vf;
        vtRef(V, N, a, s, VT_TICK) = (uint32_t)tick;
        vtRef(V, N, a, s, VT_TICK + 1) = (uint32_t)(tick >> 32);
    }
}

// ------------------------------------------------------------------ rows

// The 39 values of another car seen by the player (VantaObsGpu.cuh:653-706).
RSB_D void vantaCarPacket(const EnvView& E, const VantaView& V, const VantaTables& T, int a, int q,
                          const VBody& self, VV ballPos, bool inv, bool mirror, uint32_t av0, uint32_t av1,
                          float*& o) {
    const int N = E.N;
    const VBody world = carBody(E, a, q);
    const VBody c = canonical(world, inv, mirror);
    const VV relPos = vsub(c.pos, self.pos), relVel = vsub(c.vel, self.vel);
    const VV bPos = toBody(self, relPos), bVel = toBody(self, relVel), bAng = toBody(self, c.ang);
    const float distEgo = vlen(relPos), distBall = vlen(vsub(c.pos, ballPos));
    *o++ = c.pos.x / VA_POS_STD; *o++ = c.pos.y / VA_POS_STD; *o++ = c.pos.z / VA_POS_STD;
    *o++ = c.vel.x / VA_VEL_STD; *o++ = c.vel.y / VA_VEL_STD; *o++ = c.vel.z / VA_VEL_STD;
    *o++ = c.ang.x / VA_ANG_STD; *o++ = c.ang.y / VA_ANG_STD; *o++ = c.ang.z / VA_ANG_STD;
    *o++ = bPos.x / VA_POS_STD; *o++ = bPos.y / VA_POS_STD; *o++ = bPos.z / VA_POS_STD;
    *o++ = bVel.x / VA_VEL_STD; *o++ = bVel.y / VA_VEL_STD; *o++ = bVel.z / VA_VEL_STD;
    *o++ = bAng.x / VA_ANG_STD; *o++ = bAng.y / VA_ANG_STD; *o++ = bAng.z / VA_ANG_STD;
    *o++ = c.fwd.x; *o++ = c.fwd.y; *o++ = c.fwd.z;
    *o++ = c.up.x; *o++ = c.up.y; *o++ = c.up.z;
    const uint32_t f = carW(E, a, q, CW_FLAGS);
    *o++ = carF(E, a, q, CW_BOOST) / 100.f;
    *o++ = (f & CF_ON_GROUND) ? 1.f : 0.f;
    *o++ = flipOrJump(f, carF(E, a, q, CW_AIRSJ)) ? 1.f : 0.f;
    *o++ = (f & CF_DEMOED) ? 1.f : 0.f;
    *o++ = (f & CF_SUPERSONIC) ? 1.f : 0.f;
    *o++ = distEgo / VA_POS_STD;
    *o++ = distBall / VA_POS_STD;
    // the car's demo timer, when its timers exist
    *o++ = ((vtRef(V, N, a, q, VT_FLAGS) & VF_INIT) ? vtF(V, N, a, q, VT_DEMO) : 0.f) / VA_DEMO_STD;
    *o++ = (f & CF_IS_JUMPING) ? 1.f : 0.f;
    *o++ = (f & CF_IS_FLIPPING) ? 1.f : 0.f;
    *o++ = (f & CF_HAS_DOUBLE_JUMPED) ? 1.f : 0.f;
    *o++ = vlen(c.vel) / VA_VEL_STD;
    *o++ = (f & CF_HAS_FLIPPED) ? 1.f : 0.f;
    float inf, dens;
    smallPadStats(T, av0, av1, world.pos, inf, dens);
    *o++ = inf;
    *o++ = dens;
}

// Writes the warp's 32 staged row sections (columns [c0, c0 + len) of rows row0 .. row0 + 31)
// to the output, one row at a time with the lanes on consecutive columns: coalesced stores
// instead of 32 rows 1,464 bytes apart per store instruction.
constexpr int VANTA_THREADS = 128, VANTA_STAGE = 81;  // the longest section (ego)
RSB_D void vantaFlush(float (*buf)[VANTA_STAGE], float* rows, int row0, int numCars, int c0, int len, int lane) {
    __syncwarp();
    for (int j = 0; j < 32 && row0 + j < numCars; j++) {
        float* dst = rows + (size_t)(row0 + j) * VANTA_ROW + c0;
        for (int k = lane; k < len; k += 32) dst[k] = buf[j][k];
    }
    __syncwarp();
}

// One thread per player (packed row r = carOffset[a] + slot): VantaObs::BuildObs
// (VantaObsGpu.cuh:342-748) on the state after the arena update.  Each lane builds its row a
// section at a time in its warp's shared-memory stage (odd row stride: no bank conflicts), and
// the warp writes the section out with vantaFlush.  Lanes past the last row compute the last
// row again (so that every lane reaches every flush) and write nothing.
__global__ void __launch_bounds__(VANTA_THREADS) vantaRowKernel(EnvView E, VantaView V, VantaTables T, int numCars) {
    __shared__ float stage[VANTA_THREADS / 32][32][VANTA_STAGE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row0 = blockIdx.x * blockDim.x + warp * 32;
    const int r = min(row0 + lane, numCars - 1);
    float(*buf)[VANTA_STAGE] = stage[warp];
    float* const mine = buf[lane];
    float* o = mine;
    auto flush = [&](int c0) {
        vantaFlush(buf, V.rows, row0, numCars, c0, (int)(o - mine), lane);
        o = mine;
    };
    const int N = E.N;
    // the arena of row r: the last arena whose first row is <= r
    int lo = 0, hi = N - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (E.carOffset[mid] <= r) lo = mid;
        else hi = mid - 1;
    }
    const int a = lo, s = r - E.carOffset[a], M = 2 * E.teamSize[a];

    const uint32_t pf = carW(E, a, s, CW_FLAGS);
    const VBody world = carBody(E, a, s);
    const bool inv = (pf & CF_TEAM_ORANGE) != 0;
    const bool mirror = world.pos.x < 0.f;
    const VBody self = canonical(world, inv, mirror);
    VBody ballW;
    ballW.pos = vv(ballF(E, a, BW_POS) * kBtToUu, ballF(E, a, BW_POS + 1) * kBtToUu, ballF(E, a, BW_POS + 2) * kBtToUu);
    ballW.vel = vv(ballF(E, a, BW_LIN) * kBtToUu, ballF(E, a, BW_LIN + 1) * kBtToUu, ballF(E, a, BW_LIN + 2) * kBtToUu);
    ballW.ang = vv(ballF(E, a, BW_ANG), ballF(E, a, BW_ANG + 1), ballF(E, a, BW_ANG + 2));
    ballW.fwd = vv(1.f, 0.f, 0.f);
    ballW.right = vv(0.f, 1.f, 0.f);
    ballW.up = vv(0.f, 0.f, 1.f);
    const VBody ball = canonical(ballW, inv, mirror);
    const uint32_t av0 = vaW(V, N, a, VA_AVAIL), av1 = vaW(V, N, a, VA_AVAIL + 1);

    // ---- ego (81)
    const VV posDiff = vsub(ball.pos, self.pos), velDiff = vsub(ball.vel, self.vel);
    {
        const VV relPos = toBody(self, posDiff), relVel = toBody(self, velDiff), angBody = toBody(self, self.ang);
        *o++ = self.pos.x / VA_POS_STD; *o++ = self.pos.y / VA_POS_STD; *o++ = self.pos.z / VA_POS_STD;
        *o++ = self.vel.x / VA_VEL_STD; *o++ = self.vel.y / VA_VEL_STD; *o++ = self.vel.z / VA_VEL_STD;
        *o++ = self.ang.x / VA_ANG_STD; *o++ = self.ang.y / VA_ANG_STD; *o++ = self.ang.z / VA_ANG_STD;
        *o++ = relPos.x / VA_POS_STD; *o++ = relPos.y / VA_POS_STD; *o++ = relPos.z / VA_POS_STD;
        *o++ = relVel.x / VA_BALL_VEL_STD; *o++ = relVel.y / VA_BALL_VEL_STD; *o++ = relVel.z / VA_BALL_VEL_STD;
        *o++ = self.fwd.x; *o++ = self.fwd.y; *o++ = self.fwd.z;
        *o++ = self.up.x; *o++ = self.up.y; *o++ = self.up.z;
        *o++ = angBody.x / VA_ANG_STD; *o++ = angBody.y / VA_ANG_STD; *o++ = angBody.z / VA_ANG_STD;
        *o++ = vlen(self.vel) / VA_VEL_STD;
        const float boost = carF(E, a, s, CW_BOOST);
        const bool fj = flipOrJump(pf, carF(E, a, s, CW_AIRSJ));
        const bool ground = pf & CF_ON_GROUND, jumped = pf & CF_HAS_JUMPED;
        *o++ = boost / 100.f;
        *o++ = ground ? 1.f : 0.f;
        *o++ = fj ? 1.f : 0.f;
        *o++ = (pf & CF_DEMOED) ? 1.f : 0.f;
        *o++ = jumped ? 1.f : 0.f;
        *o++ = (pf & CF_SUPERSONIC) ? 1.f : 0.f;
        float wheels = 0.f;
        for (int i = 0; i < 4; i++) wheels += (pf & (CF_WHEEL0 << i)) ? 1.f : 0.f;
        *o++ = wheels / 4.f;
        *o++ = (!ground && fj && !jumped) ? 1.f : 0.f;  // has a flip reset
        *o++ = (!ground && !jumped) ? 1.f : 0.f;        // got a flip reset
        *o++ = carF(E, a, s, CW_HANDBRAKE);
        *o++ = mirror ? 1.f : 0.f;
        *o++ = inv ? 1.f : 0.f;
        // threat frame: along the ball -> own goal direction and across it
        {
            const VV ownGoal = vv(0.f, -5120.f, 0.f);
            const VV toGoal = vsub(ownGoal, ball.pos);
            const float len = vlen(toGoal);
            const VV danger = len > 1.f ? vdiv(toGoal, len) : vv(0.f, -1.f, 0.f);
            VV lateral = vv(-danger.y, danger.x, 0.f);
            const float latLen = vlen(lateral);
            if (latLen > 1e-6f) lateral = vdiv(lateral, latLen);
            *o++ = vdot(ball.vel, danger) / VA_BALL_VEL_STD;
            *o++ = vdot(self.vel, danger) / VA_VEL_STD;
            *o++ = vdot(self.vel, lateral) / VA_VEL_STD;
            const VV carToBall = vsub(ball.pos, self.pos);
            *o++ = vdot(carToBall, danger) / VA_POS_STD;
            *o++ = vdot(carToBall, lateral) / VA_POS_STD;
            *o++ = vlen(vsub(ownGoal, ball.pos)) / (2.f * VA_POS_STD);
        }
        // alignment
        {
            const VV attackGoal = vv(0.f, 5120.f, 0.f);
            const VV velN = vunit(self.vel), toBallN = vunit(vsub(ball.pos, self.pos));
            const VV toGoalN = vunit(vsub(attackGoal, self.pos));
            *o++ = vdot(self.fwd, toBallN);
            *o++ = vdot(self.fwd, toGoalN);
            *o++ = vdot(velN, toBallN);
            *o++ = vdot(self.up, vv(0.f, 0.f, 1.f));
        }
        // previous action, steer / yaw / roll mirrored with the frame
        {
            const uint32_t bits = carW(E, a, s, CW_LASTCTLBITS);
            const float steer = carF(E, a, s, CW_LASTCTL + 1), yaw = carF(E, a, s, CW_LASTCTL + 3);
            const float roll = carF(E, a, s, CW_LASTCTL + 4);
            *o++ = carF(E, a, s, CW_LASTCTL + 0);
            *o++ = mirror ? -steer : steer;
            *o++ = carF(E, a, s, CW_LASTCTL + 2);
            *o++ = mirror ? -yaw : yaw;
            *o++ = mirror ? -roll : roll;
            *o++ = (bits & 1u) ? 1.f : 0.f;
            *o++ = (bits & 2u) ? 1.f : 0.f;
            *o++ = (bits & 4u) ? 1.f : 0.f;
        }
        const bool contact = pf & CF_WORLD_CONTACT;
        const VV wcn = vv(carF(E, a, s, CW_WCN), carF(E, a, s, CW_WCN + 1), carF(E, a, s, CW_WCN + 2));
        *o++ = (contact && wcn.z < 0.7f) ? 1.f : 0.f;  // wall / ceiling contact
        // the player's timers
        const uint32_t vf = vtRef(V, N, a, s, VT_FLAGS);
        *o++ = vtF(V, N, a, s, VT_DEMO) / VA_DEMO_STD;
        *o++ = vtF(V, N, a, s, VT_BOOST) / 12.f;
        *o++ = vtF(V, N, a, s, VT_JUMP) / 24.f;
        *o++ = vtF(V, N, a, s, VT_AIR) / 150.f;
        *o++ = vtF(V, N, a, s, VT_FLIP) / 78.f;
        *o++ = vtF(V, N, a, s, VT_HANDBRAKE);
        const float fdx = vtF(V, N, a, s, VT_FLIPDIR);
        *o++ = mirror ? -fdx : fdx;
        *o++ = vtF(V, N, a, s, VT_FLIPDIR + 1);
        *o++ = vtF(V, N, a, s, VT_BOOST_HOLD) / 12.f;
        *o++ = (vf & VF_JUMPING) ? 1.f : 0.f;
        *o++ = (vf & VF_FLIPPED) ? 1.f : 0.f;
        *o++ = (vf & VF_DOUBLE) ? 1.f : 0.f;
        // enrichments
        const float boostFrac = boost / 100.f;
        const float distToBall = vlen(posDiff);
        const float closing = distToBall > 1e-3f ? (-vdot(velDiff, posDiff) / distToBall) / VA_VEL_STD : 0.f;
        *o++ = sqrtf(fmaxf(0.f, boostFrac));
        *o++ = (ball.pos.z > self.pos.z + 200.f) ? 1.f : 0.f;
        *o++ = closing;
        *o++ = distToBall / VA_POS_STD;
        // surface contact and its normal in the canonical frame
        VV n = vv(0.f, 0.f, 0.f);
        if (contact) {
            n = wcn;
            if (inv) { n.x = -n.x; n.y = -n.y; }
            if (mirror) n.x = -n.x;
        }
        *o++ = contact ? 1.f : 0.f;
        *o++ = n.x; *o++ = n.y; *o++ = n.z;
        *o++ = (pf & CF_IS_FLIPPING) ? 1.f : 0.f;
        *o++ = 0.f;  // headroom slot
        // kickoff side: the team frame's x, not mirrored
        *o++ = ((inv ? world.pos.x * -1.f : world.pos.x) < 0.f) ? 1.f : 0.f;
        float inf, dens;
        smallPadStats(T, av0, av1, world.pos, inf, dens);
        *o++ = inf;
        *o++ = dens;
    }

    flush(0);

    // ---- ball (29)
    *o++ = ball.pos.x / VA_POS_STD; *o++ = ball.pos.y / VA_POS_STD; *o++ = ball.pos.z / VA_POS_STD;
    *o++ = ball.vel.x / VA_BALL_VEL_STD; *o++ = ball.vel.y / VA_BALL_VEL_STD; *o++ = ball.vel.z / VA_BALL_VEL_STD;
    *o++ = ball.ang.x / VA_ANG_STD; *o++ = ball.ang.y / VA_ANG_STD; *o++ = ball.ang.z / VA_ANG_STD;
    *o++ = vlen(ball.vel) / VA_BALL_VEL_STD;
    *o++ = (ball.pos.z <= 100.f) ? 1.f : 0.f;
    for (int k = 0; k < 3; k++) {
        if (V.pred) {
            const rsb_ball_state& p = V.pred[(size_t)a * 3 + k];
            VBody b = ballW;
            b.pos = vv(p.pos.x, p.pos.y, p.pos.z);
            b.vel = vv(p.vel.x, p.vel.y, p.vel.z);
            b.ang = vv(0.f, 0.f, 0.f);
            b = canonical(b, inv, mirror);
            *o++ = b.pos.x / VA_POS_STD; *o++ = b.pos.y / VA_POS_STD; *o++ = b.pos.z / VA_POS_STD;
            *o++ = b.vel.x / VA_BALL_VEL_STD; *o++ = b.vel.y / VA_BALL_VEL_STD; *o++ = b.vel.z / VA_BALL_VEL_STD;
        } else {
            for (int j = 0; j < 6; j++) *o++ = 0.f;
        }
    }

    flush(81);

    // ---- goal context (16)
    {
        const VV opp = vv(0.f, 5120.f, 0.f), own = vv(0.f, -5120.f, 0.f);
        const VV sOpp = vsub(opp, self.pos), sOwn = vsub(own, self.pos);
        const VV lOpp = toBody(self, sOpp), lOwn = toBody(self, sOwn);
        *o++ = lOpp.x * VA_GOAL_COEF; *o++ = lOpp.y * VA_GOAL_COEF; *o++ = lOpp.z * VA_GOAL_COEF;
        *o++ = vlen(sOpp) * VA_GOAL_COEF;
        *o++ = lOwn.x * VA_GOAL_COEF; *o++ = lOwn.y * VA_GOAL_COEF; *o++ = lOwn.z * VA_GOAL_COEF;
        *o++ = vlen(sOwn) * VA_GOAL_COEF;
        const VV bOpp = vsub(opp, ball.pos), bOwn = vsub(own, ball.pos);
        *o++ = bOpp.x * VA_GOAL_COEF; *o++ = bOpp.y * VA_GOAL_COEF; *o++ = bOpp.z * VA_GOAL_COEF;
        *o++ = vlen(bOpp) * VA_GOAL_COEF;
        *o++ = bOwn.x * VA_GOAL_COEF; *o++ = bOwn.y * VA_GOAL_COEF; *o++ = bOwn.z * VA_GOAL_COEF;
        *o++ = vlen(bOwn) * VA_GOAL_COEF;
    }

    // ---- team context (6): who touched the ball last, team sizes, ball half
    {
        int touchSlot = -1;
        uint64_t best = 0;
        for (int q = 0; q < M; q++) {
            const uint64_t t = (uint64_t)carW(E, a, q, CW_HIT) | ((uint64_t)carW(E, a, q, CW_HIT + 1) << 32);
            if ((carW(E, a, q, CW_FLAGS) & CF_BALL_HIT_VALID) && t != ~0ull && t >= best) {
                best = t;
                touchSlot = q;
            }
        }
        int who = -1;
        if (touchSlot >= 0)
            who = touchSlot == s ? 0 : (((carW(E, a, touchSlot, CW_FLAGS) & CF_TEAM_ORANGE) != 0) == inv ? 1 : 2);
        *o++ = who == 0 ? 1.f : 0.f;
        *o++ = who == 1 ? 1.f : 0.f;
        *o++ = who == 2 ? 1.f : 0.f;
        int orange = 0;
        for (int q = 0; q < M; q++) orange += (carW(E, a, q, CW_FLAGS) & CF_TEAM_ORANGE) ? 1 : 0;
        const int blue = M - orange;
        *o++ = (float)(inv ? orange : blue) / 3.f;
        *o++ = (float)(inv ? blue : orange) / 3.f;
        *o++ = (ball.pos.y < 0.f) ? 1.f : 0.f;
    }

    flush(110);  // goal and team context

    // ---- teammates and opponents by canonical distance to the ball (stable on ties)
    int mate[MAX_CARS], opp[MAX_CARS];
    float mateD[MAX_CARS], oppD[MAX_CARS];
    int nm = 0, no = 0;
    for (int q = 0; q < M; q++) {
        if (q == s) continue;
        const uint32_t f = carW(E, a, q, CW_FLAGS);
        float d = 3.402823466e+38f;
        if (!(f & CF_DEMOED)) d = vlen(vsub(canonical(carBody(E, a, q), inv, mirror).pos, ball.pos));
        const bool same = ((f & CF_TEAM_ORANGE) != 0) == inv;
        int* idx = same ? mate : opp;
        float* dist = same ? mateD : oppD;
        int& n = same ? nm : no;
        int j = n - 1;
        while (j >= 0 && dist[j] > d) {
            idx[j + 1] = idx[j];
            dist[j + 1] = dist[j];
            j--;
        }
        idx[j + 1] = q;
        dist[j + 1] = d;
        n++;
    }
    for (int i = 0; i < 2; i++) {
        if (i < nm) vantaCarPacket(E, V, T, a, mate[i], self, ball.pos, inv, mirror, av0, av1, o);
        else for (int k = 0; k < 39; k++) *o++ = 0.f;
        flush(132 + 39 * i);
    }
    const int oppLimit = V.onlyClosestOpp ? 1 : 3;
    for (int i = 0; i < 3; i++) {
        if (i < oppLimit && i < no) vantaCarPacket(E, V, T, a, opp[i], self, ball.pos, inv, mirror, av0, av1, o);
        else for (int k = 0; k < 39; k++) *o++ = 0.f;
        flush(132 + 39 * (2 + i));
    }
    for (int i = 0; i < 2; i++) *o++ = i < nm ? 1.f : 0.f;
    for (int i = 0; i < 3; i++) *o++ = (i < oppLimit && i < no) ? 1.f : 0.f;

    // ---- boost pads (34), in the player's frame
    for (int i = 0; i < NUM_PADS; i++) {
        int idx = inv ? NUM_PADS - 1 - i : i;
        if (mirror) idx = T.mirror[idx];
        const bool on = ((idx < 32 ? av0 >> idx : av1 >> (idx - 32)) & 1u) != 0;
        if (on) {
            *o++ = 1.f;
        } else {
            const float tMax = T.z[idx] > 72.f ? 10.f : 4.f;
            *o++ = 1.f / (1.f + __uint_as_float(vaW(V, N, a, VA_TIMER + idx)) / tMax);
        }
    }
    flush(327);  // validity mask and pads
}

}  // namespace rsb
