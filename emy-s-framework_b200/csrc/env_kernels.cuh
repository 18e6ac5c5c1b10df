// Env layer of the collector's GPU path, on the device: what GigaLearnCPP's EnvSet does
// around each arena step, for every arena of the batch at once.
//
//   obsKernel ...... AdvancedObs rows and DefaultAction masks of every player
//                    (RLGymCPP AdvancedObs.cpp:4-65, StateUtil.cpp:3-17 InvertPhys,
//                    GameState.cpp:96-116 boost-pad order, DefaultAction.cpp:94-118)
//   rewardKernel ... the four stub rewards and the terminal conditions of one env step
//                    (CommonRewards.h:33-98, ZeroSumReward.cpp:3-31, GoalScoreCondition.h,
//                    NoTouchCondition.h, EnvSet.cpp:184-254)
//   resetKernel .... seeded arena resets: kickoff (Arena::ResetToRandomKickoff
//                    Arena.cpp:112-216), random state (RandomState.cpp:9-60), the reference
//                    batch's curriculum (RocketSimCudaApi.cuh:203-442), high-contact
//
// Player order.  EnvSet walks the players of an arena in Arena::_cars order, which the
// physics kernel takes to be reverse creation order (the order libstdc++'s unordered_set
// visits the cars when each pointer hashes to its own bucket).  Observation rows and
// reward slots are indexed by creation slot (the C ABI's packed player order), but the
// teammate / opponent blocks inside a row, and the team sums of ZeroSumReward, follow the
// reverse-slot order, as the reference's loops do.
//
// Floating point follows the reference expression by expression (RocketSim Vec: dot
// products add a fourth "w" product, which is +0 here; divisions are IEEE divisions).
#pragma once
#include <stddef.h>

#include "phys/state.h"
#include "phys/engine_core.h"

namespace rsb {

// AdvancedObs coefficients (AdvancedObs.h:10-13)
constexpr float OBS_POS = 1 / 5000.f, OBS_VEL = 1 / 2300.f, OBS_ANG = 1 / 3.f;
// CommonValues.h:17-45
constexpr float CV_BACK_NET_Y = 6000.f, CV_GOAL_HEIGHT = 642.775f, CV_BALL_MAX_SPEED = 6000.f,
                CV_CAR_MAX_SPEED = 2300.f, CV_BALL_RADIUS = 92.75f;

// Per-launch constant tables, built on the host at create (engine_host.h).
struct EnvTables {
    int32_t padMap[NUM_PADS];    // RLGymCPP pad index (CommonValues::BOOST_LOCATIONS) -> arena pad
    uint32_t ground[3], air[3], jump[3], boost[3];  // DefaultAction masks as 90-bit sets
    float kickRot[2][NUM_KICKOFF_SPAWNS][9];         // kickoff bases (rows), blue / orange
    float kickX[NUM_KICKOFF_SPAWNS], kickY[NUM_KICKOFF_SPAWNS];
};

struct RewardParams {
    float w[4];               // GoalReward, TouchBallReward, VelocityBallToGoal, VelocityPlayerToBall
    float concede, teamSpirit, oppScale;
    int32_t zeroSum;          // bit k: reward k wrapped in ZeroSumReward
    int32_t episodeMaxTicks;  // truncation after this many ticks since the reset (0 = off)
    float noTouchTimeout;     // NoTouchCondition seconds (0 = off)
    float goalBaseY, ballRadius;
};

struct EnvView {
    uint32_t* ball;
    uint32_t* car;
    uint32_t* pad;
    uint32_t* arena;
    int N;
    const int32_t* teamSize;
    const int32_t* carOffset;
    CtlRec* controls;
    float* obs;
    int stride;
    uint8_t* masks;
    float* rewards;
    uint8_t* terminals;
    uint32_t* vantaArena;  // VantaObs builder state (VANTA_ARENA_WORDS planes), null when off
    uint32_t* vantaCar;    // VANTA_CAR_WORDS planes of [MAX_CARS][N]
};
// Words of the VantaObs builder's state per arena and per car (laid out in vanta.cuh); an arena
// reset clears them, as the reference's ResetArena clears the builder's state
// (RocketSimCudaApi.cuh:265-275).
constexpr int VANTA_ARENA_WORDS = NUM_PADS + 5, VANTA_CAR_WORDS = 13;

// word indices inside the records
#define RSB_W(T, f) ((int)(offsetof(T, f) / 4))
constexpr int BW_POS = RSB_W(BallP, pos), BW_ROT = RSB_W(BallP, rot), BW_LIN = RSB_W(BallP, lin), BW_ANG = RSB_W(BallP, ang);
constexpr int CW_POS = RSB_W(CarP, pos), CW_ROT = RSB_W(CarP, rot), CW_LIN = RSB_W(CarP, lin), CW_ANG = RSB_W(CarP, ang);
constexpr int CW_BOOST = RSB_W(CarP, boost), CW_AIRSJ = RSB_W(CarP, airTimeSinceJump);
constexpr int CW_WCN = RSB_W(CarP, worldContactNormal), CW_FLAGS = RSB_W(CarP, flags);
constexpr int CW_HIT = RSB_W(CarP, ballHitTick), CW_HITX = RSB_W(CarP, ballHitExtraTick), CW_ROTMAT = RSB_W(CarP, rotMat);
constexpr int CW_STATE0 = RSB_W(CarP, boost), CW_STATE1 = RSB_W(CarP, steerAngle);  // CarState words
constexpr int AW_TICK = RSB_W(ArenaP, tick), AW_EPISODE = RSB_W(ArenaP, episodeTicks), AW_STATUS = RSB_W(ArenaP, status);
constexpr int AW_GOALTEAM = RSB_W(ArenaP, goalTeam), AW_TOUCHED = RSB_W(ArenaP, touchedMask);
constexpr int AW_NOTOUCH = RSB_W(ArenaP, noTouchTimer), AW_SCORED = RSB_W(ArenaP, scored);
#undef RSB_W

RSB_D uint32_t ballW(const EnvView& E, int a, int w) { return E.ball[(size_t)w * E.N + a]; }
RSB_D uint32_t carW(const EnvView& E, int a, int s, int w) { return E.car[((size_t)w * MAX_CARS + s) * E.N + a]; }
RSB_D float ballF(const EnvView& E, int a, int w) { return __uint_as_float(ballW(E, a, w)); }
RSB_D float carF(const EnvView& E, int a, int s, int w) { return __uint_as_float(carW(E, a, s, w)); }

// RocketSim Vec::Dot with its fourth (zero) component: ((x*x' + y*y') + z*z') + 0*0
RSB_D float vdot4(float ax, float ay, float az, float bx, float by, float bz) {
    return ((ax * bx + ay * by) + az * bz) + 0.f;
}

// ------------------------------------------------------------------ observations

// A row of AdvancedObs (AdvancedObs.cpp:25-65) for player p of an arena of team size T, in
// the frame of p's team (orange = InvertPhys): ball (9), p's action (8), pad values (34),
// then 2T car blocks of 29 (p, its teammates by descending slot, the opponents by descending
// slot), then zeros up to the batch's row stride.
constexpr int OBS_STRIDE_MAX = RSB_OBS_BASE + RSB_OBS_PER_CAR * MAX_CARS;
constexpr int OBS_COL_PREV = 9, OBS_COL_PAD = 17, OBS_COL_CAR = RSB_OBS_BASE;

// Index of car q's block in the row of viewer p (q, p of one arena of team size T): the
// inverse of the order above.
RSB_HD int obsCarIndex(int T, int p, int q) {
    const bool orange = p >= T;
    const int ownFirst = orange ? T : 0, oppFirst = orange ? 0 : T;
    if (q == p) return 0;
    if (q >= ownFirst && q < ownFirst + T) return 1 + (ownFirst + T - 1 - q) - (p > q ? 1 : 0);
    return T + (oppFirst + T - 1 - q);
}

// Per-arena inputs of the car blocks, staged in shared memory, one column per arena.
constexpr int OBS_ARENAS = 8;
constexpr int OI_BALL = 0;                        // ball pos, vel (uu)
constexpr int OI_CAR = 6;                         // per car, OI_CAR_N words
constexpr int OI_CAR_N = 21;                      // pos vel ang fwd right up boost flags, 1 pad word
                                                  // (an odd stride keeps the cars on distinct banks)
constexpr int OI_MASK = OI_CAR + MAX_CARS * OI_CAR_N;  // per car, 3 mask words
constexpr int OI_WORDS = OI_MASK + MAX_CARS * 3;
// flag bits of the staged car
constexpr uint32_t OF_GROUND = 1, OF_FLIPJUMP = 2, OF_DEMOED = 4, OF_JUMPED = 8;

struct ObsShared {
    // the block's rows, flat, at the same offset modulo 16 bytes as in the output buffer
    __align__(16) float stage[OBS_ARENAS * MAX_CARS * OBS_STRIDE_MAX + 4];
    float in[OI_WORDS][OBS_ARENAS];
    uint8_t rowBase[OBS_ARENAS];              // first row of each arena, in the block
    uint8_t team[OBS_ARENAS];
    uint8_t rowOf[OBS_ARENAS * MAX_CARS];     // block row -> arena | slot << 4
};

// The 29 values of car q's block in one frame (inv: the orange frame, InvertPhys), written to
// o[0..29) (AdvancedObs::AddPlayerToObs, AdvancedObs.cpp:25-49: position, forward, up,
// velocity, angular velocity, the three rotMat.Dot rows, boost, four flags).
RSB_D void obsCarBlock(const ObsShared& S, int la, int q, bool inv, float* o) {
    const int b = OI_CAR + q * OI_CAR_N;
    float g[18];
    for (int k = 0; k < 18; k++) g[k] = S.in[b + k][la];
    if (inv)
        for (int k = 0; k < 18; k += 3) { g[k] = -g[k]; g[k + 1] = -g[k + 1]; }
    // pos 0..2, vel 3..5, ang 6..8, forward 9..11, right 12..14, up 15..17
    o[0] = g[0] * OBS_POS; o[1] = g[1] * OBS_POS; o[2] = g[2] * OBS_POS;
    o[3] = g[9]; o[4] = g[10]; o[5] = g[11];
    o[6] = g[15]; o[7] = g[16]; o[8] = g[17];
    o[9] = g[3] * OBS_VEL; o[10] = g[4] * OBS_VEL; o[11] = g[5] * OBS_VEL;
    o[12] = g[6] * OBS_ANG; o[13] = g[7] * OBS_ANG; o[14] = g[8] * OBS_ANG;
    float bp[3], bv[3];
    for (int k = 0; k < 3; k++) {
        bp[k] = S.in[OI_BALL + k][la];
        bv[k] = S.in[OI_BALL + 3 + k][la];
    }
    if (inv) { bp[0] = -bp[0]; bp[1] = -bp[1]; bv[0] = -bv[0]; bv[1] = -bv[1]; }
    const float rp[3] = {bp[0] - g[0], bp[1] - g[1], bp[2] - g[2]};
    const float rv[3] = {bv[0] - g[3], bv[1] - g[4], bv[2] - g[5]};
    for (int r = 0; r < 3; r++) {
        const float* bk = g + 9 + 3 * r;  // forward, right, up
        o[15 + r] = vdot4(g[6], g[7], g[8], bk[0], bk[1], bk[2]) * OBS_ANG;
        o[18 + r] = vdot4(rp[0], rp[1], rp[2], bk[0], bk[1], bk[2]) * OBS_POS;
        o[21 + r] = vdot4(rv[0], rv[1], rv[2], bk[0], bk[1], bk[2]) * OBS_VEL;
    }
    o[24] = S.in[b + 18][la] / 100.f;
    const uint32_t f = __float_as_uint(S.in[b + 19][la]);
    o[25] = (f & OF_GROUND) ? 1.f : 0.f;
    o[26] = (f & OF_FLIPJUMP) ? 1.f : 0.f;
    o[27] = (f & OF_DEMOED) ? 1.f : 0.f;
    o[28] = (f & OF_JUMPED) ? 1.f : 0.f;
}

// Four mask bits from bit b of a 96-bit action mask, spread to four bytes of 0 / 1 (byte t of
// the little-endian word = bit b + t).
RSB_D uint32_t maskNibbleBytes(uint32_t m0, uint32_t m1, uint32_t m2, int b) {
    const int w = b >> 5;
    const uint32_t lo = w == 0 ? m0 : (w == 1 ? m1 : m2), hi = w == 0 ? m1 : (w == 1 ? m2 : 0u);
    const uint32_t x = __funnelshift_r(lo, hi, b & 31) & 15u;
    return (x * 0x00204081u) & 0x01010101u;
}

// A block of 512 threads serves 8 arenas (47 KB of shared memory, at most 40 registers a
// thread: 3 blocks per SM) in three phases, every thread taking part in each, one item per
// thread where the items allow (so that a thread's reads are issued together, not behind one
// another):
//   A. read the arenas' word planes (consecutive threads on consecutive arenas of one word),
//      stage what the car blocks need, and write the ball, action and pad columns of every
//      row straight into the staged rows;
//   B. write every car's 29-value block, per team frame and viewer, into that viewer's row,
//      and the mask bytes of the block's rows to the output as 32-bit words;
//   C. send the staged rows out: the 16-byte-aligned middle as one bulk copy from shared
//      memory (cp.async.bulk), the few elements either side as plain stores.
constexpr int OBS_THREADS = 512;
__global__ void __launch_bounds__(OBS_THREADS, 3) obsKernel(EnvView E, EnvTables Tb) {
    __shared__ ObsShared S;
    const int tid = threadIdx.x;
    const int a0 = blockIdx.x * OBS_ARENAS;
    if (a0 >= E.N) return;
    const int na = min(OBS_ARENAS, E.N - a0);
    const int row0 = E.carOffset[a0];
    const int rows = E.carOffset[a0 + na] - row0;
    const int stride = E.stride;
    float* out = E.obs + (size_t)row0 * stride;
    const int mis = (int)((reinterpret_cast<uintptr_t>(out) >> 2) & 3);
    float* st = S.stage + mis;

    // ---- A
    constexpr int nCar = 2 * MAX_CARS * OBS_ARENAS, nBall = 9 * OBS_ARENAS, nPad = NUM_PADS * OBS_ARENAS;
    for (int i = tid; i < nCar + nBall + nPad; i += OBS_THREADS) {
        if (i < nCar) {
            // (arena, slot, half): half 0 the kinematics, half 1 flags, masks and the action
            const int la = i % OBS_ARENAS, s = (i / OBS_ARENAS) % MAX_CARS, half = i / (OBS_ARENAS * MAX_CARS);
            const int a = a0 + la;
            if (la >= na) continue;
            // every slot's words are in the planes: read them before the team size arrives
            const int o = OI_CAR + s * OI_CAR_N;
            if (half == 0) {
                float v[18];
                for (int k = 0; k < 3; k++) {
                    v[k] = carF(E, a, s, CW_POS + k) * kBtToUu;
                    v[3 + k] = carF(E, a, s, CW_LIN + k) * kBtToUu;
                    v[6 + k] = carF(E, a, s, CW_ANG + k);
                    // CarState::rotMat columns: forward, right, up (basis rows stored)
                    v[9 + k] = carF(E, a, s, CW_ROTMAT + 3 * k + 0);
                    v[12 + k] = carF(E, a, s, CW_ROTMAT + 3 * k + 1);
                    v[15 + k] = carF(E, a, s, CW_ROTMAT + 3 * k + 2);
                }
                for (int k = 0; k < 18; k++) S.in[o + k][la] = v[k];
                continue;
            }
            const int T = E.teamSize[a], base = E.carOffset[a];
            const float boost = carF(E, a, s, CW_BOOST), airSinceJump = carF(E, a, s, CW_AIRSJ);
            const float wcnZ = carF(E, a, s, CW_WCN + 2);
            const uint32_t cf = carW(E, a, s, CW_FLAGS);
            if (s >= 2 * T) continue;
            const int rb = base - row0;
            if (s == 0) {
                S.rowBase[la] = (uint8_t)rb;
                S.team[la] = (uint8_t)T;
            }
            S.rowOf[rb + s] = (uint8_t)(la | (s << 4));
            S.in[o + 18][la] = boost;
            const bool ground = cf & CF_ON_GROUND;
            // CarState::HasFlipOrJump (Car.cpp:285-289)
            const bool flipJump = ground || (!(cf & CF_HAS_FLIPPED) && !(cf & CF_HAS_DOUBLE_JUMPED) &&
                                             airSinceJump < DOUBLEJUMP_MAX_DELAY);
            const uint32_t of = (ground ? OF_GROUND : 0u) | (flipJump ? OF_FLIPJUMP : 0u) |
                                ((cf & CF_DEMOED) ? OF_DEMOED : 0u) | ((cf & CF_HAS_JUMPED) ? OF_JUMPED : 0u);
            S.in[o + 19][la] = __uint_as_float(of);
            // DefaultAction::GetActionMask
            const bool turtled = (cf & CF_WORLD_CONTACT) && wcnZ > 0.9f;
            for (int w = 0; w < 3; w++) {
                uint32_t m = ground ? Tb.ground[w] : Tb.air[w];
                if (boost == 0.f) m &= ~Tb.boost[w];
                if (flipJump || turtled) m |= Tb.jump[w];
                S.in[OI_MASK + s * 3 + w][la] = __uint_as_float(m);
            }
            // the step's action (EnvSet passes the parsed Action as prevAction)
            const CtlRec c = E.controls[base + s];
            float* r = st + (rb + s) * stride + OBS_COL_PREV;
            for (int k = 0; k < 5; k++) r[k] = c.v[k];
            r[5] = c.jump ? 1.f : 0.f;
            r[6] = c.boost ? 1.f : 0.f;
            r[7] = c.handbrake ? 1.f : 0.f;
        } else if (i < nCar + nBall) {
            // ball word w in both frames, into the first 9 columns of every row
            const int j = i - nCar, la = j % OBS_ARENAS, w = j / OBS_ARENAS, a = a0 + la;
            if (la >= na) continue;
            const int k = w % 3;
            const float v = w < 3 ? ballF(E, a, BW_POS + k) * kBtToUu
                                  : (w < 6 ? ballF(E, a, BW_LIN + k) * kBtToUu : ballF(E, a, BW_ANG + k));
            if (w < 6) S.in[OI_BALL + w][la] = v;
            const float blue = v * (w < 3 ? OBS_POS : (w < 6 ? OBS_VEL : OBS_ANG));
            const float orange = k < 2 ? -blue : blue;
            const int T = E.teamSize[a];
            float* r = st + (E.carOffset[a] - row0) * stride + w;
            for (int p = 0; p < 2 * T; p++) r[p * stride] = p < T ? blue : orange;
        } else {
            // boost pads in RLGymCPP order; GameState::GetBoostPadTimers returns the mirrored
            // timers for the blue frame and the direct ones for the orange frame
            // (GameState.h:56-62), and AdvancedObs pairs them with the frame's pads
            const int j = i - nCar - nBall, la = j % OBS_ARENAS, pi = j / OBS_ARENAS, a = a0 + la;
            if (la >= na) continue;
            const int d = Tb.padMap[pi], m = Tb.padMap[NUM_PADS - 1 - pi];
            const float coolD = __uint_as_float(E.pad[(size_t)d * E.N + a]);
            const float coolM = __uint_as_float(E.pad[(size_t)m * E.N + a]);
            const bool actD = E.pad[((size_t)NUM_PADS + d) * E.N + a] & 1u;
            const bool actM = E.pad[((size_t)NUM_PADS + m) * E.N + a] & 1u;
            const float blue = actD ? 1.f : 1.f / (1.f + coolM);
            const float orange = actM ? 1.f : 1.f / (1.f + coolD);
            const int T = E.teamSize[a];
            float* r = st + (E.carOffset[a] - row0) * stride + OBS_COL_PAD + pi;
            for (int p = 0; p < 2 * T; p++) r[p * stride] = p < T ? blue : orange;
        }
    }
    __syncthreads();

    // ---- B
    int tmin = RSB_MAX_TEAM_SIZE;
    for (int la = 0; la < na; la++) tmin = min(tmin, (int)S.team[la]);
    const int zcols = stride - (OBS_COL_CAR + 2 * RSB_OBS_PER_CAR * tmin);  // padding of the smallest arenas
    const int nMask = rows / 2 * 45;  // a pair of rows is 180 mask bytes: 45 words
    const int nZero = zcols > 0 ? rows * zcols : 0;
    uint32_t* mout = reinterpret_cast<uint32_t*>(E.masks + (size_t)row0 * RSB_NUM_ACTIONS);
    constexpr int nView = 2 * OBS_ARENAS * MAX_CARS * RSB_MAX_TEAM_SIZE;  // (arena, car, frame, viewer)
    for (int i = tid; i < nView + nMask + nZero; i += OBS_THREADS) {
        if (i < nView) {
            // car q's block in frame f, into the row of viewer v of that frame's team
            const int la = i % OBS_ARENAS, q = (i / OBS_ARENAS) % MAX_CARS, f = (i / (OBS_ARENAS * MAX_CARS)) & 1,
                      v = i / (2 * OBS_ARENAS * MAX_CARS);
            if (la >= na) continue;
            const int T = S.team[la];
            if (q >= 2 * T || v >= T) continue;
            const int p = f * T + v;
            obsCarBlock(S, la, q, f == 1,
                        st + (S.rowBase[la] + p) * stride + OBS_COL_CAR + RSB_OBS_PER_CAR * obsCarIndex(T, p, q));
        } else if (i < nView + nMask) {
            // mask word w of row pair k (rows 2k, 2k+1: one arena, slots s, s + 1)
            const int j = i - nView, k = j / 45, w = j - 45 * k;
            const int ro = S.rowOf[2 * k], la = ro & 15, s = ro >> 4;
            const int sm = OI_MASK + s * 3;
            uint32_t word;
            if (w < 22) {
                word = maskNibbleBytes(__float_as_uint(S.in[sm][la]), __float_as_uint(S.in[sm + 1][la]),
                                       __float_as_uint(S.in[sm + 2][la]), 4 * w);
            } else if (w > 22) {
                word = maskNibbleBytes(__float_as_uint(S.in[sm + 3][la]), __float_as_uint(S.in[sm + 4][la]),
                                       __float_as_uint(S.in[sm + 5][la]), 4 * (w - 23) + 2);
            } else {
                // bytes 88, 89 of the first row, 0, 1 of the second
                const uint32_t x = ((__float_as_uint(S.in[sm + 2][la]) >> 24) & 3u) |
                                   ((__float_as_uint(S.in[sm + 3][la]) & 3u) << 2);
                word = (x * 0x00204081u) & 0x01010101u;
            }
            mout[j] = word;
        } else {
            // zero columns after the last car block of arenas smaller than the largest
            const int j = i - nView - nMask, r = j / zcols, c = stride - zcols + (j - r * zcols);
            const int la = S.rowOf[r] & 15;
            if (c >= OBS_COL_CAR + 2 * RSB_OBS_PER_CAR * S.team[la]) st[r * stride + c] = 0.f;
        }
    }
    // the staged rows are read by the bulk copy (async proxy) next
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    // ---- C
    const int total = rows * stride;
    const int e0 = min(total, (4 - mis) & 3);
    const int e1 = e0 + ((total - e0) & ~3);
    if (tid == 0 && e1 > e0) {
        const uint32_t src = (uint32_t)__cvta_generic_to_shared(st + e0);
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                     :: "l"(out + e0), "r"(src), "r"((e1 - e0) * 4) : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
    if (tid < e0) out[tid] = st[tid];
    else if (tid >= 4 && tid - 4 < total - e1) out[e1 + tid - 4] = st[e1 + tid - 4];
    // the shared memory must outlive the copy's reads of it; the writes complete with the grid
    if (tid == 0 && e1 > e0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// The seed counter of a captured env step: advanced once per replay.
__global__ void advanceSeedKernel(uint64_t* seed) { *seed += 1; }

// ------------------------------------------------------------------ rewards and terminals

__global__ void rewardKernel(EnvView E, RewardParams R, int stepTicks) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= E.N) return;
    const int T = E.teamSize[a], M = 2 * T, base = E.carOffset[a];
    const float bx = ballF(E, a, BW_POS + 0) * kBtToUu, by = ballF(E, a, BW_POS + 1) * kBtToUu,
                bz = ballF(E, a, BW_POS + 2) * kBtToUu;
    const float bvx = ballF(E, a, BW_LIN + 0) * kBtToUu, bvy = ballF(E, a, BW_LIN + 1) * kBtToUu,
                bvz = ballF(E, a, BW_LIN + 2) * kBtToUu;
    const uint64_t tick = (uint64_t)E.arena[(size_t)AW_TICK * E.N + a] |
                          ((uint64_t)E.arena[(size_t)(AW_TICK + 1) * E.N + a] << 32);
    // GameState::UpdateFromArena: tickSkip = ticks since the last update
    const uint64_t skip = min((uint64_t)(stepTicks > 0 ? stepTicks : 0), tick);
    bool touched[MAX_CARS];
    bool anyTouch = false;
    for (int s = 0; s < M; s++) {
        const uint32_t cf = carW(E, a, s, CW_FLAGS);
        const uint64_t hit = (uint64_t)carW(E, a, s, CW_HIT) | ((uint64_t)carW(E, a, s, CW_HIT + 1) << 32);
        touched[s] = (cf & CF_BALL_HIT_VALID) && hit >= tick - skip;
        anyTouch |= touched[s];
    }
    // Arena::IsBallScored (Arena.cpp:949-957)
    const bool goal = fabsf(by) > (R.goalBaseY + R.ballRadius);

    // terminals (EnvSet.cpp:184-205): a normal terminal beats a truncation
    uint8_t type = 0;
    if (R.noTouchTimeout > 0.f) {
        float t = __uint_as_float(E.arena[(size_t)AW_NOTOUCH * E.N + a]);
        if (anyTouch) {
            t = 0.f;
        } else {
            t += (float)(int)skip * (1 / 120.f);
            if (t >= R.noTouchTimeout) type = 2;
        }
        E.arena[(size_t)AW_NOTOUCH * E.N + a] = __float_as_uint(t);
    }
    if (R.episodeMaxTicks > 0 && (int32_t)E.arena[(size_t)AW_EPISODE * E.N + a] >= R.episodeMaxTicks && type == 0)
        type = 2;
    if (goal) type = 1;
    E.terminals[a] = type;

    float all[MAX_CARS];
    for (int s = 0; s < M; s++) all[s] = 0.f;
    for (int k = 0; k < 4; k++) {
        if (R.w[k] == 0.f) continue;
        float out[MAX_CARS];
        for (int s = 0; s < M; s++) {
            const bool orange = s >= T;
            float r;
            if (k == 0) {
                // GoalReward: RS_TEAM_FROM_Y(ball y) is the team whose half holds the ball
                r = goal ? ((orange != (by >= 0.f)) ? 1.f : R.concede) : 0.f;
            } else if (k == 1) {
                r = touched[s] ? 1.f : 0.f;
            } else if (k == 2) {
                // VelocityBallToGoalReward: toward CommonValues::ORANGE_GOAL_BACK for blue
                const float tx = 0.f, ty = orange ? -CV_BACK_NET_Y : CV_BACK_NET_Y, tz = CV_GOAL_HEIGHT / 2;
                float dx = tx - bx, dy = ty - by, dz = tz - bz;
                float l2 = vdot4(dx, dy, dz, dx, dy, dz);
                float l = l2 > 0.f ? sqrtf(l2) : 0.f;
                if (l > kEpsilon * kEpsilon) { dx = dx / l; dy = dy / l; dz = dz / l; }
                else { dx = dy = dz = 0.f; }
                r = vdot4(dx, dy, dz, bvx / CV_BALL_MAX_SPEED, bvy / CV_BALL_MAX_SPEED, bvz / CV_BALL_MAX_SPEED);
            } else {
                // VelocityPlayerToBallReward
                const float px = carF(E, a, s, CW_POS + 0) * kBtToUu, py = carF(E, a, s, CW_POS + 1) * kBtToUu,
                            pz = carF(E, a, s, CW_POS + 2) * kBtToUu;
                const float vx = carF(E, a, s, CW_LIN + 0) * kBtToUu, vy = carF(E, a, s, CW_LIN + 1) * kBtToUu,
                            vz = carF(E, a, s, CW_LIN + 2) * kBtToUu;
                float dx = bx - px, dy = by - py, dz = bz - pz;
                float l2 = vdot4(dx, dy, dz, dx, dy, dz);
                float l = l2 > 0.f ? sqrtf(l2) : 0.f;
                if (l > kEpsilon * kEpsilon) { dx = dx / l; dy = dy / l; dz = dz / l; }
                else { dx = dy = dz = 0.f; }
                r = vdot4(dx, dy, dz, vx / CV_CAR_MAX_SPEED, vy / CV_CAR_MAX_SPEED, vz / CV_CAR_MAX_SPEED);
            }
            out[s] = r;
        }
        if (R.zeroSum & (1 << k)) {
            // ZeroSumReward::GetAllRewards over the players in Arena::_cars order
            int cnt[2] = {0, 0};
            float avg[2] = {0.f, 0.f};
            for (int s = M - 1; s >= 0; s--) {
                const int t = s >= T;
                cnt[t]++;
                avg[t] += out[s];
            }
            for (int t = 0; t < 2; t++) avg[t] /= (float)(cnt[t] > 1 ? cnt[t] : 1);
            for (int s = 0; s < M; s++) {
                const int t = s >= T;
                out[s] = out[s] * (1 - R.teamSpirit) + (avg[t] * R.teamSpirit) - (avg[1 - t] * R.oppScale);
            }
        }
        for (int s = 0; s < M; s++) all[s] += out[s] * R.w[k];
    }
    for (int s = 0; s < M; s++) E.rewards[base + s] = all[s];
}

// ------------------------------------------------------------------ resets

// Counter-based draws for the resets: splitmix64 of (seed, arena, counter).
struct ResetRng {
    uint64_t key;
    uint32_t ctr;
    RSB_D uint32_t next() {
        uint64_t z = key + 0x9E3779B97F4A7C15ull * (uint64_t)(++ctr);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return (uint32_t)((z ^ (z >> 31)) >> 32);
    }
    // RocketSim Math::RandFloat: min + u * (max - min), u in [0, 1]
    RSB_D float uni(float lo, float hi) { return lo + ((float)(next() >> 8) * (1.f / 16777216.f)) * (hi - lo); }
};

RSB_D V3 randNormVec(ResetRng& g) {
    V3 v{g.uni(-1, 1), g.uni(-1, 1), g.uni(-1, 1)};
    return rsNormalized(v);
}

RSB_D void putCarW(const EnvView& E, int a, int s, int w, uint32_t v) {
    E.car[((size_t)w * MAX_CARS + s) * E.N + a] = v;
}
RSB_D void putCarF(const EnvView& E, int a, int s, int w, float v) { putCarW(E, a, s, w, __float_as_uint(v)); }

// Car::SetState of a default CarState with the given placement (Car.cpp:23-36,
// Car.h:15-100): the transform, the velocities and every CarState field are replaced;
// the broadphase registration and the vehicle's wheel values are kept.
RSB_D void resetCarFlags(const EnvView& E, int a, int s, V3 posUu, const M3& rot, V3 velUu, V3 ang, float boost,
                         uint32_t flags) {
    // the team and the body's contact-response flag survive Car::SetState
    const uint32_t team = carW(E, a, s, CW_FLAGS) & (CF_TEAM_ORANGE | CF_NO_RESPONSE);
    const V3 p = posUu * kUuToBt, v = velUu * kUuToBt;
    const float pv[3] = {p.x, p.y, p.z}, vv[3] = {v.x, v.y, v.z}, av[3] = {ang.x, ang.y, ang.z};
    for (int k = 0; k < 3; k++) {
        putCarF(E, a, s, CW_POS + k, pv[k]);
        putCarF(E, a, s, CW_LIN + k, vv[k]);
        putCarF(E, a, s, CW_ANG + k, av[k]);
        putCarF(E, a, s, CW_ROT + 3 * k + 0, rot.r[k].x);
        putCarF(E, a, s, CW_ROT + 3 * k + 1, rot.r[k].y);
        putCarF(E, a, s, CW_ROT + 3 * k + 2, rot.r[k].z);
    }
    // CarState words (boost .. lastCtlBits): defaults, then the placement
    for (int w = CW_STATE0; w < CW_STATE1; w++) putCarW(E, a, s, w, 0u);
    putCarF(E, a, s, CW_BOOST, boost);
    putCarW(E, a, s, CW_FLAGS, flags | team);
    for (int k = 0; k < 2; k++) {
        putCarW(E, a, s, CW_HIT + k, 0xffffffffu);
        putCarW(E, a, s, CW_HITX + k, 0xffffffffu);
    }
    for (int k = 0; k < 3; k++) {
        putCarF(E, a, s, CW_ROTMAT + 3 * k + 0, rot.r[k].x);
        putCarF(E, a, s, CW_ROTMAT + 3 * k + 1, rot.r[k].y);
        putCarF(E, a, s, CW_ROTMAT + 3 * k + 2, rot.r[k].z);
    }
}

RSB_D void resetCar(const EnvView& E, int a, int s, V3 posUu, const M3& rot, V3 velUu, V3 ang, float boost) {
    resetCarFlags(E, a, s, posUu, rot, velUu, ang, boost, CF_ON_GROUND);
}

// Weights of the curriculum reset (RocketSimCudaBatch::SetResetCurriculum) and the no-touch
// timeout whose timer it staggers.
struct ResetCurriculum {
    float w[4];  // kickoff, fuzzed kickoff, aerial, ball chase
    float noTouchTimeout;
};

RSB_D M3 rowsToM3(const float* r) { return m3(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8]); }

// Angle(yaw, pitch, roll).ToRotMat() = btMatrix3x3::setEulerYPR(yaw, -pitch, -roll)
// (MathTypes.cpp:73-78)
RSB_D M3 angleRot(float yaw, float pitch, float roll) { return m3fromEulerZYX(-roll, -pitch, yaw); }

// Arena i of the list `idx` (every arena when idx is null; with `onlyDone`, only the
// arenas whose terminal flag is set).
__global__ void resetKernel(EnvView E, EnvTables Tb, ResetCurriculum Cu, const int32_t* idx, int n, uint64_t seed,
                            int mode, bool onlyDone, const uint64_t* seedPtr = nullptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (seedPtr) seed = *seedPtr;  // a replayed graph reads the seed of this launch from the device
    const int a = idx ? idx[i] : i;
    if (onlyDone && E.terminals[a] == 0) return;
    if (E.vantaArena) {
        for (int w = 0; w < VANTA_ARENA_WORDS; w++) E.vantaArena[(size_t)w * E.N + a] = 0u;
        for (int w = 0; w < VANTA_CAR_WORDS * MAX_CARS; w++) E.vantaCar[(size_t)w * E.N + a] = 0u;
    }
    const int T = E.teamSize[a], M = 2 * T, base = E.carOffset[a];
    ResetRng g{seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(a + 1)), 0};
    constexpr float PI = 3.14159265358979323846f;
    // curriculum: 0 kickoff, 1 fuzzed kickoff, 2 aerial, 3 ball chase, drawn by weight
    // (RocketSimCudaBatch::ResetArena, RocketSimCudaApi.cuh:216-245)
    int cur = -1;
    if (mode == RSB_RESET_CURRICULUM) {
        const float tot = Cu.w[0] + Cu.w[1] + Cu.w[2] + Cu.w[3];
        const float r = g.uni(0.f, 1.f) * tot;
        cur = r < Cu.w[0] ? 0 : (r < Cu.w[0] + Cu.w[1] ? 1 : (r < Cu.w[0] + Cu.w[1] + Cu.w[2] ? 2 : 3));
    }
    auto sgn = [&](float amp) { return g.uni(-amp, amp); };

    // kickoff layout (always applied first, as RandomState does): a shuffled spawn per
    // kickoff rank, rank i of each team taking the i-th car in Arena::_cars order
    int order[NUM_KICKOFF_SPAWNS] = {0, 1, 2, 3, 4};
    for (int k = NUM_KICKOFF_SPAWNS - 1; k > 0; k--) {
        int j = (int)(g.next() % (uint32_t)(k + 1));
        int t = order[k]; order[k] = order[j]; order[j] = t;
    }
    for (int r = 0; r < T; r++) {
        const int sp = order[r];
        for (int team = 0; team < 2; team++) {
            const int s = team * T + (T - 1 - r);
            V3 pos{Tb.kickX[sp], Tb.kickY[sp], CAR_SPAWN_REST_Z};
            if (team) pos = pos * V3{-1.f, -1.f, 1.f};
            if (cur == 1) {  // fuzzed kickoff: the slot and yaw kept, the position moved a little
                pos.x += sgn(40.f);
                pos.y += sgn(40.f);
            }
            resetCar(E, a, s, pos, rowsToM3(Tb.kickRot[team][sp]), v3zero(), v3zero(), BOOST_SPAWN_AMOUNT);
        }
    }
    V3 ballPos{0.f, 0.f, BALL_REST_Z}, ballVel = v3zero(), ballAng = v3zero();

    if (mode == RSB_RESET_RANDOM_STATE) {
        // RandomState(randBallSpeed, randCarSpeed, carsOnGround = false)
        const float X = 3500.f, Y = 4000.f, Z = 1820.f;
        ballPos = V3{g.uni(-X, X), g.uni(-Y, Y), g.uni(CV_BALL_RADIUS, Z)};
        ballVel = randNormVec(g) * g.uni(0.f, 4000.f);
        ballAng = V3{g.uni(-4.f, 4.f), g.uni(-4.f, 4.f), g.uni(-4.f, 4.f)};
        for (int s = M - 1; s >= 0; s--) {
            V3 pos{g.uni(-X, X), g.uni(-Y, Y), g.uni(150.f, Z)};
            V3 vel = randNormVec(g) * g.uni(0.f, CV_CAR_MAX_SPEED);
            V3 ang = randNormVec(g) * 5.5f;
            float yaw = g.uni(-PI, PI), pitch = g.uni(-PI / 2, PI / 2), roll = g.uni(-PI, PI);
            const bool onGround = g.uni(0.f, 1.f) > 0.5f;
            if (onGround) {
                pos.z = CAR_SPAWN_REST_Z;
                pitch = roll = 0.f;
                vel.z = 0.f;
                ang = v3zero();
            }
            resetCar(E, a, s, pos, angleRot(yaw, pitch, roll), vel, ang, g.uni(0.f, 100.f));
        }
    } else if (cur == 1) {
        // fuzzed kickoff: the ball a little off the spot with a mild velocity
        ballPos = V3{sgn(180.f), sgn(220.f), BALL_REST_Z};
        ballVel = V3{sgn(90.f), sgn(90.f), sgn(35.f)};
    } else if (cur == 2) {
        // aerial: the ball raised near midfield, one car below it moving toward it
        ballPos = V3{sgn(1400.f), sgn(1600.f), 420.f + g.uni(0.f, 360.f)};
        ballVel = V3{sgn(100.f), sgn(100.f), sgn(50.f)};
        const int s = (int)(g.uni(0.f, 1.f) * (float)M) % M;
        V3 d{sgn(1.f), sgn(1.f), 0.f};
        float len = sqrtf(d.x * d.x + d.y * d.y);
        if (len < 1e-3f) { d = V3{1.f, 0.f, 0.f}; len = 1.f; }
        d = V3{d.x / len, d.y / len, 0.f};
        const float dist = 180.f + g.uni(0.f, 160.f);
        V3 pos{ballPos.x - d.x * dist, ballPos.y - d.y * dist, ballPos.z - (40.f + g.uni(0.f, 120.f))};
        if (pos.z < CAR_SPAWN_REST_Z) pos.z = CAR_SPAWN_REST_Z + 80.f;
        const float yaw = rsAtan2f(ballPos.y - pos.y, ballPos.x - pos.x);
        const float spd = 500.f + g.uni(0.f, 400.f);
        const V3 vel{d.x * spd, d.y * spd, 80.f + g.uni(0.f, 120.f)};
        const bool jumped = g.uni(0.f, 1.f) < 0.55f;
        resetCarFlags(E, a, s, pos, angleRot(yaw, 0.f, 0.f), vel, v3zero(), 55.f + g.uni(0.f, 45.f),
                      jumped ? CF_HAS_JUMPED : 0u);
    } else if (cur == 3) {
        // ball chase: the ball in play on the ground, every car near it on the ground facing it
        ballPos = V3{sgn(1900.f), sgn(2200.f), BALL_REST_Z};
        ballVel = V3{sgn(500.f), sgn(500.f), sgn(80.f)};
        for (int s = 0; s < M; s++) {
            V3 d{sgn(1.f), sgn(1.f), 0.f};
            float len = sqrtf(d.x * d.x + d.y * d.y);
            if (len < 1e-3f) { d = V3{1.f, 0.f, 0.f}; len = 1.f; }
            d = V3{d.x / len, d.y / len, 0.f};
            const float dist = 450.f + g.uni(0.f, 1400.f);
            V3 pos{fminf(fmaxf(ballPos.x + d.x * dist, -3500.f), 3500.f),
                   fminf(fmaxf(ballPos.y + d.y * dist, -4500.f), 4500.f), CAR_SPAWN_REST_Z};
            const float yaw = rsAtan2f(ballPos.y - pos.y, ballPos.x - pos.x);
            const float spd = g.uni(0.f, 600.f);
            const float tx = ballPos.x - pos.x, ty = ballPos.y - pos.y, tl = sqrtf(tx * tx + ty * ty);
            const V3 vel = tl > 1.f ? V3{tx / tl * spd, ty / tl * spd, 0.f} : v3zero();
            resetCar(E, a, s, pos, angleRot(yaw, 0.f, 0.f), vel, v3zero(), 30.f + g.uni(0.f, 70.f));
        }
    } else if (mode == RSB_RESET_HIGH_CONTACT) {
        // cars within 300 uu of the ball or of another car, 1500-2300 uu/s toward it,
        // half airborne; some start on a side wall or under the ceiling
        ballPos = V3{g.uni(-3000.f, 3000.f), g.uni(-3600.f, 3600.f), g.uni(CV_BALL_RADIUS, 1200.f)};
        ballVel = randNormVec(g) * g.uni(0.f, 1500.f);
        V3 prev = ballPos;
        bool prevFree = false;  // the previous car is a free start (a valid anchor)
        for (int s = M - 1; s >= 0; s--) {
            const V3 anchor = (prevFree && g.uni(0.f, 1.f) >= 0.5f) ? prev : ballPos;
            const float kind = g.uni(0.f, 1.f);
            V3 pos;
            float pitch = 0.f, roll = 0.f;
            bool air = g.uni(0.f, 1.f) < 0.5f;
            const bool free = kind >= 0.15f;
            if (kind < 0.1f) {
                // side wall start, wheels on the wall
                const float side = g.uni(0.f, 1.f) < 0.5f ? -1.f : 1.f;
                pos = V3{side * 4000.f, g.uni(-3500.f, 3500.f), g.uni(300.f, 1500.f)};
                roll = side * (PI / 2);
                air = true;
            } else if (!free) {
                // under the ceiling, upside down
                pos = V3{g.uni(-3000.f, 3000.f), g.uni(-3800.f, 3800.f), 1950.f};
                roll = PI;
                air = true;
            } else {
                // within 150-300 uu (horizontally) of the anchor
                const float r = g.uni(150.f, 300.f), t = g.uni(-PI, PI);
                pos = V3{anchor.x + r * rsCosf(t), anchor.y + r * rsSinf(t), 0.f};
                pos.z = air ? fminf(fmaxf(anchor.z + g.uni(-300.f, 300.f), 150.f), 1900.f) : CAR_SPAWN_REST_Z;
            }
            V3 to = anchor - pos;
            if (!air) to.z = 0.f;
            V3 dir = rsNormalized(to);
            if (dir == v3zero()) dir = V3{1.f, 0.f, 0.f};
            const V3 vel = dir * g.uni(1500.f, 2300.f);
            const float yaw = rsAtan2f(dir.y, dir.x);
            if (air && free) pitch = g.uni(-PI / 4, PI / 4);
            resetCar(E, a, s, pos, angleRot(yaw, pitch, roll), vel, v3zero(), g.uni(0.f, 100.f));
            prev = pos;
            prevFree = free;
        }
    }

    // Ball::SetState (Ball.cpp:35-49) of a BallState with that placement
    uint32_t* ball = E.ball;
    const V3 bp = ballPos * kUuToBt, bv = ballVel * kUuToBt;
    const float bpv[3] = {bp.x, bp.y, bp.z}, bvv[3] = {bv.x, bv.y, bv.z}, bav[3] = {ballAng.x, ballAng.y, ballAng.z};
    for (int k = 0; k < 3; k++) {
        ball[(size_t)(BW_POS + k) * E.N + a] = __float_as_uint(bpv[k]);
        ball[(size_t)(BW_LIN + k) * E.N + a] = __float_as_uint(bvv[k]);
        ball[(size_t)(BW_ANG + k) * E.N + a] = __float_as_uint(bav[k]);
        for (int c = 0; c < 3; c++) ball[(size_t)(BW_ROT + 3 * k + c) * E.N + a] = __float_as_uint(k == c ? 1.f : 0.f);
    }
    // BoostPad::SetState(BoostPadState())
    uint32_t* pad = E.pad;
    for (int p = 0; p < NUM_PADS; p++) {
        pad[((size_t)0 * NUM_PADS + p) * E.N + a] = __float_as_uint(0.f);
        pad[((size_t)1 * NUM_PADS + p) * E.N + a] = 1u;
    }
    E.arena[(size_t)AW_EPISODE * E.N + a] = 0;
    E.arena[(size_t)AW_STATUS * E.N + a] = 0;
    E.arena[(size_t)AW_GOALTEAM * E.N + a] = (uint32_t)-1;
    E.arena[(size_t)AW_TOUCHED * E.N + a] = 0;
    // the curriculum staggers the no-touch timers so that arenas reset together do not all
    // time out on the same step (RocketSimCudaApi.cuh:417-427)
    E.arena[(size_t)AW_NOTOUCH * E.N + a] =
        (cur >= 0 && Cu.noTouchTimeout > 0.f) ? __float_as_uint(g.uni(0.f, 1.f) * Cu.noTouchTimeout * 0.9f) : 0u;
    // every reset places the ball inside the field (|y| <= 4000 uu), short of a goal line
    E.arena[(size_t)AW_SCORED * E.N + a] = 0;
    // the new state's players carry default (zero) actions
    for (int s = 0; s < M; s++) E.controls[base + s] = CtlRec{};
}

}  // namespace rsb
