// REFERENCE VANTAOBS BUILDER — test infrastructure only.  Compiles the reference's own device
// builder (RocketSimCuda/src/VantaObsGpu.cuh, with RocketSimCuda/src/GpuTypes.cuh) from where
// it lies in the reference tree (oracle/Makefile) and drives it with the engine's state, so that
// the engine's VantaObs rows can be checked against it on identical inputs.  The reference tree
// holds no CPU VantaObs (RLGymCPP/OBSBuilders/VantaObs.h is not in it), so this device builder
// is the pin.  Nothing in the product links this file.
//
// What the harness adds around the reference's device functions is the reference batch's own
// glue, restated: the two kernels of RocketSimCudaBatch::BuildVantaObs
// (RocketSimCudaObs.cuh:70-186: the per-arena update with the ball-prediction slices, and the
// per-player row with the last-touch search) and the pad tables of initTrainingConstantMemory
// (RocketSimCudaHostUtils.cuh:56-91).  The ball-prediction slices are an input here (the engine's
// own, pinned separately against RocketSim's ball-only arenas): this checks the row assembly.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "GpuTypes.cuh"
#include "VantaObsGpu.cuh"
#include "rsb.h"

using namespace rsc;

namespace {

// RLGym pad order -> the reference batch's pad index (RocketSimCudaHostUtils.cuh:56-59)
const int kRefPadMap[BoostPadData::NUM_TOTAL] = {0,  1,  2,  32, 33, 3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 28, 13,
                                                 14, 29, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 30, 31, 25, 26, 27};

struct Pin {
    int n = 0, maxCars = 0;
    GpuVantaArenaState* va = nullptr;
    GpuVantaTimers* vt = nullptr;
    GpuCarState* cars = nullptr;
    GpuBallState* balls = nullptr;
    GpuBoostPadState* pads = nullptr;
    int* numCars = nullptr;
    uint64_t* ticks = nullptr;
    Vec3* pred = nullptr;  // [n][3] pos, then [n][3] vel
    int* padMap = nullptr;
    Vec3* locs = nullptr;
    int* mirror = nullptr;
    int* rowOf = nullptr;  // flat player -> packed row, -1 for an empty slot
    float* rows = nullptr;
};

// vantaArenaUpdateKernel (RocketSimCudaObs.cuh:70-126) with the slices given
__global__ void pinArenaKernel(Pin P, int usePred, float dt) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n) return;
    GpuVantaArenaState& va = P.va[a];
    if (usePred) {
        for (int k = 0; k < 3; k++) {
            va.predPos[k] = P.pred[a * 3 + k];
            va.predVel[k] = P.pred[(P.n + a) * 3 + k];
        }
        va.hasPred = 1;
    } else {
        va.hasPred = 0;
    }
    vanta_update_arena(va, &P.vt[a * P.maxCars], &P.cars[a * P.maxCars], P.numCars[a],
                       &P.pads[a * BoostPadData::NUM_TOTAL], P.padMap, P.locs, P.ticks[a], dt);
}

// vantaObsKernel (RocketSimCudaObs.cuh:128-186), rows written packed
__global__ void pinRowKernel(Pin P, float dt, float deadzone, int onlyClosestOpp) {
    const int flat = blockIdx.x * blockDim.x + threadIdx.x;
    if (flat >= P.n * P.maxCars) return;
    const int a = flat / P.maxCars, c = flat % P.maxCars;
    if (c >= P.numCars[a] || P.rowOf[flat] < 0) return;
    const GpuCarState* cars = &P.cars[a * P.maxCars];
    uint32_t lastTouch = 0;
    uint64_t best = 0;
    for (int i = 0; i < P.numCars[a]; i++) {
        if (cars[i].ballHitValid && cars[i].ballHitTickCount != ~0ULL && cars[i].ballHitTickCount >= best) {
            best = cars[i].ballHitTickCount;
            lastTouch = cars[i].id;
        }
    }
    vanta_build_obs(P.rows + (size_t)P.rowOf[flat] * VantaConst::TOTAL_OBS_SIZE, cars, P.numCars[a], c,
                    P.balls[a], P.va[a], &P.vt[a * P.maxCars], P.padMap, P.locs, P.mirror, lastTouch, P.ticks[a],
                    dt, deadzone, onlyClosestOpp != 0);
}

Vec3 v3of(const rsb_vec3& v) { return Vec3{v.x, v.y, v.z}; }

template <class T>
bool upload(T* dst, const std::vector<T>& src) {
    return cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
}

}  // namespace

extern "C" {

// A builder for n arenas of at most max_cars cars, in its default (cleared) state.
void* vantaref_create(int32_t n, int32_t max_cars) {
    if (n <= 0 || max_cars < 2 || max_cars > 6) return nullptr;
    Pin* p = new Pin();
    p->n = n;
    p->maxCars = max_cars;
    const size_t F = (size_t)n * max_cars, NP = BoostPadData::NUM_TOTAL;
    bool ok = cudaMalloc(&p->va, n * sizeof(GpuVantaArenaState)) == cudaSuccess &&
              cudaMalloc(&p->vt, F * sizeof(GpuVantaTimers)) == cudaSuccess &&
              cudaMalloc(&p->cars, F * sizeof(GpuCarState)) == cudaSuccess &&
              cudaMalloc(&p->balls, n * sizeof(GpuBallState)) == cudaSuccess &&
              cudaMalloc(&p->pads, n * NP * sizeof(GpuBoostPadState)) == cudaSuccess &&
              cudaMalloc(&p->numCars, n * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&p->ticks, n * sizeof(uint64_t)) == cudaSuccess &&
              cudaMalloc(&p->pred, 6 * (size_t)n * sizeof(Vec3)) == cudaSuccess &&
              cudaMalloc(&p->padMap, NP * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&p->locs, NP * sizeof(Vec3)) == cudaSuccess &&
              cudaMalloc(&p->mirror, NP * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&p->rowOf, F * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&p->rows, F * VantaConst::TOTAL_OBS_SIZE * sizeof(float)) == cudaSuccess;
    if (ok) ok = cudaMemset(p->va, 0, n * sizeof(GpuVantaArenaState)) == cudaSuccess &&
                 cudaMemset(p->vt, 0, F * sizeof(GpuVantaTimers)) == cudaSuccess;
    if (ok) {
        // pad locations in RLGym order and their x-mirror permutation
        // (RocketSimCudaHostUtils.cuh:66-86)
        std::vector<int> map(kRefPadMap, kRefPadMap + NP), mirror(NP);
        std::vector<Vec3> locs(NP);
        for (size_t i = 0; i < NP; i++) locs[i] = BoostPadData::POSITIONS[kRefPadMap[i]];
        for (size_t i = 0; i < NP; i++) {
            int m = (int)i;
            for (size_t j = 0; j < NP; j++)
                if (std::fabs(locs[j].x + locs[i].x) < 1.f && std::fabs(locs[j].y - locs[i].y) < 1.f &&
                    std::fabs(locs[j].z - locs[i].z) < 1.f) {
                    m = (int)j;
                    break;
                }
            mirror[i] = m;
        }
        ok = upload(p->padMap, map) && upload(p->locs, locs) && upload(p->mirror, mirror);
    }
    if (!ok) {
        delete p;
        return nullptr;
    }
    return p;
}

void vantaref_destroy(void* h) {
    Pin* p = static_cast<Pin*>(h);
    if (!p) return;
    for (void* q : {(void*)p->va, (void*)p->vt, (void*)p->cars, (void*)p->balls, (void*)p->pads, (void*)p->numCars,
                    (void*)p->ticks, (void*)p->pred, (void*)p->padMap, (void*)p->locs, (void*)p->mirror,
                    (void*)p->rowOf, (void*)p->rows})
        cudaFree(q);
    delete p;
}

// ResetArena's clearing of the builder's state (RocketSimCudaApi.cuh:265-275).
int32_t vantaref_reset(void* h, const int32_t* idx, int32_t count) {
    Pin* p = static_cast<Pin*>(h);
    if (!p || (count > 0 && !idx)) return -1;
    for (int i = 0; i < count; i++) {
        const int a = idx[i];
        if (a < 0 || a >= p->n) return -1;
        if (cudaMemset(p->va + a, 0, sizeof(GpuVantaArenaState)) != cudaSuccess ||
            cudaMemset(p->vt + (size_t)a * p->maxCars, 0, p->maxCars * sizeof(GpuVantaTimers)) != cudaSuccess)
            return -2;
    }
    return 0;
}

// One BuildVantaObs on the given state.  cars: the engine's packed cars (car_offset[n] of them,
// creation order within each arena); pads: [n][34] in the order of pad_xyz (the engine's pad
// locations), mapped to the reference's pad order by location; pred: [n][3] ball states at
// 120 / 240 / 360 ticks, or null; ticks: each arena's tick count.  out: [car_offset[n]][366].
int32_t vantaref_build(void* h, const rsb_car_state* cars, const int32_t* car_offset, const rsb_ball_state* balls,
                       const rsb_pad_state* pads, const float* pad_xyz, const rsb_ball_state* pred,
                       const uint64_t* ticks, int32_t tick_skip, float deadzone, int32_t only_closest_opp,
                       float* out) {
    Pin* p = static_cast<Pin*>(h);
    if (!p || !cars || !car_offset || !balls || !pads || !pad_xyz || !ticks || !out || tick_skip <= 0) return -1;
    const int n = p->n, M = p->maxCars, NP = BoostPadData::NUM_TOTAL;
    // engine pad index of each reference pad, by location
    int ours[BoostPadData::NUM_TOTAL];
    for (int j = 0; j < NP; j++) {
        ours[j] = -1;
        for (int q = 0; q < NP; q++)
            if (std::fabs(pad_xyz[3 * q] - BoostPadData::POSITIONS[j].x) < 1.f &&
                std::fabs(pad_xyz[3 * q + 1] - BoostPadData::POSITIONS[j].y) < 1.f)
                ours[j] = q;
        if (ours[j] < 0) return -3;
    }
    std::vector<GpuCarState> gc((size_t)n * M);
    std::vector<int> num(n), rowOf((size_t)n * M, -1);
    std::vector<GpuBallState> gb(n);
    std::vector<GpuBoostPadState> gp((size_t)n * NP);
    std::vector<Vec3> pv(6 * (size_t)n);
    std::vector<uint64_t> tk(ticks, ticks + n);
    for (int a = 0; a < n; a++) {
        num[a] = car_offset[a + 1] - car_offset[a];
        if (num[a] < 0 || num[a] > M) return -1;
        for (int c = 0; c < num[a]; c++) {
            const rsb_car_state& s = cars[car_offset[a] + c];
            GpuCarState& g = gc[(size_t)a * M + c];
            std::memset(&g, 0, sizeof g);
            g.pos = v3of(s.pos);
            g.rotMat = RotMat{v3of(s.rot.forward), v3of(s.rot.right), v3of(s.rot.up)};
            g.vel = v3of(s.vel);
            g.angVel = v3of(s.ang_vel);
            g.boost = s.boost;
            g.isOnGround = s.is_on_ground;
            g.hasJumped = s.has_jumped;
            g.hasDoubleJumped = s.has_double_jumped;
            g.hasFlipped = s.has_flipped;
            g.isFlipping = s.is_flipping;
            g.isJumping = s.is_jumping;
            g.airTimeSinceJump = s.air_time_since_jump;
            g.isSupersonic = s.is_supersonic;
            g.handbrakeVal = s.handbrake_val;
            g.isDemoed = s.is_demoed;
            g.worldContactHasContact = s.world_contact;
            g.worldContactNormal = v3of(s.world_contact_normal);
            g.ballHitValid = s.ball_hit_valid;
            g.ballHitTickCount = s.ball_hit_tick;
            for (int w = 0; w < 4; w++) g.wheels[w].isInContact = s.wheels_with_contact[w] != 0;
            g.lastControls.throttle = s.last_controls.throttle;
            g.lastControls.steer = s.last_controls.steer;
            g.lastControls.pitch = s.last_controls.pitch;
            g.lastControls.yaw = s.last_controls.yaw;
            g.lastControls.roll = s.last_controls.roll;
            g.lastControls.jump = s.last_controls.jump != 0;
            g.lastControls.boost = s.last_controls.boost != 0;
            g.lastControls.handbrake = s.last_controls.handbrake != 0;
            g.team = s.team;
            g.id = s.id;
            rowOf[(size_t)a * M + c] = car_offset[a] + c;
        }
        std::memset(&gb[a], 0, sizeof gb[a]);
        gb[a].pos = v3of(balls[a].pos);
        gb[a].rotMat = RotMat{v3of(balls[a].rot.forward), v3of(balls[a].rot.right), v3of(balls[a].rot.up)};
        gb[a].vel = v3of(balls[a].vel);
        gb[a].angVel = v3of(balls[a].ang_vel);
        for (int j = 0; j < NP; j++) {
            GpuBoostPadState& g = gp[(size_t)a * NP + j];
            std::memset(&g, 0, sizeof g);
            g.isActive = pads[(size_t)a * NP + ours[j]].is_active != 0;
        }
        if (pred)
            for (int k = 0; k < 3; k++) {
                pv[(size_t)a * 3 + k] = v3of(pred[(size_t)a * 3 + k].pos);
                pv[((size_t)n + a) * 3 + k] = v3of(pred[(size_t)a * 3 + k].vel);
            }
    }
    if (!upload(p->cars, gc) || !upload(p->balls, gb) || !upload(p->pads, gp) || !upload(p->numCars, num) ||
        !upload(p->ticks, tk) || !upload(p->pred, pv) || !upload(p->rowOf, rowOf))
        return -2;
    const float dt = (float)tick_skip / 120.f;
    pinArenaKernel<<<(n + 63) / 64, 64>>>(*p, pred ? 1 : 0, dt);
    pinRowKernel<<<(n * M + 127) / 128, 128>>>(*p, dt, deadzone, only_closest_opp);
    const size_t rows = (size_t)car_offset[n];
    if (cudaMemcpy(out, p->rows, rows * VantaConst::TOTAL_OBS_SIZE * sizeof(float), cudaMemcpyDeviceToHost) !=
            cudaSuccess ||
        cudaGetLastError() != cudaSuccess)
        return -2;
    return 0;
}

}  // extern "C"
