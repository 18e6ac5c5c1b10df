// REFERENCE GPU COMPARATOR — test and benchmark infrastructure only.  Puts the reference's
// own batched GPU simulator, rsc::RocketSimCudaBatch (RocketSimCuda/include/RocketSimCuda.h:
// 258-455, stepArenaKernel in RocketSimCuda/src/RocketSimCudaPhysics.cuh:10-188), compiled
// for sm_100a from a scratch copy of its sources by oracle/Makefile, behind a few C entry
// points so that bench.py can time the reference's env step on the same B200 and the same
// workload as the engine.  Nothing in the product links this file.
//
// The reference's env step, as CudaEnvSet drives it (CudaEnvSet.cpp:378-421):
//   SnapshotTrainingState, SetDiscreteActionsFromIndices, Step(tickSkip),
//   BuildAdvancedObsAndDefaultMasks, BuildRewardsAndTerminals(tickSkip).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "RocketSimCuda.h"
#include "rsb.h"

namespace {

struct RefGpu {
    rsc::RocketSimCudaBatch batch;
    int n = 0, carsPerArena = 0, teamSize = 0;
};

rsc::Vec3 v3(const rsb_vec3& v) { return rsc::Vec3{v.x, v.y, v.z}; }

}  // namespace

extern "C" {

// N arenas of team_size v team_size (blue cars first, then orange, as rsb.h lays them out),
// reset to the reference's kickoff; meshes: the folder holding soccar/mesh_*.cmf.
void* rscref_create(int32_t n, int32_t team_size, const char* meshes) {
    if (n <= 0 || team_size < 1 || team_size > 3 || !meshes) return nullptr;
    RefGpu* r = new RefGpu();
    r->n = n;
    r->teamSize = team_size;
    r->carsPerArena = 2 * team_size;
    rsc::BatchConfig cfg;
    cfg.numArenas = n;
    cfg.maxCarsPerArena = r->carsPerArena;
    cfg.tickRate = 120.f;
    cfg.collisionMeshesPath = meshes;
    r->batch.Init(cfg);
    for (int a = 0; a < n; a++) {
        for (int t = 0; t < team_size; t++) r->batch.AddCar(a, rsc::Team::BLUE);
        for (int t = 0; t < team_size; t++) r->batch.AddCar(a, rsc::Team::ORANGE);
    }
    r->batch.ResetAllArenas();
    if (cudaDeviceSynchronize() != cudaSuccess) {
        delete r;
        return nullptr;
    }
    return r;
}

void rscref_destroy(void* h) { delete static_cast<RefGpu*>(h); }

// UploadDiscreteActionLut with rsb_controls entries.
int32_t rscref_set_lut(void* h, const rsb_controls* lut, int32_t count) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r || !lut || count <= 0) return -1;
    std::vector<rsc::CarControls> c((size_t)count);
    for (int i = 0; i < count; i++) {
        c[i].throttle = lut[i].throttle;
        c[i].steer = lut[i].steer;
        c[i].pitch = lut[i].pitch;
        c[i].yaw = lut[i].yaw;
        c[i].roll = lut[i].roll;
        c[i].jump = lut[i].jump != 0;
        c[i].boost = lut[i].boost != 0;
        c[i].handbrake = lut[i].handbrake != 0;
    }
    r->batch.UploadDiscreteActionLut(c.data(), count);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

// SetCarState / SetBallState of every car and ball from the rsb.h states (kinematics, boost,
// on-ground and jump flags); the other fields keep the reference's defaults.
int32_t rscref_set_states(void* h, const rsb_car_state* cars, const rsb_ball_state* balls) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r || !cars || !balls) return -1;
    std::vector<rsc::CarState> cur((size_t)r->n * r->carsPerArena);
    r->batch.GetAllCarStates(cur.data());  // team, id and preset of every car
    for (int a = 0; a < r->n; a++) {
        for (int c = 0; c < r->carsPerArena; c++) {
            const rsb_car_state& s = cars[(size_t)a * r->carsPerArena + c];
            rsc::CarState o = cur[(size_t)a * r->carsPerArena + c];
            o.pos = v3(s.pos);
            o.rotMat = rsc::RotMat{v3(s.rot.forward), v3(s.rot.right), v3(s.rot.up)};
            o.vel = v3(s.vel);
            o.angVel = v3(s.ang_vel);
            o.boost = s.boost;
            o.isOnGround = s.is_on_ground != 0;
            o.hasJumped = s.has_jumped != 0;
            o.hasDoubleJumped = s.has_double_jumped != 0;
            o.hasFlipped = s.has_flipped != 0;
            r->batch.SetCarState(a, c, o);
        }
        const rsb_ball_state& b = balls[a];
        rsc::BallState o;
        o.pos = v3(b.pos);
        o.rotMat = rsc::RotMat{v3(b.rot.forward), v3(b.rot.right), v3(b.rot.up)};
        o.vel = v3(b.vel);
        o.angVel = v3(b.ang_vel);
        r->batch.SetBallState(a, o);
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

// Runs warmup + steps env steps of `ticks` ticks (actions[s * num_players + p] for step s, the
// warm-up steps first) and returns the device time of the timed steps in *ms (CUDA events on
// the legacy stream the reference launches on, kernels chained without per-op sync).
int32_t rscref_time_env_steps(void* h, const int32_t* actions, int32_t warmup, int32_t steps, int32_t ticks,
                              float* ms) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r || !actions || warmup < 0 || steps <= 0 || ticks <= 0 || !ms) return -1;
    const int P = r->n * r->carsPerArena;
    r->batch.SetKernelSync(false);
    auto envStep = [&](int s) {
        r->batch.SnapshotTrainingState();
        r->batch.SetDiscreteActionsFromIndices(actions + (size_t)s * P, P);
        r->batch.Step(ticks);
        r->batch.BuildAdvancedObsAndDefaultMasks();
        r->batch.BuildRewardsAndTerminals(ticks);
    };
    for (int s = 0; s < warmup; s++) envStep(s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    for (int s = 0; s < steps; s++) envStep(warmup + s);
    cudaEventRecord(e1, 0);
    const cudaError_t e = cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    r->batch.SetKernelSync(true);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// SetAllCarControls with rsb_controls, then Step(ticks), synchronously.
int32_t rscref_step(void* h, const rsb_controls* ctl, int32_t ticks) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r || !ctl || ticks <= 0) return -1;
    std::vector<rsc::CarControls> c((size_t)r->n * r->carsPerArena);
    for (size_t i = 0; i < c.size(); i++) {
        c[i].throttle = ctl[i].throttle;
        c[i].steer = ctl[i].steer;
        c[i].pitch = ctl[i].pitch;
        c[i].yaw = ctl[i].yaw;
        c[i].roll = ctl[i].roll;
        c[i].jump = ctl[i].jump != 0;
        c[i].boost = ctl[i].boost != 0;
        c[i].handbrake = ctl[i].handbrake != 0;
    }
    r->batch.SetKernelSync(true);
    r->batch.SetAllCarControls(c.data());
    r->batch.Step(ticks);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Positions (x, y, z) and on-ground flags of every car, positions of every ball.
int32_t rscref_cars_ground(void* h, float* car_xyz, uint8_t* on_ground, float* ball_xyz) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r || !car_xyz || !on_ground || !ball_xyz) return -1;
    std::vector<rsc::CarState> cs((size_t)r->n * r->carsPerArena);
    std::vector<rsc::BallState> bs((size_t)r->n);
    r->batch.GetAllCarStates(cs.data());
    r->batch.GetAllBallStates(bs.data());
    for (size_t i = 0; i < cs.size(); i++) {
        std::memcpy(car_xyz + 3 * i, &cs[i].pos, 12);
        on_ground[i] = cs[i].isOnGround ? 1 : 0;
    }
    for (size_t i = 0; i < bs.size(); i++) std::memcpy(ball_xyz + 3 * i, &bs[i].pos, 12);
    return 0;
}

// Positions of every car (x, y, z per car) and ball, to check the comparator ran.
int32_t rscref_positions(void* h, float* car_xyz, float* ball_xyz) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r || !car_xyz || !ball_xyz) return -1;
    std::vector<rsc::CarState> cs((size_t)r->n * r->carsPerArena);
    std::vector<rsc::BallState> bs((size_t)r->n);
    r->batch.GetAllCarStates(cs.data());
    r->batch.GetAllBallStates(bs.data());
    for (size_t i = 0; i < cs.size(); i++) std::memcpy(car_xyz + 3 * i, &cs[i].pos, 12);
    for (size_t i = 0; i < bs.size(); i++) std::memcpy(ball_xyz + 3 * i, &bs[i].pos, 12);
    return 0;
}

}  // extern "C"
