// rsb_batch.hpp — a C++ facade over the C ABI of rsb.h with the method names and call flow of
// the reference batch simulator, rsc::RocketSimCudaBatch (RocketSimCuda/include/
// RocketSimCuda.h:258-455), so that a collector written against that class (GigaLearnCPP's
// CudaEnvSet, CudaEnvSet.cpp:202-481) changes its include and its namespace, not its calls.
//
// Differences a caller sees:
//   - the arenas are created when their cars are known: Init stores the configuration, AddCar
//     lays out the cars, and the first call that needs the simulation creates them.  Every
//     arena must receive maxCarsPerArena cars, its blue cars before its orange ones, half of
//     each (ragged batches are created directly with rsb_config.team_sizes);
//   - errors are kept instead of printed: Ok() and LastError() report the last failure, and a
//     failed call leaves the batch unchanged;
//   - the state structs are the rsb_* layouts (same fields and units as RocketSim's states).
// Header-only; link with librsb.so.
#pragma once

#include <string>
#include <vector>

#include "rsb.h"

namespace rsb {

enum class Team { BLUE = 0, ORANGE = 1 };

using CarControls = rsb_controls;
using CarState = rsb_car_state;
using BallState = rsb_ball_state;
using BoostPadState = rsb_pad_state;
using ArenaInfo = rsb_arena_info;

// RocketSimCuda.h BatchConfig, with the fields this library uses.
struct BatchConfig {
    int numArenas = 1;
    int maxCarsPerArena = 2;
    float tickRate = 120.f;
    const char* collisionMeshesPath = nullptr;
    int tickSkip = 8;
    unsigned long long seed = 0;
    int device = 0;
    const rsb_mutators* mutators = nullptr;      // nullptr: RocketSim's soccar defaults
    const rsb_reward_config* rewards = nullptr;  // nullptr: no rewards or terminals (rsb_default_rewards gives the stub set)
};

class RocketSimCudaBatch {
public:
    RocketSimCudaBatch() = default;
    RocketSimCudaBatch(const RocketSimCudaBatch&) = delete;
    RocketSimCudaBatch& operator=(const RocketSimCudaBatch&) = delete;
    ~RocketSimCudaBatch() { Destroy(); }

    // RocketSimCudaBatch::Init (:264): stores the configuration.
    void Init(const BatchConfig& config) {
        Destroy();
        cfg_ = config;
        if (cfg_.numArenas <= 0 || cfg_.maxCarsPerArena < 0 || cfg_.maxCarsPerArena > RSB_MAX_CARS_PER_ARENA ||
            cfg_.maxCarsPerArena % 2 != 0) {
            setError(RSB_ERR_INVALID, "Init: numArenas > 0 and an even maxCarsPerArena <= 6 are required");
            return;
        }
        blue_.assign((size_t)cfg_.numArenas, 0);
        orange_.assign((size_t)cfg_.numArenas, 0);
        initialized_ = true;
    }

    // RocketSimCudaBatch::Destroy (:267).
    void Destroy() {
        if (h_) rsb_destroy(h_);
        h_ = nullptr;
        initialized_ = false;
    }

    // RocketSimCudaBatch::AddCar (:272): the car's slot in its arena, or -1 (arena full, arena
    // already created, or a blue car after an orange one).
    int AddCar(int arenaIdx, Team team) {
        if (!initialized_ || h_ || arenaIdx < 0 || arenaIdx >= cfg_.numArenas) return -1;
        const int half = cfg_.maxCarsPerArena / 2;
        int& b = blue_[(size_t)arenaIdx];
        int& o = orange_[(size_t)arenaIdx];
        if (team == Team::BLUE) {
            if (b >= half || o > 0) return -1;
            return b++;
        }
        if (o >= half) return -1;
        return half + o++;
    }

    // RocketSimCudaBatch::ResetArena / ResetAllArenas (:275-278): kickoff, or the curriculum
    // mix once SetResetCurriculum has been called.
    void ResetArena(int arenaIdx) {
        if (!ensure()) return;
        const int32_t idx = arenaIdx;
        check(rsb_reset_arenas(h_, &idx, 1, nextSeed(), resetMode_));
    }
    void ResetAllArenas() {
        if (ensure()) check(rsb_reset_all(h_, nextSeed(), resetMode_));
    }
    // RocketSimCudaBatch::SetResetCurriculum (:283).
    void SetResetCurriculum(float kickoffW, float fuzzedW, float aerialW, float chaseW = 0.f) {
        if (!ensure()) return;
        if (check(rsb_set_reset_curriculum(h_, kickoffW, fuzzedW, aerialW, chaseW))) resetMode_ = RSB_RESET_CURRICULUM;
    }

    void SetCarControls(int arenaIdx, int carIdx, const CarControls& c) {
        if (ensure()) check(rsb_set_car_controls_at(h_, arenaIdx, carIdx, &c));
    }
    void SetAllCarControls(const CarControls* c) {
        if (ensure()) check(rsb_set_controls(h_, c, GetNumPlayers()));
    }
    void UploadDiscreteActionLut(const CarControls* lut, int actionCount) {
        if (ensure()) check(rsb_set_action_lut(h_, lut, actionCount));
    }
    void SetDiscreteActionsFromIndices(const int* indices, int count) {
        if (ensure()) check(rsb_set_actions_host(h_, indices, count));
    }
    void SetDiscreteActionsFromDevice(const int* deviceIndices, int count) {
        if (ensure()) check(rsb_set_actions_device(h_, deviceIndices, count, nullptr));
    }

    void Step(int ticksToSimulate = 1) {
        if (ensure()) check(rsb_step(h_, ticksToSimulate, nullptr));
    }

    void BuildAdvancedObsAndDefaultMasks() {
        if (ensure()) check(rsb_build_obs(h_, nullptr));
    }
    void SnapshotTrainingState() {
        if (ensure()) check(rsb_snapshot(h_, nullptr));
    }
    void BuildRewardsAndTerminals(int stepTicks) {
        if (ensure()) check(rsb_build_rewards_terminals(h_, stepTicks, nullptr));
    }
    void CopyBuiltAdvancedObs(float* out) {
        if (ensure()) check(rsb_copy_obs(h_, out, (size_t)GetNumPlayers() * GetAdvancedObsSize()));
    }
    void CopyBuiltDefaultActionMasks(uint8_t* out) {
        if (ensure()) check(rsb_copy_masks(h_, out, (size_t)GetNumPlayers() * RSB_NUM_ACTIONS));
    }
    void CopyBuiltRewards(float* out) {
        if (ensure()) check(rsb_copy_rewards(h_, out, (size_t)GetNumPlayers()));
    }
    void CopyBuiltTerminals(uint8_t* out) {
        if (ensure()) check(rsb_copy_terminals(h_, out, (size_t)cfg_.numArenas));
    }
    void Synchronize() {
        if (ensure()) check(rsb_sync(h_));
    }

    CarState GetCarState(int arenaIdx, int carIdx) {
        CarState s{};
        if (ensure()) check(rsb_get_car_at(h_, arenaIdx, carIdx, &s));
        return s;
    }
    void GetAllCarStates(CarState* out) {
        if (ensure()) check(rsb_get_cars(h_, out, GetNumPlayers()));
    }
    BallState GetBallState(int arenaIdx) {
        BallState s{};
        if (ensure()) check(rsb_get_ball_at(h_, arenaIdx, &s));
        return s;
    }
    void GetAllBallStates(BallState* out) {
        if (ensure()) check(rsb_get_balls(h_, out, cfg_.numArenas));
    }
    void GetBoostPadStates(int arenaIdx, BoostPadState* out) {
        if (ensure()) check(rsb_get_pads_at(h_, arenaIdx, out));
    }
    void GetAllBoostPadStates(BoostPadState* out) {
        if (ensure()) check(rsb_get_pads(h_, out, cfg_.numArenas * RSB_NUM_PADS));
    }
    ArenaInfo GetArenaInfo(int arenaIdx) {
        ArenaInfo s{};
        if (ensure()) check(rsb_get_arena_info_at(h_, arenaIdx, &s));
        return s;
    }
    void GetAllArenaInfos(ArenaInfo* out) {
        if (ensure()) check(rsb_get_arena_info(h_, out, cfg_.numArenas));
    }
    void SetCarState(int arenaIdx, int carIdx, const CarState& s) {
        if (ensure()) check(rsb_set_car_at(h_, arenaIdx, carIdx, &s));
    }
    void SetBallState(int arenaIdx, const BallState& s) {
        if (ensure()) check(rsb_set_ball_at(h_, arenaIdx, &s));
    }
    void SetBoostPadStates(int arenaIdx, const BoostPadState* s) {
        if (ensure()) check(rsb_set_pads_at(h_, arenaIdx, s));
    }
    void SetAllBoostPadStates(const BoostPadState* s) {
        if (ensure()) check(rsb_set_pads(h_, s, cfg_.numArenas * RSB_NUM_PADS));
    }

    void* GetBuiltAdvancedObsDevicePtr() { return devicePtr(RSB_BUF_OBS); }
    void* GetBuiltDefaultActionMasksDevicePtr() { return devicePtr(RSB_BUF_MASKS); }
    void* GetBuiltRewardsDevicePtr() { return devicePtr(RSB_BUF_REWARDS); }
    void* GetBuiltTerminalsDevicePtr() { return devicePtr(RSB_BUF_TERMINALS); }
    void* GetControlsDevicePtr() { return devicePtr(RSB_BUF_CONTROLS); }

    int GetNumArenas() const { return cfg_.numArenas; }
    int GetMaxCarsPerArena() const { return cfg_.maxCarsPerArena; }
    int GetNumPlayers() const { return cfg_.numArenas * cfg_.maxCarsPerArena; }
    int GetAdvancedObsSize() const { return RSB_OBS_BASE + RSB_OBS_PER_CAR * cfg_.maxCarsPerArena; }
    float GetTickTime() const { return 1.f / cfg_.tickRate; }
    const BatchConfig& GetConfig() const { return cfg_; }

    bool Ok() const { return status_ == RSB_OK; }
    rsb_status Status() const { return status_; }
    const std::string& LastError() const { return error_; }
    rsb_handle* Handle() { return ensure() ? h_ : nullptr; }

private:
    // creates the arenas once every arena has its cars
    bool ensure() {
        if (h_) return true;
        if (!initialized_) return setError(RSB_ERR_STATE, "Init was not called");
        const int half = cfg_.maxCarsPerArena / 2;
        for (int a = 0; a < cfg_.numArenas; a++)
            if (blue_[(size_t)a] != half || orange_[(size_t)a] != half)
                return setError(RSB_ERR_STATE, "every arena needs maxCarsPerArena cars, half blue and half orange");
        rsb_config c{};
        c.num_arenas = cfg_.numArenas;
        c.team_size = half;
        c.tick_rate = cfg_.tickRate;
        c.tick_skip = cfg_.tickSkip;
        c.meshes_path = cfg_.collisionMeshesPath;
        c.mutators = cfg_.mutators;
        c.rewards = cfg_.rewards;
        c.seed = cfg_.seed;
        c.device = cfg_.device;
        const rsb_status st = rsb_create(&c, &h_);
        if (st != RSB_OK) {
            char msg[512];
            rsb_last_error(nullptr, msg, sizeof msg);
            h_ = nullptr;
            return setError(st, msg);
        }
        return true;
    }
    bool check(rsb_status st) {
        if (st == RSB_OK) return true;
        char msg[512];
        rsb_last_error(h_, msg, sizeof msg);
        return setError(st, msg);
    }
    bool setError(rsb_status st, const std::string& msg) {
        status_ = st;
        error_ = msg;
        return false;
    }
    void* devicePtr(int32_t which) {
        void* p = nullptr;
        if (ensure()) check(rsb_device_ptr(h_, which, &p));
        return p;
    }
    uint64_t nextSeed() { return cfg_.seed + 0x9E3779B97F4A7C15ull * ++resets_; }

    BatchConfig cfg_{};
    rsb_handle* h_ = nullptr;
    bool initialized_ = false;
    std::vector<int> blue_, orange_;
    uint64_t resets_ = 0;
    int32_t resetMode_ = RSB_RESET_KICKOFF;
    rsb_status status_ = RSB_OK;
    std::string error_;
};

}  // namespace rsb
