// rsb_envset.hpp — the GPU-native path of GigaLearnCPP's GGL::CudaEnvSet
// (GigaLearnCPP/src/public/GigaLearnCPP/Sim/CudaEnvSet.{h,cpp}) over this library, so that the
// PPO collector's calls (StepDiscrete, StepDiscreteDevice, Reset, ResetAll, the state ring)
// and the host mirrors it reads (obs, actionMasks, rewards_out, terminals) stay as they are.
//
// One env step runs the reference's sequence (CudaEnvSet.cpp:364-421):
//   SnapshotTrainingState -> SetDiscreteActionsFrom{Indices,Device} -> Step(tickSkip)
//   -> BuildAdvancedObsAndDefaultMasks -> BuildRewardsAndTerminals(tickSkip)
//   -> CopyGpuTrainingBuffers (fence, then obs / masks / rewards / terminals to the host)
//   -> ResetTerminalArenasGpu unless skipHostObsCopy (reset every finished arena, clear its
//      host terminal, rebuild and copy obs and masks)
//   -> MaybeCaptureStateRing.
// Arenas are created as the reference creates them (CudaEnvSet.cpp:202-224): carsPerTeam
// blue and orange cars each, then ResetAllArenas; the DefaultAction table is uploaded.
// Differences: the hybrid CPU-bridge mode, continuous actions and the runtime reward
// registry are not provided (the stub rewards and terminals come from rsb_reward_config),
// and resets draw from a seeded counter stream instead of the reference's host LCG.
// Header-only; link with librsb.so.
#pragma once

#include <cstdint>
#include <vector>

#include "rsb_batch.hpp"

namespace rsb {

struct EnvSetConfig {
    int numArenas = 1;
    int carsPerTeam = 1;
    int tickSkip = 8;
    const char* collisionMeshesPath = nullptr;
    unsigned long long seed = 0;
    int device = 0;
    float noTouchSeconds = 0.f;      // NoTouchCondition (0 = off)
    int episodeMaxTicks = 0;         // truncation after this many ticks since a reset (0 = off)
    const rsb_mutators* mutators = nullptr;
};

class CudaEnvSet {
public:
    int numArenas = 0, carsPerArena = 0, tickSkip = 0, numPlayers = 0;
    int obsSize = 0, actionCount = RSB_NUM_ACTIONS;
    bool skipHostObsCopy = false;
    RocketSimCudaBatch batch;
    std::vector<float> obs;              // [numPlayers][obsSize]
    std::vector<uint8_t> actionMasks;    // [numPlayers][actionCount]
    std::vector<float> rewards_out;      // [numPlayers]
    std::vector<uint8_t> terminals;      // [numArenas] (RLGymCPP TerminalType)

    explicit CudaEnvSet(const EnvSetConfig& c) : cfg_(c) {
        numArenas = c.numArenas;
        carsPerArena = 2 * c.carsPerTeam;
        tickSkip = c.tickSkip;
        numPlayers = numArenas * carsPerArena;
        rsb_default_rewards(&rewards_);
        rewards_.no_touch_timeout_s = c.noTouchSeconds;
        rewards_.episode_max_ticks = c.episodeMaxTicks;
        BatchConfig bc;
        bc.numArenas = numArenas;
        bc.maxCarsPerArena = carsPerArena;
        bc.tickSkip = tickSkip;
        bc.collisionMeshesPath = c.collisionMeshesPath;
        bc.seed = c.seed;
        bc.device = c.device;
        bc.mutators = c.mutators;
        bc.rewards = &rewards_;
        batch.Init(bc);
        for (int a = 0; a < numArenas; a++)
            for (int t = 0; t < c.carsPerTeam; t++) batch.AddCar(a, Team::BLUE);
        for (int a = 0; a < numArenas; a++)
            for (int t = 0; t < c.carsPerTeam; t++) batch.AddCar(a, Team::ORANGE);
        batch.ResetAllArenas();
        rsb_controls lut[RSB_NUM_ACTIONS];
        actionCount = rsb_default_action_lut(lut, RSB_NUM_ACTIONS) == RSB_OK ? RSB_NUM_ACTIONS : 0;
        batch.UploadDiscreteActionLut(lut, actionCount);
        obsSize = batch.GetAdvancedObsSize();
        obs.assign((size_t)numPlayers * obsSize, 0.f);
        actionMasks.assign((size_t)numPlayers * RSB_NUM_ACTIONS, 0);
        rewards_out.assign((size_t)numPlayers, 0.f);
        terminals.assign((size_t)numArenas, 0);
    }

    // CudaEnvSet::StepDiscrete, GPU-native branch (CudaEnvSet.cpp:378-421).
    void StepDiscrete(const std::vector<int>& actions) {
        if ((int)actions.size() != numPlayers) return;
        batch.SnapshotTrainingState();
        batch.SetDiscreteActionsFromIndices(actions.data(), numPlayers);
        finishStep();
    }
    // CudaEnvSet::StepDiscreteDevice (CudaEnvSet.cpp:364-376): indices already on the device.
    void StepDiscreteDevice(const int* deviceActionIndices) {
        if (!deviceActionIndices) return;
        batch.SnapshotTrainingState();
        batch.SetDiscreteActionsFromDevice(deviceActionIndices, numPlayers);
        finishStep();
    }
    // CudaEnvSet::Reset / ResetAll: every arena back to a (curriculum) kickoff, fresh outputs.
    void Reset() { ResetAll(); }
    void ResetAll() {
        batch.ResetAllArenas();
        batch.BuildAdvancedObsAndDefaultMasks();
        batch.CopyBuiltAdvancedObs(obs.data());
        batch.CopyBuiltDefaultActionMasks(actionMasks.data());
        std::fill(terminals.begin(), terminals.end(), 0);
    }
    // CudaEnvSet::EnableThroughputSyncMode: device-resident outputs, no host mirrors or resets.
    void EnableThroughputSyncMode(bool enable) { skipHostObsCopy = enable; }

    // State ring (CudaEnvSet.h:100-125): device slots, same configuration fields.
    void ConfigureStateRing(const rsb_ring_config& c) {
        if (rsb_handle* h = batch.Handle()) ringOn_ = rsb_ring_configure(h, &c) == RSB_OK && c.depth > 0;
    }
    void MaybeCaptureStateRing() {
        if (!ringOn_) return;
        if (rsb_handle* h = batch.Handle()) rsb_ring_maybe_capture(h, nullptr);
    }
    int RestoreStateRingReplay(float restoreFraction = -1.f, int lookbackSlots = -1, float fuzzScale = 1.f,
                               int maxArenas = -1) {
        rsb_handle* h = batch.Handle();
        int32_t restored = 0;
        if (!ringOn_ || !h) return 0;
        if (rsb_ring_restore(h, restoreFraction, lookbackSlots, fuzzScale, maxArenas, &restored, nullptr) != RSB_OK)
            return 0;
        if (restored > 0) batch.BuildAdvancedObsAndDefaultMasks();
        return restored;
    }

private:
    void finishStep() {
        batch.Step(tickSkip);
        batch.BuildAdvancedObsAndDefaultMasks();
        batch.BuildRewardsAndTerminals(tickSkip);
        if (!skipHostObsCopy) {
            copyTrainingBuffers();
            resetTerminalArenas();
        }
        MaybeCaptureStateRing();
    }
    // CopyGpuTrainingBuffers (CudaEnvSet.cpp:148-168)
    void copyTrainingBuffers() {
        batch.Synchronize();
        batch.CopyBuiltAdvancedObs(obs.data());
        batch.CopyBuiltDefaultActionMasks(actionMasks.data());
        batch.CopyBuiltRewards(rewards_out.data());
        batch.CopyBuiltTerminals(terminals.data());
    }
    // ResetTerminalArenasGpu (CudaEnvSet.cpp:182-200)
    void resetTerminalArenas() {
        bool any = false;
        for (int a = 0; a < numArenas; a++) {
            if (!terminals[(size_t)a]) continue;
            batch.ResetArena(a);
            terminals[(size_t)a] = 0;
            any = true;
        }
        if (!any) return;
        batch.BuildAdvancedObsAndDefaultMasks();
        batch.CopyBuiltAdvancedObs(obs.data());
        batch.CopyBuiltDefaultActionMasks(actionMasks.data());
        batch.Synchronize();
    }

    EnvSetConfig cfg_;
    rsb_reward_config rewards_{};
    bool ringOn_ = false;
};

}  // namespace rsb
