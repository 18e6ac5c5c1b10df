// Drives the CudaEnvSet-compatible adapter (include/rsb_envset.hpp) and, beside it, the same
// collector step written out as raw C-ABI calls in the reference's order
// (CudaEnvSet.cpp:364-421: snapshot, actions, step, obs, rewards/terminals, copies, resets of
// finished arenas with an obs rebuild), and checks after every env step that the host mirrors
// (observations, masks, rewards, terminals) are byte-identical.  Half the steps go through
// StepDiscrete (host indices), half through StepDiscreteDevice (indices in device memory).
//
//   envset_adapter_test <meshes dir> [--no-gpu]
// With --no-gpu the adapter must report the missing device instead of crashing.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "rsb_envset.hpp"

namespace {

constexpr int kArenas = 192, kPerTeam = 2, kTickSkip = 8, kSteps = 80;
constexpr unsigned long long kSeed = 0x5EED0001ull;

int fail(const char* what, int step) {
    std::printf("MISMATCH %s at step %d\n", what, step);
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::printf("usage: %s <meshes dir> [--no-gpu]\n", argv[0]);
        return 2;
    }
    const bool noGpu = argc > 2 && std::strcmp(argv[2], "--no-gpu") == 0;
    rsb::EnvSetConfig ec;
    ec.numArenas = kArenas;
    ec.carsPerTeam = kPerTeam;
    ec.tickSkip = kTickSkip;
    ec.collisionMeshesPath = argv[1];
    ec.seed = kSeed;
    ec.episodeMaxTicks = 200;  // truncations every 25 env steps exercise the terminal resets
    rsb::CudaEnvSet env(ec);
    if (noGpu) {
        if (env.batch.Ok() || env.batch.Status() != RSB_ERR_CUDA) {
            std::printf("expected a missing-device error, got status %d\n", env.batch.Status());
            return 1;
        }
        std::printf("adapter reports: %s\n", env.batch.LastError().c_str());
        return 0;
    }
    if (!env.batch.Ok()) {
        std::printf("adapter failed: %s\n", env.batch.LastError().c_str());
        return 1;
    }

    // the raw sequence on its own handle, with the facade's reset seeds
    rsb_reward_config rew;
    rsb_default_rewards(&rew);
    rew.episode_max_ticks = ec.episodeMaxTicks;
    rsb_config rc{};
    rc.num_arenas = kArenas;
    rc.team_size = kPerTeam;
    rc.tick_rate = 120.f;
    rc.tick_skip = kTickSkip;
    rc.meshes_path = argv[1];
    rc.rewards = &rew;
    rc.seed = kSeed;
    rsb_handle* h = nullptr;
    if (rsb_create(&rc, &h) != RSB_OK) return fail("rsb_create", -1);
    unsigned long long resets = 0;
    auto nextSeed = [&] { return kSeed + 0x9E3779B97F4A7C15ull * ++resets; };
    if (rsb_reset_all(h, nextSeed(), RSB_RESET_KICKOFF) != RSB_OK) return fail("reset_all", -1);
    rsb_controls lut[RSB_NUM_ACTIONS];
    rsb_default_action_lut(lut, RSB_NUM_ACTIONS);
    rsb_set_action_lut(h, lut, RSB_NUM_ACTIONS);

    const int P = env.numPlayers, S = env.obsSize;
    std::vector<float> obs((size_t)P * S), rewards((size_t)P);
    std::vector<uint8_t> masks((size_t)P * RSB_NUM_ACTIONS), terms((size_t)kArenas);
    std::vector<int> actions((size_t)P);
    int* dActions = nullptr;
    if (cudaMalloc(&dActions, sizeof(int) * P) != cudaSuccess) return fail("cudaMalloc", -1);
    uint32_t lcg = 12345u;
    int finished = 0;
    for (int step = 0; step < kSteps; step++) {
        for (int p = 0; p < P; p++) {
            lcg = lcg * 1664525u + 1013904223u;
            actions[(size_t)p] = (int)((lcg >> 8) % RSB_NUM_ACTIONS);
        }
        const bool device = step % 2 == 1;
        if (device) {
            cudaMemcpy(dActions, actions.data(), sizeof(int) * P, cudaMemcpyHostToDevice);
            env.StepDiscreteDevice(dActions);
        } else {
            env.StepDiscrete(actions);
        }
        if (!env.batch.Ok()) {
            std::printf("adapter step failed: %s\n", env.batch.LastError().c_str());
            return 1;
        }
        rsb_snapshot(h, nullptr);
        if (device) rsb_set_actions_device(h, dActions, P, nullptr);
        else rsb_set_actions_host(h, actions.data(), P);
        rsb_step(h, kTickSkip, nullptr);
        rsb_build_obs(h, nullptr);
        rsb_build_rewards_terminals(h, kTickSkip, nullptr);
        rsb_sync(h);
        rsb_copy_obs(h, obs.data(), obs.size());
        rsb_copy_masks(h, masks.data(), masks.size());
        rsb_copy_rewards(h, rewards.data(), rewards.size());
        rsb_copy_terminals(h, terms.data(), terms.size());
        bool any = false;
        for (int a = 0; a < kArenas; a++) {
            if (!terms[(size_t)a]) continue;
            const int32_t idx = a;
            rsb_reset_arenas(h, &idx, 1, nextSeed(), RSB_RESET_KICKOFF);
            terms[(size_t)a] = 0;
            any = true;
            finished++;
        }
        if (any) {
            rsb_build_obs(h, nullptr);
            rsb_copy_obs(h, obs.data(), obs.size());
            rsb_copy_masks(h, masks.data(), masks.size());
        }
        if (std::memcmp(obs.data(), env.obs.data(), obs.size() * 4)) return fail("observations", step);
        if (std::memcmp(masks.data(), env.actionMasks.data(), masks.size())) return fail("masks", step);
        if (std::memcmp(rewards.data(), env.rewards_out.data(), rewards.size() * 4)) return fail("rewards", step);
        if (std::memcmp(terms.data(), env.terminals.data(), terms.size())) return fail("terminals", step);
    }
    cudaFree(dActions);
    rsb_destroy(h);
    if (finished == 0) {
        std::printf("no arena finished: the terminal resets were not exercised\n");
        return 1;
    }
    std::printf("envset adapter ok: %d env steps, %d finished arenas reset\n", kSteps, finished);
    return 0;
}
