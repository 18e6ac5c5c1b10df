// The C++ facade (include/rsb_batch.hpp) driven the way GigaLearnCPP's CudaEnvSet drives the
// reference batch (CudaEnvSet.cpp:210-225 set-up, :364-421 env step), against the same steps
// through the C ABI directly: identical states, observations, masks, rewards and terminals.
//   batch_facade_test <meshes dir>            (GPU: the equivalence run)
//   batch_facade_test <meshes dir> --no-gpu   (no device: the facade reports the error)
#include <cstdio>
#include <cstring>
#include <vector>

#include "rsb_batch.hpp"

#define CHECK(c)                                                  \
    do {                                                          \
        if (!(c)) {                                               \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
            return 1;                                             \
        }                                                         \
    } while (0)

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const bool noGpu = argc > 2 && std::strcmp(argv[2], "--no-gpu") == 0;
    const int N = 24, M = 4;
    rsb_reward_config rewards{};
    CHECK(rsb_default_rewards(&rewards) == RSB_OK);

    rsb::BatchConfig cfg;
    cfg.numArenas = N;
    cfg.maxCarsPerArena = M;
    cfg.collisionMeshesPath = argv[1];
    cfg.seed = 77;
    cfg.rewards = &rewards;
    rsb::RocketSimCudaBatch batch;
    batch.Init(cfg);
    CHECK(batch.Ok());
    for (int a = 0; a < N; a++) {
        for (int t = 0; t < M / 2; t++) CHECK(batch.AddCar(a, rsb::Team::BLUE) == t);
        for (int t = 0; t < M / 2; t++) CHECK(batch.AddCar(a, rsb::Team::ORANGE) == M / 2 + t);
    }
    CHECK(batch.AddCar(0, rsb::Team::ORANGE) == -1);  // full
    batch.ResetAllArenas();
    if (noGpu) {
        CHECK(!batch.Ok() && batch.Status() == RSB_ERR_CUDA);
        std::printf("facade reports: %s\n", batch.LastError().c_str());
        return 0;
    }
    CHECK(batch.Ok());
    CHECK(batch.AddCar(1, rsb::Team::BLUE) == -1);  // arenas already created

    // the same batch through the C ABI
    rsb_config c{};
    c.num_arenas = N;
    c.team_size = M / 2;
    c.tick_rate = 120.f;
    c.tick_skip = 8;
    c.meshes_path = argv[1];
    c.seed = 77;
    c.rewards = &rewards;
    rsb_handle* h = nullptr;
    CHECK(rsb_create(&c, &h) == RSB_OK);
    // the facade's first reset seed (seed + golden-ratio step), so both start identical
    CHECK(rsb_reset_all(h, 77ull + 0x9E3779B97F4A7C15ull, RSB_RESET_KICKOFF) == RSB_OK);
    std::vector<rsb_car_state> cars(N * M);
    std::vector<rsb_controls> lut(RSB_NUM_ACTIONS);
    CHECK(rsb_default_action_lut(lut.data(), RSB_NUM_ACTIONS) == RSB_OK);
    batch.UploadDiscreteActionLut(lut.data(), RSB_NUM_ACTIONS);
    CHECK(rsb_set_action_lut(h, lut.data(), RSB_NUM_ACTIONS) == RSB_OK);

    const int P = N * M, R = batch.GetAdvancedObsSize();
    CHECK(R == RSB_OBS_BASE + RSB_OBS_PER_CAR * M);
    std::vector<int> idx(P);
    std::vector<float> obsA(P * R), obsB(P * R), rewA(P), rewB(P);
    std::vector<uint8_t> maskA(P * RSB_NUM_ACTIONS), maskB(P * RSB_NUM_ACTIONS), termA(N), termB(N);
    std::vector<rsb_car_state> carsB(P);
    unsigned s = 12345;
    for (int step = 0; step < 12; step++) {
        for (int i = 0; i < P; i++) idx[i] = (int)((s = s * 1103515245u + 12345u) >> 16) % RSB_NUM_ACTIONS;
        // CudaEnvSet::StepDiscrete on the facade
        batch.SnapshotTrainingState();
        batch.SetDiscreteActionsFromIndices(idx.data(), P);
        if (step == 5) {  // one car overridden after the action expansion
            rsb_controls over{};
            over.throttle = -1.f;
            over.handbrake = 1;
            batch.SetCarControls(3, 1, over);
        }
        batch.Step(8);
        batch.BuildAdvancedObsAndDefaultMasks();
        batch.BuildRewardsAndTerminals(8);
        batch.CopyBuiltAdvancedObs(obsA.data());
        batch.CopyBuiltDefaultActionMasks(maskA.data());
        batch.CopyBuiltRewards(rewA.data());
        batch.CopyBuiltTerminals(termA.data());
        // the same through the C ABI
        CHECK(rsb_snapshot(h, nullptr) == RSB_OK);
        CHECK(rsb_set_actions_host(h, idx.data(), P) == RSB_OK);
        if (step == 5) {
            std::vector<rsb_controls> all(P);
            for (int i = 0; i < P; i++) all[i] = lut[idx[i]];
            all[3 * M + 1] = rsb_controls{};
            all[3 * M + 1].throttle = -1.f;
            all[3 * M + 1].handbrake = 1;
            CHECK(rsb_set_controls(h, all.data(), P) == RSB_OK);
        }
        CHECK(rsb_step(h, 8, nullptr) == RSB_OK);
        CHECK(rsb_build_obs(h, nullptr) == RSB_OK);
        CHECK(rsb_build_rewards_terminals(h, 8, nullptr) == RSB_OK);
        CHECK(rsb_copy_outputs(h, obsB.data(), maskB.data(), rewB.data(), termB.data()) == RSB_OK);
        CHECK(batch.Ok());
        CHECK(std::memcmp(obsA.data(), obsB.data(), obsA.size() * 4) == 0);
        CHECK(std::memcmp(maskA.data(), maskB.data(), maskA.size()) == 0);
        CHECK(std::memcmp(rewA.data(), rewB.data(), rewA.size() * 4) == 0);
        CHECK(std::memcmp(termA.data(), termB.data(), termA.size()) == 0);
        batch.GetAllCarStates(cars.data());
        CHECK(rsb_get_cars(h, carsB.data(), P) == RSB_OK);
        CHECK(std::memcmp(cars.data(), carsB.data(), cars.size() * sizeof(rsb_car_state)) == 0);
    }
    // one-arena access matches the batch access
    rsb::CarState one = batch.GetCarState(7, 2);
    CHECK(std::memcmp(&one, &cars[7 * M + 2], sizeof one) == 0);
    rsb::ArenaInfo info = batch.GetArenaInfo(7);
    CHECK(info.num_cars == M && info.team_size == M / 2);
    CHECK(batch.GetBuiltAdvancedObsDevicePtr() != nullptr);
    rsb_destroy(h);
    std::printf("facade ok\n");
    return 0;
}
