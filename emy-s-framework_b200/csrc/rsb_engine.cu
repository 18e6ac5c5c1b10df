// CUDA engine behind the C ABI of include/rsb.h.
//
// One kernel thread advances one arena through all requested ticks with the arena's
// state held in registers / thread-local memory; state is read from and written back to
// the word-plane layout of phys/state.h at the launch boundaries.  Static arena data
// (meshes, BVHs, grids) is built once on the host and shared by every handle on a device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "rsb.h"
#include "arena_build.h"
#include "engine_host.h"
#include "env_kernels.cuh"

using namespace rsb;

namespace {

std::string g_createError;

#define RSB_CUDA(call)                                                             \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return cudaFail(h, #call, e_);                      \
    } while (0)

struct DevStatic {
    BvhNode* nodes = nullptr;
    BvhSubtree* subs = nullptr;
    V3* triVerts = nullptr;
    TriEdgeInfo* triInfo = nullptr;
    uint32_t* bpCells = nullptr;
    ArenaStatic view{};
};

// Host build + device copy of the arena data, shared per (device, meshes folder).
struct StaticCache {
    std::mutex mu;
    std::map<std::string, std::shared_ptr<ArenaStaticHost>> host;
    std::map<std::pair<int, std::string>, std::shared_ptr<DevStatic>> dev;
};
StaticCache& cache() {
    static StaticCache c;
    return c;
}

static_assert(sizeof(CtlRec) == sizeof(rsb_controls), "controls record layout");

// Staging array of rsb_set_actions_host_static: part of the module image, so using it
// allocates nothing.  Every call overwrites the first n entries before the expansion
// kernel reads them; nothing needs to start at zero.
__device__ __align__(256) int32_t g_staticActions[RSB_STATIC_ACTIONS_MAX];

// Device address of g_staticActions, looked up once per device (cudaGetSymbolAddress
// with that device current).
struct StaticActionsAddr {
    std::mutex mu;
    std::map<int, int32_t*> ptr;
};
StaticActionsAddr& staticActionsAddr() {
    static StaticActionsAddr s;
    return s;
}

}  // namespace

struct rsb_handle {
    int device = 0;
    int N = 0;
    int numCars = 0;
    int maxCars = 0;
    uint64_t seed = 0;
    std::vector<int32_t> teamSize, carOffset;
    std::shared_ptr<DevStatic> stat;
    WorldParams P{};
    rsb_mutators mut{};
    cudaStream_t stream = nullptr;
    int32_t* dTeamSize = nullptr;
    int32_t* dCarOffset = nullptr;
    uint32_t* dBall = nullptr;
    uint32_t* dCar = nullptr;
    uint32_t* dPad = nullptr;
    uint32_t* dArena = nullptr;
    rsb_controls* dControls = nullptr;
    rsb_controls* dLut = nullptr;
    int lutCount = 0;
    int32_t* dActions = nullptr;
    // env layer
    int obsStride = 0;
    float* dObs = nullptr;
    uint8_t* dMasks = nullptr;
    float* dRewards = nullptr;
    uint8_t* dTerminals = nullptr;
    int32_t* dResetIdx = nullptr;
    // launch configuration of the step kernel (indices into kStepVariants / kStepBlocks)
    int stepVariant = 0, stepBlock = 2;
    uint32_t* dScratch = nullptr;   // the autotuner's copy of the arena records
    EnvTables tables{};
    bool hasRewards = false;
    RewardParams rewardParams{};
    std::string err;
    rsb_stats stats{};
};

static rsb_status fail(rsb_handle* h, rsb_status code, const std::string& msg) {
    if (h) h->err = msg;
    else g_createError = msg;
    return code;
}
static rsb_status cudaFail(rsb_handle* h, const char* what, cudaError_t e) {
    return fail(h, RSB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ kernels

// One thread advances one arena.  MINB is the minimum number of 128-thread blocks per SM
// the compiler must fit, which caps the registers per thread; the autotuner picks the
// variant and the block size.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) stepKernel(EngineView D, int ticks) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= D.N) return;
    ArenaSim A;
    EpaWork epa;
    A.W.epa = &epa;
    stepArena(D, a, ticks, A);
}

struct StepVariant {
    void (*fn)(EngineView, int);
    int minBlocks;
};
static const StepVariant kStepVariants[] = {{stepKernel<1>, 1}, {stepKernel<3>, 3}, {stepKernel<4>, 4}};
constexpr int kNumStepVariants = sizeof(kStepVariants) / sizeof(kStepVariants[0]);
static const int kStepBlocks[] = {32, 64, 128};
constexpr int kNumStepBlocks = sizeof(kStepBlocks) / sizeof(kStepBlocks[0]);

__global__ void expandActionsKernel(const int32_t* idx, const rsb_controls* lut, int lutCount, rsb_controls* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = idx[i];
    k = k < 0 ? 0 : (k >= lutCount ? lutCount - 1 : k);
    out[i] = lut[k];
}

// ------------------------------------------------------------------ host helpers

static rsb_status download(rsb_handle* h, const uint32_t* d, std::vector<uint32_t>& host, size_t words) {
    host.resize(words);
    RSB_CUDA(cudaMemcpyAsync(host.data(), d, words * 4, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}
static rsb_status upload(rsb_handle* h, uint32_t* d, const std::vector<uint32_t>& host) {
    RSB_CUDA(cudaMemcpyAsync(d, host.data(), host.size() * 4, cudaMemcpyHostToDevice, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

static EngineView devView(rsb_handle* h) {
    EngineView D;
    D.S = h->stat->view;
    D.P = h->P;
    D.N = h->N;
    D.teamSize = h->dTeamSize;
    D.carOffset = h->dCarOffset;
    D.ball = h->dBall;
    D.car = h->dCar;
    D.pad = h->dPad;
    D.arena = h->dArena;
    D.controls = reinterpret_cast<const CtlRec*>(h->dControls);
    D.seed = (uint32_t)(h->seed ^ (h->seed >> 32));
    return D;
}

static EnvView envView(rsb_handle* h) {
    EnvView E;
    E.ball = h->dBall;
    E.car = h->dCar;
    E.pad = h->dPad;
    E.arena = h->dArena;
    E.N = h->N;
    E.teamSize = h->dTeamSize;
    E.carOffset = h->dCarOffset;
    E.controls = reinterpret_cast<CtlRec*>(h->dControls);
    E.obs = h->dObs;
    E.stride = h->obsStride;
    E.masks = h->dMasks;
    E.rewards = h->dRewards;
    E.terminals = h->dTerminals;
    return E;
}

static cudaStream_t pick(rsb_handle* h, void* s) { return s ? (cudaStream_t)s : h->stream; }

// ------------------------------------------------------------------ C ABI

extern "C" {

rsb_status rsb_default_mutators(rsb_mutators* m) {
    if (!m) return RSB_ERR_INVALID;
    defaultMutators(m);
    return RSB_OK;
}

rsb_status rsb_default_rewards(rsb_reward_config* r) {
    if (!r) return RSB_ERR_INVALID;
    *r = rsb_reward_config{};
    r->w_goal = r->w_touch = r->w_vel_ball_to_goal = r->w_vel_player_to_ball = 1.f;
    r->goal_concede_scale = -1.f;
    r->team_spirit = 0.f;
    r->opponent_scale = 1.f;
    r->zero_sum = 0;
    r->episode_max_ticks = 1800;
    r->no_touch_timeout_s = 0.f;
    return RSB_OK;
}

rsb_status rsb_create(const rsb_config* cfg, rsb_handle** out) {
    rsb_handle* h = nullptr;
    if (!cfg || !out) return fail(nullptr, RSB_ERR_INVALID, "null config or output");
    *out = nullptr;
    if (cfg->num_arenas <= 0) return fail(nullptr, RSB_ERR_INVALID, "num_arenas must be > 0");
    if (!cfg->meshes_path) return fail(nullptr, RSB_ERR_MESH, "meshes_path is required");
    if (cfg->tick_rate != 120.f) return fail(nullptr, RSB_ERR_UNSUPPORTED, "tick_rate must be 120");
    int nDev = 0;
    if (cudaGetDeviceCount(&nDev) != cudaSuccess || nDev == 0)
        return fail(nullptr, RSB_ERR_CUDA, "no CUDA device: this library runs on the GPU only");
    if (cfg->device < 0 || cfg->device >= nDev) return fail(nullptr, RSB_ERR_INVALID, "bad device ordinal");

    std::unique_ptr<rsb_handle> hp(new rsb_handle());
    h = hp.get();
    h->device = cfg->device;
    h->N = cfg->num_arenas;
    h->seed = cfg->seed;
    h->carOffset.push_back(0);
    for (int a = 0; a < h->N; a++) {
        int ts = cfg->team_sizes ? cfg->team_sizes[a] : cfg->team_size;
        if (ts < 0 || ts > RSB_MAX_TEAM_SIZE) return fail(nullptr, RSB_ERR_INVALID, "team size must be 0..3");
        h->teamSize.push_back(ts);
        h->carOffset.push_back(h->carOffset.back() + 2 * ts);
        h->maxCars = std::max(h->maxCars, 2 * ts);
    }
    h->numCars = h->carOffset.back();
    {
        // every launch reads and writes each arena's records once and reads its controls
        uint64_t words = 0;
        for (int a = 0; a < h->N; a++) words += W_BALL + W_ARENA + NUM_PADS * W_PAD + 2 * h->teamSize[a] * W_CAR;
        h->stats.state_bytes_per_step = 2 * 4 * words + (uint64_t)h->numCars * sizeof(rsb_controls) + 8 * (uint64_t)h->N;
    }
    if (cfg->mutators) h->mut = *cfg->mutators;
    else defaultMutators(&h->mut);
    computeParams(h->mut, h->P);
    h->obsStride = RSB_OBS_BASE + RSB_OBS_PER_CAR * h->maxCars;
    if (!buildEnvTables(h->tables)) return fail(nullptr, RSB_ERR_STATE, "boost pad tables do not match");
    if (cfg->rewards) {
        const rsb_reward_config& r = *cfg->rewards;
        h->hasRewards = true;
        RewardParams& R = h->rewardParams;
        R.w[0] = r.w_goal; R.w[1] = r.w_touch; R.w[2] = r.w_vel_ball_to_goal; R.w[3] = r.w_vel_player_to_ball;
        R.concede = r.goal_concede_scale;
        R.teamSpirit = r.team_spirit;
        R.oppScale = r.opponent_scale;
        R.zeroSum = r.zero_sum;
        R.episodeMaxTicks = r.episode_max_ticks;
        R.noTouchTimeout = r.no_touch_timeout_s;
        R.goalBaseY = h->mut.goal_base_threshold_y;
        R.ballRadius = h->mut.ball_radius;
    }

    // static arena data (host build shared across handles, device copy per device)
    std::string folder(cfg->meshes_path);
    {
        StaticCache& c = cache();
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.host.find(folder);
        std::shared_ptr<ArenaStaticHost> H;
        if (it == c.host.end()) {
            H = std::make_shared<ArenaStaticHost>();
            if (!buildArenaStatic(folder, *H)) return fail(nullptr, RSB_ERR_MESH, H->error);
            c.host[folder] = H;
        } else {
            H = it->second;
        }
        auto key = std::make_pair(h->device, folder);
        auto dit = c.dev.find(key);
        if (dit != c.dev.end()) {
            h->stat = dit->second;
        } else {
            if (cudaSetDevice(h->device) != cudaSuccess) return fail(nullptr, RSB_ERR_CUDA, "cudaSetDevice failed");
            auto D = std::make_shared<DevStatic>();
            auto up = [&](auto*& dst, const auto& v) -> bool {
                size_t bytes = v.size() * sizeof(v[0]);
                if (cudaMalloc((void**)&dst, bytes ? bytes : 4) != cudaSuccess) return false;
                return cudaMemcpy(dst, v.data(), bytes, cudaMemcpyHostToDevice) == cudaSuccess;
            };
            if (!up(D->nodes, H->nodes) || !up(D->subs, H->subs) || !up(D->triVerts, H->triVerts) ||
                !up(D->triInfo, H->triInfo) || !up(D->bpCells, H->bpCells))
                return fail(nullptr, RSB_ERR_CUDA, "uploading arena meshes failed");
            D->view = deviceView(*H, D->nodes, D->subs, D->triVerts, D->triInfo, D->bpCells);
            c.dev[key] = D;
            h->stat = D;
        }
    }

    if (cudaSetDevice(h->device) != cudaSuccess) return fail(nullptr, RSB_ERR_CUDA, "cudaSetDevice failed");
    {
        // the arena kernel keeps one arena's working set in thread-local memory; make the
        // per-thread stack limit cover the largest variant's frame (the default limit is
        // 1 KB), and give the L1 its largest share (the kernels use no shared memory)
        size_t need = 0;
        for (const StepVariant& v : kStepVariants) {
            cudaFuncAttributes fa{};
            if (cudaFuncGetAttributes(&fa, v.fn) != cudaSuccess)
                return fail(nullptr, RSB_ERR_CUDA, "cudaFuncGetAttributes failed");
            need = std::max(need, ((fa.localSizeBytes + 4096) + 1023) / 1024 * 1024);
            cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        }
        size_t cur = 0;
        cudaDeviceGetLimit(&cur, cudaLimitStackSize);
        if (cur < need && cudaDeviceSetLimit(cudaLimitStackSize, need) != cudaSuccess)
            return fail(nullptr, RSB_ERR_CUDA, "cannot raise the per-thread stack limit for the arena kernel");
    }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(nullptr, RSB_ERR_CUDA, "stream creation failed");
    const size_t N = h->N;
    auto dalloc = [&](auto*& p, size_t bytes) -> bool {
        return cudaMalloc((void**)&p, bytes ? bytes : 4) == cudaSuccess && cudaMemset(p, 0, bytes ? bytes : 4) == cudaSuccess;
    };
    if (!dalloc(h->dTeamSize, N * 4) || !dalloc(h->dCarOffset, (N + 1) * 4) ||
        !dalloc(h->dBall, (size_t)W_BALL * N * 4) || !dalloc(h->dCar, (size_t)W_CAR * MAX_CARS * N * 4) ||
        !dalloc(h->dPad, (size_t)W_PAD * NUM_PADS * N * 4) || !dalloc(h->dArena, (size_t)W_ARENA * N * 4) ||
        !dalloc(h->dControls, std::max<size_t>(1, h->numCars) * sizeof(rsb_controls)) ||
        !dalloc(h->dActions, std::max<size_t>(1, h->numCars) * 4) ||
        !dalloc(h->dObs, (size_t)h->numCars * h->obsStride * 4) ||
        !dalloc(h->dMasks, (size_t)h->numCars * RSB_NUM_ACTIONS) ||
        !dalloc(h->dRewards, (size_t)h->numCars * 4) || !dalloc(h->dTerminals, N) ||
        !dalloc(h->dResetIdx, N * 4))
        return fail(nullptr, RSB_ERR_NOMEM, "device allocation failed");
    cudaMemcpy(h->dTeamSize, h->teamSize.data(), N * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(h->dCarOffset, h->carOffset.data(), (N + 1) * 4, cudaMemcpyHostToDevice);
    {
        HostRecords R;
        initRecords(h->stat->view, h->P, h->teamSize, R);
        cudaMemcpy(h->dBall, R.ball.data(), R.ball.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(h->dCar, R.car.data(), R.car.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(h->dArena, R.arena.data(), R.arena.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(h->dPad, R.pad.data(), R.pad.size() * 4, cudaMemcpyHostToDevice);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(nullptr, RSB_ERR_CUDA, "initial upload failed");
    *out = hp.release();
    return RSB_OK;
}

rsb_status rsb_destroy(rsb_handle* h) {
    if (!h) return RSB_ERR_INVALID;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->dTeamSize); cudaFree(h->dCarOffset); cudaFree(h->dBall); cudaFree(h->dCar);
    cudaFree(h->dPad); cudaFree(h->dArena); cudaFree(h->dControls); cudaFree(h->dLut); cudaFree(h->dActions);
    cudaFree(h->dScratch);
    cudaFree(h->dObs); cudaFree(h->dMasks); cudaFree(h->dRewards); cudaFree(h->dTerminals); cudaFree(h->dResetIdx);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return RSB_OK;
}

rsb_status rsb_layout(const rsb_handle* h, int32_t* num_arenas, int32_t* num_cars, int32_t* car_offset,
                      int32_t* team_size) {
    if (!h) return RSB_ERR_INVALID;
    if (num_arenas) *num_arenas = h->N;
    if (num_cars) *num_cars = h->numCars;
    if (car_offset) std::memcpy(car_offset, h->carOffset.data(), h->carOffset.size() * 4);
    if (team_size) std::memcpy(team_size, h->teamSize.data(), h->teamSize.size() * 4);
    return RSB_OK;
}

rsb_status rsb_obs_stride(const rsb_handle* h, int32_t* stride) {
    if (!h || !stride) return RSB_ERR_INVALID;
    *stride = RSB_OBS_BASE + RSB_OBS_PER_CAR * h->maxCars;
    return RSB_OK;
}

rsb_status rsb_step(rsb_handle* h, int32_t ticks, void* stream) {
    if (!h || ticks < 0) return fail(h, RSB_ERR_INVALID, "bad tick count");
    if (ticks == 0) return RSB_OK;
    RSB_CUDA(cudaSetDevice(h->device));
    EngineView D = devView(h);
    int block = kStepBlocks[h->stepBlock], grid = (h->N + block - 1) / block;
    kStepVariants[h->stepVariant].fn<<<grid, block, 0, pick(h, stream)>>>(D, ticks);
    RSB_CUDA(cudaGetLastError());
    h->stats.ticks_simulated += (uint64_t)h->N * ticks;
    return RSB_OK;
}

rsb_status rsb_autotune(rsb_handle* h, int32_t ticks, rsb_tune_entry* out, int32_t cap, int32_t* count) {
    if (!h || ticks <= 0 || cap < 0) return fail(h, RSB_ERR_INVALID, "bad autotune arguments");
    RSB_CUDA(cudaSetDevice(h->device));
    const size_t wBall = (size_t)W_BALL * h->N, wCar = (size_t)W_CAR * MAX_CARS * h->N;
    const size_t wPad = (size_t)W_PAD * NUM_PADS * h->N, wArena = (size_t)W_ARENA * h->N;
    const size_t words = wBall + wCar + wPad + wArena;
    if (!h->dScratch && cudaMalloc((void**)&h->dScratch, words * 4) != cudaSuccess)
        return fail(h, RSB_ERR_NOMEM, "autotune scratch allocation failed");
    EngineView D = devView(h);
    D.ball = h->dScratch;
    D.car = D.ball + wBall;
    D.pad = D.car + wCar;
    D.arena = D.pad + wPad;
    cudaEvent_t e0, e1;
    RSB_CUDA(cudaEventCreate(&e0));
    RSB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int n = 0, bestV = h->stepVariant, bestB = h->stepBlock;
    rsb_status st = RSB_OK;
    for (int v = 0; v < kNumStepVariants && st == RSB_OK; v++)
        for (int b = 0; b < kNumStepBlocks && st == RSB_OK; b++) {
            float ms = 1e30f;
            for (int rep = 0; rep < 2; rep++) {
                // every candidate starts from the same copy of the current state
                cudaError_t e = cudaMemcpyAsync(D.ball, h->dBall, wBall * 4, cudaMemcpyDeviceToDevice, h->stream);
                if (e == cudaSuccess) e = cudaMemcpyAsync(D.car, h->dCar, wCar * 4, cudaMemcpyDeviceToDevice, h->stream);
                if (e == cudaSuccess) e = cudaMemcpyAsync(D.pad, h->dPad, wPad * 4, cudaMemcpyDeviceToDevice, h->stream);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(D.arena, h->dArena, wArena * 4, cudaMemcpyDeviceToDevice, h->stream);
                const int block = kStepBlocks[b], grid = (h->N + block - 1) / block;
                if (e == cudaSuccess) e = cudaEventRecord(e0, h->stream);
                if (e == cudaSuccess) {
                    kStepVariants[v].fn<<<grid, block, 0, h->stream>>>(D, ticks);
                    e = cudaGetLastError();
                }
                if (e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float t = 0.f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
                if (e != cudaSuccess) {
                    st = cudaFail(h, "autotune candidate", e);
                    break;
                }
                ms = std::min(ms, t);
            }
            if (st != RSB_OK) break;
            if (out && n < cap) out[n] = rsb_tune_entry{kStepVariants[v].minBlocks, kStepBlocks[b], ms};
            n++;
            if (ms < best) { best = ms; bestV = v; bestB = b; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RSB_OK) return st;
    h->stepVariant = bestV;
    h->stepBlock = bestB;
    if (count) *count = n;
    return RSB_OK;
}

rsb_status rsb_sync(rsb_handle* h) {
    if (!h) return RSB_ERR_INVALID;
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_set_controls(rsb_handle* h, const rsb_controls* c, int32_t n) {
    if (!h || !c || n != h->numCars) return fail(h, RSB_ERR_INVALID, "controls count must equal num_cars");
    if (n == 0) return RSB_OK;
    RSB_CUDA(cudaMemcpyAsync(h->dControls, c, sizeof(rsb_controls) * n, cudaMemcpyHostToDevice, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_set_action_lut(rsb_handle* h, const rsb_controls* lut, int32_t count) {
    if (!h || !lut || count <= 0) return fail(h, RSB_ERR_INVALID, "bad action table");
    if (h->dLut) cudaFree(h->dLut);
    h->dLut = nullptr;
    RSB_CUDA(cudaMalloc((void**)&h->dLut, sizeof(rsb_controls) * count));
    RSB_CUDA(cudaMemcpy(h->dLut, lut, sizeof(rsb_controls) * count, cudaMemcpyHostToDevice));
    h->lutCount = count;
    return RSB_OK;
}

rsb_status rsb_set_actions_device(rsb_handle* h, const int32_t* d_idx, int32_t n, void* stream) {
    if (!h || n != h->numCars) return fail(h, RSB_ERR_INVALID, "action count must equal num_cars");
    if (!h->dLut) return fail(h, RSB_ERR_STATE, "no action table uploaded");
    if (n == 0) return RSB_OK;
    expandActionsKernel<<<(n + 255) / 256, 256, 0, pick(h, stream)>>>(d_idx, h->dLut, h->lutCount, h->dControls, n);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

rsb_status rsb_set_actions_host(rsb_handle* h, const int32_t* idx, int32_t n) {
    if (!h || !idx || n != h->numCars) return fail(h, RSB_ERR_INVALID, "action count must equal num_cars");
    if (!h->dLut) return fail(h, RSB_ERR_STATE, "no action table uploaded");
    if (n == 0) return RSB_OK;
    RSB_CUDA(cudaMemcpyAsync(h->dActions, idx, 4 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
    return rsb_set_actions_device(h, h->dActions, n, nullptr);
}

rsb_status rsb_set_actions_host_static(rsb_handle* h, const int32_t* idx, int32_t n) {
    if (h && n > RSB_STATIC_ACTIONS_MAX)
        return fail(h, RSB_ERR_INVALID, "rsb_set_actions_host_static: more than RSB_STATIC_ACTIONS_MAX actions");
    if (!h || !idx || n != h->numCars) return fail(h, RSB_ERR_INVALID, "action count must equal num_cars");
    if (!h->dLut) return fail(h, RSB_ERR_STATE, "no action table uploaded");
    if (n == 0) return RSB_OK;
    RSB_CUDA(cudaSetDevice(h->device));
    int32_t* stage = nullptr;
    {
        StaticActionsAddr& s = staticActionsAddr();
        std::lock_guard<std::mutex> lock(s.mu);
        auto it = s.ptr.find(h->device);
        if (it == s.ptr.end()) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_staticActions);
            if (e != cudaSuccess) return cudaFail(h, "cudaGetSymbolAddress(g_staticActions)", e);
            it = s.ptr.emplace(h->device, static_cast<int32_t*>(p)).first;
        }
        stage = it->second;
    }
    RSB_CUDA(cudaMemcpyAsync(stage, idx, 4 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
    expandActionsKernel<<<(n + 255) / 256, 256, 0, h->stream>>>(stage, h->dLut, h->lutCount, h->dControls, n);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

rsb_status rsb_get_balls(rsb_handle* h, rsb_ball_state* out, int32_t n) {
    if (!h || !out || n != h->N) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dBall, planes, (size_t)W_BALL * h->N);
    if (st) return st;
    for (int a = 0; a < n; a++) {
        BallP p;
        loadPlanes(p, planes.data(), a, h->N);
        out[a] = ballStateOf(p);
    }
    return RSB_OK;
}

rsb_status rsb_set_balls(rsb_handle* h, const rsb_ball_state* in, int32_t n) {
    if (!h || !in || n != h->N) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dBall, planes, (size_t)W_BALL * h->N);
    if (st) return st;
    std::vector<uint32_t> arena;
    st = download(h, h->dArena, arena, (size_t)W_ARENA * h->N);
    if (st) return st;
    for (int a = 0; a < n; a++) {
        BallP p;
        loadPlanes(p, planes.data(), a, h->N);
        applyBallState(p, in[a]);
        storePlanes(p, planes.data(), a, h->N);
        // keep the arena's goal-line flag in step with the new ball position
        ArenaP ap;
        loadPlanes(ap, arena.data(), a, h->N);
        float y = p.pos[1] * kBtToUu;
        ap.scored = fabsf(y) > (h->P.goalBaseY + h->P.ballRadiusUu) ? (p.pos[1] > 0 ? 1 : 2) : 0;
        storePlanes(ap, arena.data(), a, h->N);
    }
    st = upload(h, h->dArena, arena);
    if (st) return st;
    return upload(h, h->dBall, planes);
}

rsb_status rsb_get_cars(rsb_handle* h, rsb_car_state* out, int32_t n) {
    if (!h || (n > 0 && !out) || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    if (n == 0) return RSB_OK;
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dCar, planes, (size_t)W_CAR * MAX_CARS * h->N);
    if (st) return st;
    for (int a = 0; a < h->N; a++)
        for (int s = 0; s < 2 * h->teamSize[a]; s++) {
            CarP p;
            loadPlanes(p, planes.data(), s * h->N + a, MAX_CARS * h->N);
            out[h->carOffset[a] + s] = carStateOf(p, (uint32_t)s + 1u);
        }
    return RSB_OK;
}

rsb_status rsb_set_cars(rsb_handle* h, const rsb_car_state* in, int32_t n) {
    if (!h || (n > 0 && !in) || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    if (n == 0) return RSB_OK;
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dCar, planes, (size_t)W_CAR * MAX_CARS * h->N);
    if (st) return st;
    for (int a = 0; a < h->N; a++)
        for (int s = 0; s < 2 * h->teamSize[a]; s++) {
            CarP p;
            loadPlanes(p, planes.data(), s * h->N + a, MAX_CARS * h->N);
            applyCarState(p, in[h->carOffset[a] + s]);
            storePlanes(p, planes.data(), s * h->N + a, MAX_CARS * h->N);
        }
    return upload(h, h->dCar, planes);
}

rsb_status rsb_get_pads(rsb_handle* h, rsb_pad_state* out, int32_t n) {
    if (!h || !out || n != h->N * RSB_NUM_PADS) return fail(h, RSB_ERR_INVALID, "pad count must equal num_arenas*34");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dPad, planes, (size_t)W_PAD * NUM_PADS * h->N);
    if (st) return st;
    for (int a = 0; a < h->N; a++)
        for (int p = 0; p < NUM_PADS; p++) {
            PadP pp;
            loadPlanes(pp, planes.data(), p * h->N + a, h->N * NUM_PADS);
            rsb_pad_state& o = out[a * NUM_PADS + p];
            o = rsb_pad_state{};
            o.is_active = pp.bits & 1;
            o.cooldown = pp.cooldown;
            o.prev_locked_car_id = pp.bits >> 8;
        }
    return RSB_OK;
}

rsb_status rsb_set_pads(rsb_handle* h, const rsb_pad_state* in, int32_t n) {
    if (!h || !in || n != h->N * RSB_NUM_PADS) return fail(h, RSB_ERR_INVALID, "pad count must equal num_arenas*34");
    std::vector<uint32_t> planes((size_t)W_PAD * NUM_PADS * h->N);
    for (int a = 0; a < h->N; a++)
        for (int p = 0; p < NUM_PADS; p++) {
            const rsb_pad_state& s = in[a * NUM_PADS + p];
            PadP pp;
            pp.cooldown = s.cooldown;
            pp.bits = (s.is_active ? 1u : 0u) | (s.prev_locked_car_id << 8);
            storePlanes(pp, planes.data(), p * h->N + a, h->N * NUM_PADS);
        }
    return upload(h, h->dPad, planes);
}

rsb_status rsb_get_arena_info(rsb_handle* h, rsb_arena_info* out, int32_t n) {
    if (!h || !out || n != h->N) return fail(h, RSB_ERR_INVALID, "info count must equal num_arenas");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dArena, planes, (size_t)W_ARENA * h->N);
    if (st) return st;
    for (int a = 0; a < n; a++) {
        ArenaP ap;
        loadPlanes(ap, planes.data(), a, h->N);
        rsb_arena_info& o = out[a];
        o = rsb_arena_info{};
        o.tick_count = (uint64_t)ap.tick[0] | ((uint64_t)ap.tick[1] << 32);
        o.num_cars = 2 * h->teamSize[a];
        o.team_size = h->teamSize[a];
        o.goal_scored = ap.scored != 0;
        o.goal_team = ap.scored == 1 ? 0 : (ap.scored == 2 ? 1 : -1);
        o.episode_ticks = ap.episodeTicks;
        o.status = ap.status;
    }
    return RSB_OK;
}

rsb_status rsb_stats_get(rsb_handle* h, rsb_stats* out) {
    if (!h || !out) return RSB_ERR_INVALID;
    *out = h->stats;
    return RSB_OK;
}

rsb_status rsb_last_error(const rsb_handle* h, char* buf, size_t n) {
    if (!buf || n == 0) return RSB_ERR_INVALID;
    const std::string& s = h ? h->err : g_createError;
    std::snprintf(buf, n, "%s", s.c_str());
    return RSB_OK;
}

rsb_status rsb_device_ptr(rsb_handle* h, int32_t which, void** out) {
    if (!h || !out) return RSB_ERR_INVALID;
    switch (which) {
        case RSB_BUF_OBS: *out = h->dObs; return RSB_OK;
        case RSB_BUF_MASKS: *out = h->dMasks; return RSB_OK;
        case RSB_BUF_REWARDS: *out = h->dRewards; return RSB_OK;
        case RSB_BUF_TERMINALS: *out = h->dTerminals; return RSB_OK;
        case RSB_BUF_CONTROLS: *out = h->dControls; return RSB_OK;
        case RSB_BUF_ACTIONS: *out = h->dActions; return RSB_OK;
        default: return fail(h, RSB_ERR_INVALID, "unknown buffer");
    }
}

rsb_status rsb_reset_arenas(rsb_handle* h, const int32_t* idx, int32_t n, uint64_t seed, int32_t mode) {
    if (!h || n < 0 || (n > 0 && !idx) || n > h->N) return fail(h, RSB_ERR_INVALID, "bad reset arena list");
    if (mode < RSB_RESET_KICKOFF || mode > RSB_RESET_HIGH_CONTACT) return fail(h, RSB_ERR_INVALID, "unknown reset mode");
    for (int i = 0; i < n; i++)
        if (idx[i] < 0 || idx[i] >= h->N) return fail(h, RSB_ERR_INVALID, "arena index out of range");
    if (n == 0) return RSB_OK;
    RSB_CUDA(cudaSetDevice(h->device));
    RSB_CUDA(cudaMemcpyAsync(h->dResetIdx, idx, 4 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
    resetKernel<<<(n + 127) / 128, 128, 0, h->stream>>>(envView(h), h->tables, h->dResetIdx, n, seed, mode, false);
    RSB_CUDA(cudaGetLastError());
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_reset_all(rsb_handle* h, uint64_t seed, int32_t mode) {
    if (!h) return RSB_ERR_INVALID;
    if (mode < RSB_RESET_KICKOFF || mode > RSB_RESET_HIGH_CONTACT) return fail(h, RSB_ERR_INVALID, "unknown reset mode");
    RSB_CUDA(cudaSetDevice(h->device));
    resetKernel<<<(h->N + 127) / 128, 128, 0, h->stream>>>(envView(h), h->tables, nullptr, h->N, seed, mode, false);
    RSB_CUDA(cudaGetLastError());
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_reset_done(rsb_handle* h, uint64_t seed, int32_t mode, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    if (mode < RSB_RESET_KICKOFF || mode > RSB_RESET_HIGH_CONTACT) return fail(h, RSB_ERR_INVALID, "unknown reset mode");
    RSB_CUDA(cudaSetDevice(h->device));
    resetKernel<<<(h->N + 127) / 128, 128, 0, pick(h, stream)>>>(envView(h), h->tables, nullptr, h->N, seed, mode, true);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

rsb_status rsb_default_action_lut(rsb_controls* out, int32_t cap) {
    if (!out || cap < RSB_NUM_ACTIONS) return RSB_ERR_INVALID;
    return defaultActionLut(out, cap) == RSB_NUM_ACTIONS ? RSB_OK : RSB_ERR_STATE;
}

// The four stub rewards read no state from before the step (CommonRewards.h:33-98), so
// there is nothing to copy; the call stays for the reference's call sequence.
rsb_status rsb_snapshot(rsb_handle* h, void*) { return h ? RSB_OK : RSB_ERR_INVALID; }

rsb_status rsb_build_obs(rsb_handle* h, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    RSB_CUDA(cudaSetDevice(h->device));
    obsKernel<<<(h->N + OBS_ARENAS - 1) / OBS_ARENAS, 32, 0, pick(h, stream)>>>(envView(h), h->tables);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

rsb_status rsb_build_rewards_terminals(rsb_handle* h, int32_t step_ticks, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    if (!h->hasRewards) return fail(h, RSB_ERR_STATE, "no reward configuration at create");
    RSB_CUDA(cudaSetDevice(h->device));
    rewardKernel<<<(h->N + 127) / 128, 128, 0, pick(h, stream)>>>(envView(h), h->rewardParams, step_ticks);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

static rsb_status copyOut(rsb_handle* h, void* out, const void* dev, size_t count, size_t expect, size_t elem,
                          const char* what) {
    if (!h || !out) return RSB_ERR_INVALID;
    if (count != expect) return fail(h, RSB_ERR_INVALID, std::string(what) + ": count must equal the buffer size");
    RSB_CUDA(cudaSetDevice(h->device));
    RSB_CUDA(cudaMemcpyAsync(out, dev, count * elem, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}
rsb_status rsb_copy_obs(rsb_handle* h, float* out, size_t n) {
    return copyOut(h, out, h ? h->dObs : nullptr, n, h ? (size_t)h->numCars * h->obsStride : 0, 4, "obs");
}
rsb_status rsb_copy_masks(rsb_handle* h, uint8_t* out, size_t n) {
    return copyOut(h, out, h ? h->dMasks : nullptr, n, h ? (size_t)h->numCars * RSB_NUM_ACTIONS : 0, 1, "masks");
}
rsb_status rsb_copy_rewards(rsb_handle* h, float* out, size_t n) {
    return copyOut(h, out, h ? h->dRewards : nullptr, n, h ? (size_t)h->numCars : 0, 4, "rewards");
}
rsb_status rsb_copy_terminals(rsb_handle* h, uint8_t* out, size_t n) {
    return copyOut(h, out, h ? h->dTerminals : nullptr, n, h ? (size_t)h->N : 0, 1, "terminals");
}

}  // extern "C"
