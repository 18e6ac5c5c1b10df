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
#include <set>
#include <string>
#include <vector>

#include "rsb.h"
#include "arena_build.h"
#include "engine_host.h"
#include "env_kernels.cuh"
#include "culler.cuh"
#include "vanta.cuh"

#include <numeric>
#include <random>

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
    uint16_t* occ = nullptr;
    uint32_t* voxOff = nullptr;
    uint32_t* voxList = nullptr;
    uint16_t* occDist = nullptr;
    ArenaStatic view{};
};

// Host build + device copy of the arena data, shared per (device, meshes folder).
struct StaticCache {
    std::mutex mu;
    std::map<std::string, std::shared_ptr<ArenaStaticHost>> host;
    std::map<std::pair<int, std::string>, std::shared_ptr<DevStatic>> dev;
    // rsqrtss table of the host CPU, sampled once; rsqrtExact is false when the CPU's
    // estimate is not a function of exponent parity and 12 mantissa bits
    bool rsqrtSampled = false, rsqrtExact = false;
    uint32_t rsqrtTable[kRsqrtTableSize];
    std::set<int> rsqrtDevices;  // devices whose g_rsqrtTable holds rsqrtTable
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
    // learned culler
    int cullMode = RSB_CULL_EXACT;
    float cullSlack = 0.f;                 // rsb_config.cull_margin: extra uu on top of the calibrated margin
    bool cullerReady = false;
    CullParams cullParams{};
    float* dCw = nullptr;                  // FP32 master weights, Adam moments, gradient (4 x CM_NPARAM)
    __nv_bfloat16* dCwBf = nullptr;        // BF16 weights used by every forward pass
    uint32_t* dCull = nullptr;             // per-arena body bits of the current launch
    unsigned long long* dCounters = nullptr;  // static tests run / culled / culled-but-hit
    float* dLog = nullptr;                 // logged body centres (uu), for training
    int64_t logCount = 0, logCap = 0;
    float* dTris = nullptr;                // mesh triangles in uu (9 floats each)
    int numTris = 0;
    std::shared_ptr<ArenaStaticHost> host;
    // launch configuration of the step kernel (indices into kStepVariants / kStepBlocks)
    int stepVariant = 0, stepBlock = 1, stepResidency = 0;
    uint32_t* dScratch = nullptr;   // the autotuner's copy of the arena records
    unsigned int* dWork = nullptr;  // claim counter of the persistent step kernel
    int persistGrid[8][4] = {};     // resident blocks (all SMs) per persistent variant and block size
    int smCount = 0;
    uint32_t* dStage = nullptr;     // staging of the per-arena getters
    rsb_ball_state* dPred = nullptr;  // ball prediction slices [num_arenas][n_slices]
    size_t predCap = 0;
    size_t stageWords = 0;
    EnvTables tables{};
    // VantaObs builder (rsb_vanta_configure)
    uint32_t* dVA = nullptr;
    uint32_t* dVT = nullptr;
    rsb_ball_state* dVantaPred = nullptr;
    float* dVantaRows = nullptr;
    rsb_vanta_config vanta{};
    VantaTables vantaTables{};
    // captured env step (rsb_env_graph_capture)
    cudaGraphExec_t envGraph = nullptr;
    uint64_t* dGraphSeed = nullptr;
    int graphTicks = 0;
    ResetCurriculum curriculum{{1.f, 0.f, 0.f, 0.f}, 0.f};
    bool hasRewards = false;
    RewardParams rewardParams{};
    std::string err;
    rsb_stats stats{};
    // state ring (rsb_ring_*)
    struct Ring {
        bool enabled = false, replayDisabled = false;
        rsb_ring_config cfg{};
        uint32_t rng = 0xA5A5A5A5u;
        uint32_t* dSlots = nullptr;  // depth slots, each [ball planes | car planes | pad planes]
        size_t slotWords = 0;
        int writeIdx = 0, filled = 0, stepsSinceCapture = 0;
        uint64_t captures = 0, restores = 0, restoreCalls = 0;
        uint32_t* dJobs = nullptr;   // per rewound arena: its index and the xorshift state of its first draw
        int jobCap = 0;
        std::vector<uint32_t> jobs;
    } ring;
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

// Persistent form: the grid holds only as many blocks as fit on the GPU at once, and each warp
// claims the next 32 arenas from a counter until none are left.  One arena per thread still,
// and the same per-arena computation; the claims pack the work that one-arena-per-thread
// blocks leave in a partial last wave (65,536 arenas are about 1.7 waves of resident warps).
// No waiting: a claim is one atomic add.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) stepKernelPersistent(EngineView D, int ticks) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int base = 0;
        if (lane == 0) base = (int)atomicAdd(D.work, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= D.N) return;
        const int a = base + lane;
        if (a < D.N) {
            ArenaSim A;
            EpaWork epa;
            A.W.epa = &epa;
            stepArena(D, a, ticks, A);
        }
    }
}

struct StepVariant {
    void (*fn)(EngineView, int);
    int minBlocks;
    bool persistent;
};
static const StepVariant kStepVariants[] = {{stepKernel<1>, 1, false},          {stepKernel<3>, 3, false},
                                            {stepKernel<4>, 4, false},          {stepKernelPersistent<1>, 1, true},
                                            {stepKernelPersistent<3>, 3, true}, {stepKernelPersistent<4>, 4, true}};
constexpr int kNumStepVariants = sizeof(kStepVariants) / sizeof(kStepVariants[0]);
static const int kStepBlocks[] = {32, 64, 128};
constexpr int kNumStepBlocks = sizeof(kStepBlocks) / sizeof(kStepBlocks[0]);
// Resident warps per SM of a persistent launch (0 = as many as fit).  The working sets of the
// arenas in flight share the L2: with every warp slot filled (about 38,000 arenas at a time)
// they do not fit, and each thread waits on DRAM; fewer arenas in flight stay in L2.
static const int kStepResidency[] = {0, 1, 2, 3, 4, 6};
constexpr int kNumStepResidency = sizeof(kStepResidency) / sizeof(kStepResidency[0]);

// xorshift32 draw in [0, 1] and range of the reference's state ring (CudaEnvSet.cpp:608-617)
RSB_HD float ringRand01(uint32_t& rng) {
    rng ^= rng << 13;
    rng ^= rng >> 17;
    rng ^= rng << 5;
    return (rng & 0xFFFFFFu) / float(0xFFFFFFu);
}
RSB_HD float ringRange(uint32_t& rng, float lo, float hi) { return lo + (hi - lo) * ringRand01(rng); }

// Rewinds the listed arenas to a ring slot (ApplyArenaSnap, CudaEnvSet.cpp:698-753): for each
// car the slot's public state (Car::GetState) jittered and written over the live car as
// Car::SetState writes it, then the ball, then the pads (their public fields).  One thread per
// listed arena; jobs[2 j] = arena, jobs[2 j + 1] = xorshift state of its first draw.
__global__ void ringRestoreKernel(uint32_t* ball, uint32_t* car, uint32_t* pad, uint32_t* arena,
                                  const int32_t* teamSize, const uint32_t* sBall, const uint32_t* sCar,
                                  const uint32_t* sPad, const uint32_t* jobs, int n, int N, float fp, float fv,
                                  float goalLine) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int a = (int)jobs[2 * j];
    uint32_t rng = jobs[2 * j + 1];
    const int cars = 2 * teamSize[a];
    for (int s = 0; s < cars; s++) {
        CarP live, snap;
        loadPlanes(live, car, s * N + a, MAX_CARS * N);
        loadPlanes(snap, sCar, s * N + a, MAX_CARS * N);
        rsb_car_state st = carStateOf(snap, (uint32_t)s + 1u);
        if (fp > 0.f) {
            st.pos.x += ringRange(rng, -fp, fp);
            st.pos.y += ringRange(rng, -fp, fp);
            const float z = st.pos.z + ringRange(rng, -fp * 0.25f, fp * 0.35f);
            st.pos.z = 17.f < z ? z : 17.f;
        }
        if (fv > 0.f) {
            st.vel.x += ringRange(rng, -fv, fv);
            st.vel.y += ringRange(rng, -fv, fv);
            st.vel.z += ringRange(rng, -fv * 0.5f, fv * 0.5f);
        }
        applyCarState(live, st);
        storePlanes(live, car, s * N + a, MAX_CARS * N);
    }
    BallP live, snap;
    loadPlanes(live, ball, a, N);
    loadPlanes(snap, sBall, a, N);
    rsb_ball_state bs = ballStateOf(snap);
    if (fp > 0.f) {
        bs.pos.x += ringRange(rng, -fp, fp);
        bs.pos.y += ringRange(rng, -fp, fp);
        const float z = bs.pos.z + ringRange(rng, -fp * 0.2f, fp * 0.4f);
        bs.pos.z = 93.f < z ? z : 93.f;
    }
    if (fv > 0.f) {
        bs.vel.x += ringRange(rng, -fv, fv);
        bs.vel.y += ringRange(rng, -fv, fv);
        bs.vel.z += ringRange(rng, -fv * 0.5f, fv * 0.5f);
    }
    applyBallState(live, bs);
    storePlanes(live, ball, a, N);
    // the goal-line flag follows the new ball position, as rsb_set_balls keeps it
    ArenaP ap;
    loadPlanes(ap, arena, a, N);
    const float y = live.pos[1] * kBtToUu;
    ap.scored = fabsf(y) > goalLine ? (live.pos[1] > 0 ? 1 : 2) : 0;
    storePlanes(ap, arena, a, N);
    for (int p = 0; p < NUM_PADS; p++) {
        PadP pp;
        loadPlanes(pp, sPad, p * N + a, N * NUM_PADS);
        pp.bits = (pp.bits & 1u) | ((pp.bits >> 8) << 8);  // is_active and prev_locked_car_id
        storePlanes(pp, pad, p * N + a, N * NUM_PADS);
    }
}

// Single-record access for the per-arena getters and setters: gathers `count` records of
// `words` words (record r at base + r * recStep, word stride `stride`) into out[r * words + w].
__global__ void gatherRecordsKernel(const uint32_t* planes, int base, int recStep, int count, int stride, int words,
                                    uint32_t* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count * words) return;
    const int r = i / words, w = i % words;
    out[i] = planes[(size_t)w * stride + base + (size_t)r * recStep];
}

// Car::SetState on one car record (the host setter's conversion, on the device).
__global__ void setCarKernel(uint32_t* car, int idx, int stride, rsb_car_state s) {
    CarP p;
    loadPlanes(p, car, idx, stride);
    applyCarState(p, s);
    storePlanes(p, car, idx, stride);
}

// Ball::SetState on one arena's ball, with the goal-line flag kept in step (as rsb_set_balls).
__global__ void setBallKernel(uint32_t* ball, uint32_t* arena, int a, int N, rsb_ball_state s, float goalLine) {
    BallP p;
    loadPlanes(p, ball, a, N);
    applyBallState(p, s);
    storePlanes(p, ball, a, N);
    ArenaP ap;
    loadPlanes(ap, arena, a, N);
    const float y = p.pos[1] * kBtToUu;
    ap.scored = fabsf(y) > goalLine ? (p.pos[1] > 0 ? 1 : 2) : 0;
    storePlanes(ap, arena, a, N);
}

struct PadSet {
    rsb_pad_state p[NUM_PADS];
};

// BoostPad::SetState on the 34 pads of one arena.
__global__ void setPadsKernel(uint32_t* pad, int a, int N, PadSet s) {
    const int p = threadIdx.x;
    if (p >= NUM_PADS) return;
    PadP pp;
    pp.cooldown = s.p[p].cooldown;
    pp.bits = (s.p[p].is_active ? 1u : 0u) | (s.p[p].prev_locked_car_id << 8);
    storePlanes(pp, pad, p * N + a, N * NUM_PADS);
}

struct PredSlices {
    int32_t t[RSB_MAX_PRED_SLICES];
    int32_t n;
};

// BallPredTracker::ForceUpdateAllPred (BallPredTracker.cpp:80-88) for every arena at once: the
// arena's ball passes through Ball::GetState / Ball::SetState into a world of its own with no
// cars, which steps one tick at a time (Arena::Step of a ball-only arena); out[a * n + k] is the
// ball after s.t[k] ticks.  The arena's own records are only read.  At most 128 registers a
// thread, so that 4 blocks share an SM and 65,536 arenas run in one wave (103 ms against 116 ms
// at 168 registers for 3v3 x 65,536 x 360 ticks; identical results).
__global__ void __launch_bounds__(128, 4) predictBallKernel(EngineView D, PredSlices s, rsb_ball_state* out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= D.N) return;
    ArenaSim A;
    EpaWork epa;
    World& W = A.W;
    W.epa = &epa;
    W.S = &D.S;
    W.P = &D.P;
    A.teamSize = A.numCars = 0;
    W.nc = 0;
    W.nb = 1;
    W.status = 0;
    W.noRot[0] = 1;
    BallP p;
    loadPlanes(p, D.ball, a, D.N);
    applyBallState(p, ballStateOf(p));
    ballBodyOf(D, p, W.b[0]);
    A.tickCount = 0;
    A.status = 0;
    A.goalTeam = -1;
    A.touchedMask = 0;
    A.rngKey = 0;
    W.cull = 0;
    W.cullAudit = 0;
    W.nStatic = W.nCulled = W.nMissed = 0;
    W.cullMissed = 0;
    W.nRows = 0;
    int t = 0;
    for (int k = 0; k < s.n; k++) {
        for (; t < s.t[k]; t++) arenaTick(A);
        out[(size_t)a * s.n + k] = ballStateOf(ballRecordOf(W.b[0]));
    }
}

__global__ void expandActionsKernel(const int32_t* idx, const rsb_controls* lut, int lutCount, rsb_controls* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = idx[i];
    k = k < 0 ? 0 : (k >= lutCount ? lutCount - 1 : k);
    out[i] = lut[k];
}

// The restated float functions of phys/refmath.h on n inputs (rsb_eval_refmath).
__global__ void refMathKernel(int fn, const float* x, const float* y, float* out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = x[i];
    float r;
    switch (fn) {
        case RSB_MATH_RSQRT_EST: r = rsqrtEstimate(v); break;
        case RSB_MATH_SIN: r = rsSinf(v); break;
        case RSB_MATH_COS: r = rsCosf(v); break;
        case RSB_MATH_ASIN: r = rsAsinf(v); break;
        default: r = rsAtan2f(v, y[i]); break;
    }
    out[i] = r;
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
    D.cull = nullptr;
    D.cullAudit = h->cullMode == RSB_CULL_LEARNED_AUDIT || h->cullMode == RSB_CULL_VOXEL_AUDIT;
    D.counters = h->dCounters;
    D.work = h->dWork;
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
    E.vantaArena = h->dVA;
    E.vantaCar = h->dVT;
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
    if (cfg->cull_mode < RSB_CULL_EXACT || cfg->cull_mode > RSB_CULL_VOXEL_AUDIT)
        return fail(nullptr, RSB_ERR_INVALID, "unknown cull mode");
    h->cullMode = cfg->cull_mode;
    h->cullSlack = cfg->cull_margin;
    {
        // reach of each body's static tests around its centre (uu): the car's box and its
        // four wheel rays, the ball's sphere, each plus its contact-breaking threshold
        const CarParams& C = h->P.car;
        float box = length(C.childOff) + length(C.boxHeM);
        float rays = 0.f;
        for (int w = 0; w < 4; w++) rays = std::max(rays, length(C.wheelConn[w]) + C.rayLen[w]);
        CullParams& cp = h->cullParams;
        cp.carReach = (std::max(box, rays) + C.cbt) * kBtToUu + 10.f;
        cp.ballReach = (h->P.ballRadius + h->P.ballCbt) * kBtToUu + 10.f;
        cp.carVmax = 5000.f;   // above the 2300 uu/s clamp: bumps land on top of it within a tick
        cp.ballVmax = 8000.f;  // above the 6000 uu/s clamp for the same reason
        cp.dt = h->P.dt;
    }
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
        h->curriculum.noTouchTimeout = r.no_touch_timeout_s;
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
        h->host = H;
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
                !up(D->triInfo, H->triInfo) || !up(D->bpCells, H->bpCells) || !up(D->occ, H->occ) ||
                !up(D->voxOff, H->voxOff) || !up(D->voxList, H->voxList) || !up(D->occDist, H->occDist))
                return fail(nullptr, RSB_ERR_CUDA, "uploading arena meshes failed");
            D->view = deviceView(*H, D->nodes, D->subs, D->triVerts, D->triInfo, D->bpCells, D->occ, D->voxOff,
                                 D->voxList, D->occDist);
            // the host CPU's rsqrtss estimate, which btVector3::normalize starts from
            if (!c.rsqrtSampled) {
                c.rsqrtExact = sampleRsqrtTable(c.rsqrtTable);
                c.rsqrtSampled = true;
            }
            if (cudaMemcpyToSymbol(g_rsqrtTable, c.rsqrtTable, sizeof(c.rsqrtTable)) != cudaSuccess)
                return fail(nullptr, RSB_ERR_CUDA, "uploading the rsqrt estimate table failed");
            c.rsqrtDevices.insert(h->device);
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
        !dalloc(h->dResetIdx, N * 4) || !dalloc(h->dCull, N * 4) ||
        !dalloc(h->dCounters, 4 * sizeof(unsigned long long)) || !dalloc(h->dWork, sizeof(unsigned int)))
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
    cudaFree(h->dCw); cudaFree(h->dCwBf); cudaFree(h->dCull); cudaFree(h->dCounters); cudaFree(h->dLog);
    cudaFree(h->dTris);
    cudaFree(h->dObs); cudaFree(h->dMasks); cudaFree(h->dRewards); cudaFree(h->dTerminals); cudaFree(h->dResetIdx);
    cudaFree(h->dVA);
    cudaFree(h->dVT);
    cudaFree(h->dVantaPred);
    cudaFree(h->dVantaRows);
    if (h->envGraph) cudaGraphExecDestroy(h->envGraph);
    cudaFree(h->dGraphSeed);
    cudaFree(h->ring.dSlots); cudaFree(h->ring.dJobs); cudaFree(h->dStage); cudaFree(h->dWork); cudaFree(h->dPred);
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

// Launches step-kernel variant v with block size index b on stream st (a persistent variant
// first zeroes its claim counter on the same stream).
static cudaError_t launchStep(rsb_handle* h, const EngineView& D, int v, int b, int ticks, cudaStream_t st,
                              int residency = 0) {
    const StepVariant& sv = kStepVariants[v];
    const int block = kStepBlocks[b];
    int grid = (h->N + block - 1) / block;
    if (sv.persistent) {
        int& g = h->persistGrid[v][b];
        if (g == 0) {
            int perSm = 0, sms = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, sv.fn, block, 0);
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
            if (e != cudaSuccess) return e;
            h->smCount = sms;
            g = std::max(1, perSm * sms);
        }
        int cap = g;
        if (kStepResidency[residency] > 0) {
            const int blocksPerSm = std::max(1, kStepResidency[residency] * 32 / block);
            cap = std::min(g, blocksPerSm * h->smCount);
        }
        grid = std::min(grid, cap);
        cudaError_t e = cudaMemsetAsync(h->dWork, 0, sizeof(unsigned int), st);
        if (e != cudaSuccess) return e;
    }
    sv.fn<<<grid, block, 0, st>>>(D, ticks);
    return cudaGetLastError();
}

rsb_status rsb_step(rsb_handle* h, int32_t ticks, void* stream) {
    if (!h || ticks < 0) return fail(h, RSB_ERR_INVALID, "bad tick count");
    if (ticks == 0) return RSB_OK;
    RSB_CUDA(cudaSetDevice(h->device));
    EngineView D = devView(h);
    cudaStream_t st = pick(h, stream);
    const bool voxel = h->cullMode == RSB_CULL_VOXEL || h->cullMode == RSB_CULL_VOXEL_AUDIT;
    if (h->cullMode != RSB_CULL_EXACT && (h->cullerReady || voxel)) {
        const ArenaStatic& S = h->stat->view;
        const VoxelBound vb{S.occDist, S.occMin, S.occInvCell, S.occX, S.occY, S.occZ};
        auto k = voxel ? cullKernel<true> : cullKernel<false>;
        k<<<(h->N + 127) / 128, 128, 0, st>>>(h->dCwBf, vb, h->cullParams, h->dBall, h->dCar, h->dArena, h->dTeamSize,
                                             h->N, ticks, h->dCull, (int)(offsetof(ArenaP, status) / 4),
                                             WS_CULL_MISS);
        RSB_CUDA(cudaGetLastError());
        D.cull = h->dCull;
    }
    RSB_CUDA(launchStep(h, D, h->stepVariant, h->stepBlock, ticks, st, h->stepResidency));
    h->stats.ticks_simulated += (uint64_t)h->N * ticks;
    return RSB_OK;
}

rsb_status rsb_predict_ball(rsb_handle* h, const int32_t* slice_ticks, int32_t n_slices, rsb_ball_state* out,
                            size_t out_count, void* stream) {
    if (!h || !slice_ticks || n_slices < 1 || n_slices > RSB_MAX_PRED_SLICES)
        return fail(h, RSB_ERR_INVALID, "rsb_predict_ball: 1..8 slice ticks are required");
    PredSlices s{};
    s.n = n_slices;
    for (int k = 0; k < n_slices; k++) {
        const int32_t prev = k ? slice_ticks[k - 1] : 0;
        if (slice_ticks[k] <= prev || slice_ticks[k] > RSB_MAX_PRED_TICKS)
            return fail(h, RSB_ERR_INVALID, "rsb_predict_ball: slice ticks must rise, from 1 to 4096");
        s.t[k] = slice_ticks[k];
    }
    const size_t need = (size_t)h->N * n_slices;
    if (out && out_count != need) return fail(h, RSB_ERR_INVALID, "rsb_predict_ball: out_count must be num_arenas * n_slices");
    RSB_CUDA(cudaSetDevice(h->device));
    if (!h->dPred) {
        // sized for the most slices once, so that the RSB_BUF_BALL_PRED pointer never changes
        const size_t cap = (size_t)h->N * RSB_MAX_PRED_SLICES;
        if (cudaMalloc((void**)&h->dPred, cap * sizeof(rsb_ball_state)) != cudaSuccess)
            return fail(h, RSB_ERR_NOMEM, "rsb_predict_ball: allocation failed");
        h->predCap = cap;
    }
    cudaStream_t st = pick(h, stream);
    predictBallKernel<<<(h->N + 127) / 128, 128, 0, st>>>(devView(h), s, h->dPred);
    RSB_CUDA(cudaGetLastError());
    if (out) {
        RSB_CUDA(cudaMemcpyAsync(out, h->dPred, need * sizeof(rsb_ball_state), cudaMemcpyDeviceToHost, st));
        RSB_CUDA(cudaStreamSynchronize(st));
    }
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
    int n = 0, bestV = h->stepVariant, bestB = h->stepBlock, bestR = h->stepResidency;
    rsb_status st = RSB_OK;
    // every (variant, block) with all warp slots filled; the residency caps on the persistent
    // variant with the largest register budget, at 32 and 64 threads per block
    struct Cand { int v, b, r; };
    std::vector<Cand> cands;
    for (int v = 0; v < kNumStepVariants; v++)
        for (int b = 0; b < kNumStepBlocks; b++) cands.push_back({v, b, 0});
    for (int v = 0; v < kNumStepVariants; v++)
        if (kStepVariants[v].persistent && kStepVariants[v].minBlocks == 1)
            for (int b = 0; b < 2; b++)
                for (int r = 1; r < kNumStepResidency; r++) cands.push_back({v, b, r});
    for (const Cand& c : cands) {
        if (st != RSB_OK) break;
        const int v = c.v, b = c.b;
        {
            float ms = 1e30f;
            for (int rep = 0; rep < 2; rep++) {
                // every candidate starts from the same copy of the current state
                cudaError_t e = cudaMemcpyAsync(D.ball, h->dBall, wBall * 4, cudaMemcpyDeviceToDevice, h->stream);
                if (e == cudaSuccess) e = cudaMemcpyAsync(D.car, h->dCar, wCar * 4, cudaMemcpyDeviceToDevice, h->stream);
                if (e == cudaSuccess) e = cudaMemcpyAsync(D.pad, h->dPad, wPad * 4, cudaMemcpyDeviceToDevice, h->stream);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(D.arena, h->dArena, wArena * 4, cudaMemcpyDeviceToDevice, h->stream);
                if (e == cudaSuccess) e = cudaEventRecord(e0, h->stream);
                if (e == cudaSuccess) e = launchStep(h, D, v, b, ticks, h->stream, c.r);
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
            if (out && n < cap)
                out[n] = rsb_tune_entry{kStepVariants[v].minBlocks, kStepBlocks[b], ms,
                                        kStepVariants[v].persistent ? 1 : 0, kStepResidency[c.r]};
            n++;
            if (ms < best) { best = ms; bestV = v; bestB = b; bestR = c.r; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RSB_OK) return st;
    h->stepVariant = bestV;
    h->stepBlock = bestB;
    h->stepResidency = bestR;
    if (count) *count = n;
    return RSB_OK;
}

rsb_status rsb_set_step_config(rsb_handle* h, const rsb_tune_entry* cfg) {
    if (!h || !cfg) return RSB_ERR_INVALID;
    int r = -1;
    for (int k = 0; k < kNumStepResidency; k++)
        if (kStepResidency[k] == cfg->warps_per_sm) r = k;
    if (r < 0 || (r > 0 && !cfg->persistent))
        return fail(h, RSB_ERR_INVALID, "rsb_set_step_config: warps_per_sm must be 0, 1, 2, 3, 4 or 6 (persistent only)");
    for (int v = 0; v < kNumStepVariants; v++)
        for (int b = 0; b < kNumStepBlocks; b++)
            if (kStepVariants[v].minBlocks == cfg->min_blocks && kStepBlocks[b] == cfg->block &&
                kStepVariants[v].persistent == (cfg->persistent != 0)) {
                h->stepVariant = v;
                h->stepBlock = b;
                h->stepResidency = r;
                return RSB_OK;
            }
    return fail(h, RSB_ERR_INVALID, "rsb_set_step_config: no such launch configuration");
}

rsb_status rsb_eval_refmath(int32_t fn, const float* x, const float* y, float* out, int64_t n, int32_t device) {
    rsb_handle* h = nullptr;
    if (fn < RSB_MATH_RSQRT_EST || fn > RSB_MATH_ATAN2 || !x || !out || n < 0 || (fn == RSB_MATH_ATAN2 && !y))
        return fail(h, RSB_ERR_INVALID, "bad function, pointer or count");
    if (n == 0) return RSB_OK;
    if (fn == RSB_MATH_RSQRT_EST) {
        StaticCache& c = cache();
        std::lock_guard<std::mutex> lock(c.mu);
        if (!c.rsqrtDevices.count(device))
            return fail(h, RSB_ERR_STATE, "no rsb_create on this device yet: the rsqrt table is not loaded");
    }
    RSB_CUDA(cudaSetDevice(device));
    const size_t bytes = (size_t)n * 4;
    float *dx = nullptr, *dy = nullptr, *dout = nullptr;
    auto release = [&] { cudaFree(dx); cudaFree(dy); cudaFree(dout); };
    cudaError_t e = cudaMalloc(&dx, bytes);
    if (e == cudaSuccess && y) e = cudaMalloc(&dy, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && y) e = cudaMemcpy(dy, y, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        refMathKernel<<<(unsigned)((n + 255) / 256), 256>>>(fn, dx, dy, dout, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost);
    release();
    if (e != cudaSuccess) return cudaFail(h, "rsb_eval_refmath", e);
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

static rsb_arena_info arenaInfoOf(const ArenaP& ap, int teamSize) {
    rsb_arena_info o{};
    o.tick_count = (uint64_t)ap.tick[0] | ((uint64_t)ap.tick[1] << 32);
    o.num_cars = 2 * teamSize;
    o.team_size = teamSize;
    o.goal_scored = ap.scored != 0;
    o.goal_team = ap.scored == 1 ? 0 : (ap.scored == 2 ? 1 : -1);
    o.episode_ticks = ap.episodeTicks;
    o.status = ap.status;
    return o;
}

rsb_status rsb_get_arena_info(rsb_handle* h, rsb_arena_info* out, int32_t n) {
    if (!h || !out || n != h->N) return fail(h, RSB_ERR_INVALID, "info count must equal num_arenas");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dArena, planes, (size_t)W_ARENA * h->N);
    if (st) return st;
    for (int a = 0; a < n; a++) {
        ArenaP ap;
        loadPlanes(ap, planes.data(), a, h->N);
        out[a] = arenaInfoOf(ap, h->teamSize[a]);
    }
    return RSB_OK;
}

// ---- one arena at a time (RocketSimCuda.h:349-378): a gather kernel and one small copy, or
// one small kernel, instead of a whole-batch transfer ----

static rsb_status gatherRecords(rsb_handle* h, const uint32_t* planes, int base, int recStep, int count, int stride,
                                int words, std::vector<uint32_t>& out) {
    RSB_CUDA(cudaSetDevice(h->device));
    const size_t need = (size_t)count * words;
    if (h->stageWords < need) {
        cudaFree(h->dStage);
        h->dStage = nullptr;
        h->stageWords = 0;
        RSB_CUDA(cudaMalloc(&h->dStage, need * 4));
        h->stageWords = need;
    }
    gatherRecordsKernel<<<(unsigned)((need + 127) / 128), 128, 0, h->stream>>>(planes, base, recStep, count, stride,
                                                                                 words, h->dStage);
    RSB_CUDA(cudaGetLastError());
    out.resize(need);
    RSB_CUDA(cudaMemcpyAsync(out.data(), h->dStage, need * 4, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

static bool carIndex(const rsb_handle* h, int32_t arena, int32_t car) {
    return arena >= 0 && arena < h->N && car >= 0 && car < 2 * h->teamSize[arena];
}

rsb_status rsb_get_car_at(rsb_handle* h, int32_t arena, int32_t car, rsb_car_state* out) {
    if (!h || !out || !carIndex(h, arena, car)) return fail(h, RSB_ERR_INVALID, "rsb_get_car_at: no such car");
    std::vector<uint32_t> w;
    rsb_status st = gatherRecords(h, h->dCar, car * h->N + arena, 0, 1, MAX_CARS * h->N, W_CAR, w);
    if (st) return st;
    CarP p;
    loadPlanes(p, w.data(), 0, 1);
    *out = carStateOf(p, (uint32_t)car + 1u);
    return RSB_OK;
}

rsb_status rsb_set_car_controls_at(rsb_handle* h, int32_t arena, int32_t car, const rsb_controls* in) {
    if (!h || !in || !carIndex(h, arena, car)) return fail(h, RSB_ERR_INVALID, "rsb_set_car_controls_at: no such car");
    RSB_CUDA(cudaSetDevice(h->device));
    RSB_CUDA(cudaMemcpyAsync(h->dControls + h->carOffset[arena] + car, in, sizeof(rsb_controls),
                             cudaMemcpyHostToDevice, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));  // the caller's struct may go away on return
    return RSB_OK;
}

rsb_status rsb_set_car_at(rsb_handle* h, int32_t arena, int32_t car, const rsb_car_state* in) {
    if (!h || !in || !carIndex(h, arena, car)) return fail(h, RSB_ERR_INVALID, "rsb_set_car_at: no such car");
    RSB_CUDA(cudaSetDevice(h->device));
    setCarKernel<<<1, 1, 0, h->stream>>>(h->dCar, car * h->N + arena, MAX_CARS * h->N, *in);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

rsb_status rsb_get_ball_at(rsb_handle* h, int32_t arena, rsb_ball_state* out) {
    if (!h || !out || arena < 0 || arena >= h->N) return fail(h, RSB_ERR_INVALID, "rsb_get_ball_at: no such arena");
    std::vector<uint32_t> w;
    rsb_status st = gatherRecords(h, h->dBall, arena, 0, 1, h->N, W_BALL, w);
    if (st) return st;
    BallP p;
    loadPlanes(p, w.data(), 0, 1);
    *out = ballStateOf(p);
    return RSB_OK;
}

rsb_status rsb_set_ball_at(rsb_handle* h, int32_t arena, const rsb_ball_state* in) {
    if (!h || !in || arena < 0 || arena >= h->N) return fail(h, RSB_ERR_INVALID, "rsb_set_ball_at: no such arena");
    RSB_CUDA(cudaSetDevice(h->device));
    setBallKernel<<<1, 1, 0, h->stream>>>(h->dBall, h->dArena, arena, h->N, *in, h->P.goalBaseY + h->P.ballRadiusUu);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

rsb_status rsb_get_pads_at(rsb_handle* h, int32_t arena, rsb_pad_state* out) {
    if (!h || !out || arena < 0 || arena >= h->N) return fail(h, RSB_ERR_INVALID, "rsb_get_pads_at: no such arena");
    std::vector<uint32_t> w;
    rsb_status st = gatherRecords(h, h->dPad, arena, h->N, NUM_PADS, h->N * NUM_PADS, W_PAD, w);
    if (st) return st;
    for (int p = 0; p < NUM_PADS; p++) {
        PadP pp;
        loadPlanes(pp, w.data() + (size_t)p * W_PAD, 0, 1);
        out[p] = rsb_pad_state{};
        out[p].is_active = pp.bits & 1;
        out[p].cooldown = pp.cooldown;
        out[p].prev_locked_car_id = pp.bits >> 8;
    }
    return RSB_OK;
}

rsb_status rsb_set_pads_at(rsb_handle* h, int32_t arena, const rsb_pad_state* in) {
    if (!h || !in || arena < 0 || arena >= h->N) return fail(h, RSB_ERR_INVALID, "rsb_set_pads_at: no such arena");
    RSB_CUDA(cudaSetDevice(h->device));
    PadSet ps;
    std::memcpy(ps.p, in, sizeof ps.p);
    setPadsKernel<<<1, 64, 0, h->stream>>>(h->dPad, arena, h->N, ps);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

rsb_status rsb_get_arena_info_at(rsb_handle* h, int32_t arena, rsb_arena_info* out) {
    if (!h || !out || arena < 0 || arena >= h->N)
        return fail(h, RSB_ERR_INVALID, "rsb_get_arena_info_at: no such arena");
    std::vector<uint32_t> w;
    rsb_status st = gatherRecords(h, h->dArena, arena, 0, 1, h->N, W_ARENA, w);
    if (st) return st;
    ArenaP ap;
    loadPlanes(ap, w.data(), 0, 1);
    *out = arenaInfoOf(ap, h->teamSize[arena]);
    return RSB_OK;
}

rsb_status rsb_stats_get(rsb_handle* h, rsb_stats* out) {
    if (!h || !out) return RSB_ERR_INVALID;
    RSB_CUDA(cudaSetDevice(h->device));
    unsigned long long c[4] = {0, 0, 0, 0};
    RSB_CUDA(cudaMemcpyAsync(c, h->dCounters, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    std::vector<uint32_t> status;
    rsb_status st = download(h, h->dArena + (size_t)(offsetof(ArenaP, status) / 4) * h->N, status, h->N);
    if (st != RSB_OK) return st;
    *out = h->stats;
    out->narrowphase_queries = c[0];
    out->culled_queries = c[1];
    out->missed_contacts = c[2];
    out->solver_rows = c[3];
    uint64_t reverted = 0, bits = 0;
    for (uint32_t v : status) {
        bits |= v;
        if (v & WS_CULL_MISS) reverted++;
    }
    out->arenas_reverted = reverted;
    out->status_bits_seen = bits;
    return RSB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ learned culler
// (the rsb_culler_* definitions keep the C linkage of their declarations in rsb.h)

__global__ void logCentresKernel(const uint32_t* ball, const uint32_t* car, const int32_t* teamSize,
                                 const int32_t* carOffset, int N, float* log, int64_t base, int64_t cap) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    auto put = [&](int64_t i, float x, float y, float z) {
        if (i < cap) {
            log[3 * i] = x * kBtToUu;
            log[3 * i + 1] = y * kBtToUu;
            log[3 * i + 2] = z * kBtToUu;
        }
    };
    put(base + a, __uint_as_float(ball[a]), __uint_as_float(ball[(size_t)N + a]), __uint_as_float(ball[(size_t)2 * N + a]));
    for (int s = 0; s < 2 * teamSize[a]; s++)
        put(base + N + carOffset[a] + s, __uint_as_float(car[((size_t)0 * MAX_CARS + s) * N + a]),
            __uint_as_float(car[((size_t)1 * MAX_CARS + s) * N + a]),
            __uint_as_float(car[((size_t)2 * MAX_CARS + s) * N + a]));
}

constexpr int64_t kCullLogCap = 8 * 1024 * 1024;

static rsb_status ensureCuller(rsb_handle* h) {
    RSB_CUDA(cudaSetDevice(h->device));
    if (!h->dCw) {
        if (cudaMalloc((void**)&h->dCw, 4 * CM_NPARAM * sizeof(float)) != cudaSuccess ||
            cudaMalloc((void**)&h->dCwBf, CM_NPARAM * sizeof(__nv_bfloat16)) != cudaSuccess)
            return fail(h, RSB_ERR_NOMEM, "culler weight allocation failed");
        RSB_CUDA(cudaMemset(h->dCw, 0, 4 * CM_NPARAM * sizeof(float)));
        RSB_CUDA(cudaFuncSetAttribute(mlpTrainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TR_SMEM));
    }
    if (!h->dTris) {
        const ArenaStaticHost& H = *h->host;
        std::vector<float> t;
        t.reserve(H.triVerts.size() * 3);
        for (const V3& v : H.triVerts) {
            t.push_back(v.x * kBtToUu);
            t.push_back(v.y * kBtToUu);
            t.push_back(v.z * kBtToUu);
        }
        h->numTris = (int)(H.triVerts.size() / 3);
        if (cudaMalloc((void**)&h->dTris, t.size() * sizeof(float)) != cudaSuccess)
            return fail(h, RSB_ERR_NOMEM, "triangle allocation failed");
        RSB_CUDA(cudaMemcpy(h->dTris, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    return RSB_OK;
}

// Device buffer that frees itself.
template <class T>
struct DevBuf {
    T* p = nullptr;
    ~DevBuf() { cudaFree(p); }
    bool alloc(size_t n) { return cudaMalloc((void**)&p, std::max<size_t>(1, n) * sizeof(T)) == cudaSuccess; }
};

static rsb_status meshDistances(rsb_handle* h, const float* dPts, int64_t n, float* dOut) {
    for (int64_t i0 = 0; i0 < n; i0 += (1 << 22)) {
        const int cnt = (int)std::min<int64_t>(n - i0, 1 << 22);
        meshDistanceKernel<<<(cnt + 255) / 256, 256, 0, h->stream>>>(dPts + 3 * i0, cnt, h->dTris, h->numTris, dOut + i0);
        RSB_CUDA(cudaGetLastError());
    }
    return RSB_OK;
}

static rsb_status uploadWeights(rsb_handle* h, const float* w) {
    std::vector<__nv_bfloat16> bf(CM_NPARAM);
    for (int k = 0; k < CM_NPARAM; k++) bf[k] = __float2bfloat16_rn(w[k]);
    RSB_CUDA(cudaMemcpy(h->dCw, w, CM_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    RSB_CUDA(cudaMemcpy(h->dCwBf, bf.data(), CM_NPARAM * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    return RSB_OK;
}

rsb_status rsb_culler_log(rsb_handle* h, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    RSB_CUDA(cudaSetDevice(h->device));
    if (!h->dLog) {
        if (cudaMalloc((void**)&h->dLog, 3 * kCullLogCap * sizeof(float)) != cudaSuccess)
            return fail(h, RSB_ERR_NOMEM, "culler log allocation failed");
        h->logCap = kCullLogCap;
    }
    if (h->logCount >= h->logCap) return RSB_OK;
    logCentresKernel<<<(h->N + 127) / 128, 128, 0, pick(h, stream)>>>(h->dBall, h->dCar, h->dTeamSize, h->dCarOffset,
                                                                        h->N, h->dLog, h->logCount, h->logCap);
    RSB_CUDA(cudaGetLastError());
    h->logCount = std::min<int64_t>(h->logCap, h->logCount + h->N + h->numCars);
    return RSB_OK;
}

rsb_status rsb_culler_distance(rsb_handle* h, const float* pts, int32_t n, float* out) {
    if (!h || n < 0 || (n > 0 && (!pts || !out))) return fail(h, RSB_ERR_INVALID, "bad distance query");
    rsb_status st = ensureCuller(h);
    if (st != RSB_OK || n == 0) return st;
    DevBuf<float> dp, dd;
    if (!dp.alloc(3 * (size_t)n) || !dd.alloc(n)) return fail(h, RSB_ERR_NOMEM, "distance buffers");
    RSB_CUDA(cudaMemcpy(dp.p, pts, 12 * (size_t)n, cudaMemcpyHostToDevice));
    if ((st = meshDistances(h, dp.p, n, dd.p)) != RSB_OK) return st;
    RSB_CUDA(cudaMemcpyAsync(out, dd.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_culler_predict(rsb_handle* h, const float* pts, int32_t n, float* out) {
    if (!h || n < 0 || (n > 0 && (!pts || !out))) return fail(h, RSB_ERR_INVALID, "bad predict query");
    rsb_status st = ensureCuller(h);
    if (st != RSB_OK || n == 0) return st;
    DevBuf<float> dp, dd;
    if (!dp.alloc(3 * (size_t)n) || !dd.alloc(n)) return fail(h, RSB_ERR_NOMEM, "predict buffers");
    RSB_CUDA(cudaMemcpy(dp.p, pts, 12 * (size_t)n, cudaMemcpyHostToDevice));
    mlpPredictKernel<<<(n + 255) / 256, 256, 0, h->stream>>>(h->dCwBf, dp.p, n, dd.p);
    RSB_CUDA(cudaGetLastError());
    RSB_CUDA(cudaMemcpyAsync(out, dd.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_culler_gradients(rsb_handle* h, const float* pts, const float* target, int32_t n, float over_weight,
                                float* grad, float* loss) {
    if (!h || n <= 0 || !pts || !target || !grad) return fail(h, RSB_ERR_INVALID, "bad gradient query");
    rsb_status st = ensureCuller(h);
    if (st != RSB_OK) return st;
    DevBuf<float> dp, dt, dg, dl;
    if (!dp.alloc(3 * (size_t)n) || !dt.alloc(n) || !dg.alloc(CM_NPARAM) || !dl.alloc(1))
        return fail(h, RSB_ERR_NOMEM, "gradient buffers");
    RSB_CUDA(cudaMemcpy(dp.p, pts, 12 * (size_t)n, cudaMemcpyHostToDevice));
    RSB_CUDA(cudaMemcpy(dt.p, target, 4 * (size_t)n, cudaMemcpyHostToDevice));
    RSB_CUDA(cudaMemset(dg.p, 0, CM_NPARAM * sizeof(float)));
    RSB_CUDA(cudaMemset(dl.p, 0, sizeof(float)));
    mlpTrainKernel<<<(n + TR_TILE - 1) / TR_TILE, TR_TILE, TR_SMEM, h->stream>>>(h->dCwBf, dp.p, dt.p, n, 1.f / n,
                                                                                 over_weight, dg.p, dl.p);
    RSB_CUDA(cudaGetLastError());
    RSB_CUDA(cudaMemcpyAsync(grad, dg.p, CM_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    float l = 0.f;
    RSB_CUDA(cudaMemcpyAsync(&l, dl.p, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    if (loss) *loss = l;
    return RSB_OK;
}

rsb_status rsb_set_cull_mode(rsb_handle* h, int32_t mode) {
    if (!h || mode < RSB_CULL_EXACT || mode > RSB_CULL_VOXEL_AUDIT) return fail(h, RSB_ERR_INVALID, "unknown cull mode");
    h->cullMode = mode;
    return RSB_OK;
}

rsb_status rsb_culler_get(rsb_handle* h, float* params, float* margin) {
    if (!h) return RSB_ERR_INVALID;
    rsb_status st = ensureCuller(h);
    if (st != RSB_OK) return st;
    if (params) RSB_CUDA(cudaMemcpy(params, h->dCw, CM_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    if (margin) *margin = h->cullParams.margin;
    return RSB_OK;
}

rsb_status rsb_culler_set(rsb_handle* h, const float* params, float margin) {
    if (!h || !params || !(margin >= 0.f)) return fail(h, RSB_ERR_INVALID, "bad culler parameters");
    rsb_status st = ensureCuller(h);
    if (st != RSB_OK) return st;
    if ((st = uploadWeights(h, params)) != RSB_OK) return st;
    h->cullParams.margin = margin + h->cullSlack;
    h->cullerReady = true;
    return RSB_OK;
}

rsb_status rsb_culler_train(rsb_handle* h, const rsb_culler_config* cfg, rsb_culler_report* rep) {
    if (!h || !cfg || cfg->train_points <= 0 || cfg->heldout_points <= 0 || cfg->epochs <= 0 || cfg->batch <= 0)
        return fail(h, RSB_ERR_INVALID, "bad culler training configuration");
    rsb_status st = ensureCuller(h);
    if (st != RSB_OK) return st;
    cudaEvent_t t0, t1;
    RSB_CUDA(cudaEventCreate(&t0));
    RSB_CUDA(cudaEventCreate(&t1));
    RSB_CUDA(cudaEventRecord(t0, h->stream));
    std::mt19937_64 rng(cfg->seed);
    std::normal_distribution<float> gauss(0.f, 1.f);
    std::uniform_real_distribution<float> uni(0.f, 1.f);
    const int64_t total = (int64_t)cfg->train_points + cfg->heldout_points;

    // 1. logged centres and their distances (near-surface ones seed the jittered points)
    std::vector<float> logged(3 * (size_t)h->logCount), loggedD(h->logCount);
    if (h->logCount) {
        RSB_CUDA(cudaStreamSynchronize(h->stream));
        RSB_CUDA(cudaMemcpy(logged.data(), h->dLog, logged.size() * 4, cudaMemcpyDeviceToHost));
        DevBuf<float> dd;
        if (!dd.alloc(h->logCount)) return fail(h, RSB_ERR_NOMEM, "distance buffer");
        if ((st = meshDistances(h, h->dLog, h->logCount, dd.p)) != RSB_OK) return st;
        RSB_CUDA(cudaMemcpyAsync(loggedD.data(), dd.p, loggedD.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        RSB_CUDA(cudaStreamSynchronize(h->stream));
    }
    std::vector<int64_t> near;
    for (int64_t i = 0; i < h->logCount; i++)
        if (loggedD[i] < cfg->near_surface) near.push_back(i);

    // 2. the point set: logged centres, jittered near-surface centres, uniform points
    std::vector<float> pts(3 * (size_t)total);
    const float ux = ARENA_EXTENT_X + 200.f, uy = 6100.f, uz = ARENA_HEIGHT + 100.f;
    for (int64_t i = 0; i < total; i++) {
        float* p = &pts[3 * i];
        const float r = uni(rng);
        if (h->logCount && r < cfg->logged_fraction) {
            int64_t k = (int64_t)(uni(rng) * h->logCount) % h->logCount;
            p[0] = logged[3 * k]; p[1] = logged[3 * k + 1]; p[2] = logged[3 * k + 2];
        } else if (!near.empty() && r < cfg->logged_fraction + cfg->jitter_fraction) {
            int64_t k = near[(size_t)(uni(rng) * near.size()) % near.size()];
            for (int c = 0; c < 3; c++) p[c] = logged[3 * k + c] + cfg->jitter_sigma * gauss(rng);
        } else {
            p[0] = (2.f * uni(rng) - 1.f) * ux;
            p[1] = (2.f * uni(rng) - 1.f) * uy;
            p[2] = -100.f + uni(rng) * uz;
        }
    }
    DevBuf<float> dPts, dDist, dLoss, dPred;
    if (!dPts.alloc(pts.size()) || !dDist.alloc(total) || !dLoss.alloc(1) || !dPred.alloc(cfg->heldout_points))
        return fail(h, RSB_ERR_NOMEM, "training buffers");
    RSB_CUDA(cudaMemcpy(dPts.p, pts.data(), pts.size() * 4, cudaMemcpyHostToDevice));
    if ((st = meshDistances(h, dPts.p, total, dDist.p)) != RSB_OK) return st;
    std::vector<float> dist(total);
    RSB_CUDA(cudaMemcpyAsync(dist.data(), dDist.p, total * 4, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    // training targets are clamped: the bound only has to be tight where culling is decided
    std::vector<float> target(dist);
    for (float& d : target) d = std::min(d, cfg->target_cap);
    DevBuf<float> dTarget;
    if (!dTarget.alloc(total)) return fail(h, RSB_ERR_NOMEM, "target buffer");
    RSB_CUDA(cudaMemcpy(dTarget.p, target.data(), total * 4, cudaMemcpyHostToDevice));

    // 3. initial weights (He-uniform), Adam state cleared
    std::vector<float> w(CM_NPARAM, 0.f);
    auto fill = [&](int off, int cnt, int fanIn) {
        const float b = std::sqrt(6.f / fanIn);
        for (int k = 0; k < cnt; k++) w[off + k] = (2.f * uni(rng) - 1.f) * b;
    };
    fill(CP_W1, 3 * CM_H, 3);
    fill(CP_W2, CM_H * CM_H, CM_H);
    fill(CP_W3, CM_H, CM_H);
    for (int k = 0; k < CM_H; k++) w[CP_B1 + k] = 0.01f;
    if ((st = uploadWeights(h, w.data())) != RSB_OK) return st;
    RSB_CUDA(cudaMemset(h->dCw + CM_NPARAM, 0, 3 * CM_NPARAM * sizeof(float)));
    float* dM = h->dCw + CM_NPARAM;
    float* dV = dM + CM_NPARAM;
    float* dG = dV + CM_NPARAM;

    // 4. Adam over shuffled mini-batches of the training part (points are already random)
    const int64_t ntrain = cfg->train_points;
    const int bsz = cfg->batch;
    int steps = 0;
    float lastLoss = 0.f;
    const float b1 = 0.9f, b2 = 0.999f;
    const int stepsPerEpoch = (int)((ntrain + bsz - 1) / bsz);
    const int totalSteps = stepsPerEpoch * cfg->epochs;
    for (int ep = 0; ep < cfg->epochs; ep++) {
        RSB_CUDA(cudaMemsetAsync(dLoss.p, 0, sizeof(float), h->stream));
        const int64_t shift = (int64_t)(uni(rng) * bsz);  // vary the batch boundaries per epoch
        for (int64_t b0 = 0; b0 < ntrain; b0 += bsz) {
            const int64_t start = (b0 + shift) % ntrain;
            const int cnt = (int)std::min<int64_t>(bsz, ntrain - start);
            mlpTrainKernel<<<(cnt + TR_TILE - 1) / TR_TILE, TR_TILE, TR_SMEM, h->stream>>>(
                h->dCwBf, dPts.p + 3 * start, dTarget.p + start, cnt, 1.f / cnt, cfg->over_weight, dG,
                dLoss.p);
            steps++;
            // cosine decay of the learning rate
            const float lr = cfg->lr * 0.5f * (1.f + std::cos(3.14159265f * (float)steps / (float)totalSteps));
            const float c1 = 1.f - std::pow(b1, (float)steps), c2 = 1.f - std::pow(b2, (float)steps);
            adamKernel<<<(CM_NPARAM + 255) / 256, 256, 0, h->stream>>>(h->dCw, dM, dV, dG, h->dCwBf, lr, b1, b2, c1,
                                                                      c2, 1e-8f);
        }
        RSB_CUDA(cudaGetLastError());
        RSB_CUDA(cudaMemcpyAsync(&lastLoss, dLoss.p, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        RSB_CUDA(cudaStreamSynchronize(h->stream));
        lastLoss /= (float)stepsPerEpoch;
    }

    // 5. margin: the largest over-estimate on the held-out points, so that the bound
    // holds on every one of them
    const int nh = cfg->heldout_points;
    mlpPredictKernel<<<(nh + 255) / 256, 256, 0, h->stream>>>(h->dCwBf, dPts.p + 3 * ntrain, nh, dPred.p);
    RSB_CUDA(cudaGetLastError());
    std::vector<float> pred(nh);
    RSB_CUDA(cudaMemcpyAsync(pred.data(), dPred.p, nh * 4, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaEventRecord(t1, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    double mae = 0.0;
    float maxOver = 0.f;
    for (int i = 0; i < nh; i++) {
        const float d = dist[ntrain + i];
        mae += std::fabs(std::min(pred[i], cfg->target_cap) - std::min(d, cfg->target_cap));
        maxOver = std::max(maxOver, pred[i] - d);
    }
    const float margin = maxOver + cfg->margin_slack;
    int misses = 0, clear = 0;
    const float carNeed = h->cullParams.carReach + h->cullParams.carVmax * 8 * h->P.dt;
    for (int i = 0; i < nh; i++) {
        const float b = pred[i] - margin;
        if (b > dist[ntrain + i]) misses++;
        if (b >= carNeed) clear++;
    }
    h->cullParams.margin = margin + h->cullSlack;
    h->cullerReady = true;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rep) {
        *rep = rsb_culler_report{};
        rep->train_points = cfg->train_points;
        rep->heldout_points = nh;
        rep->logged_points = (int32_t)h->logCount;
        rep->epochs = cfg->epochs;
        rep->steps = steps;
        rep->final_loss = lastLoss;
        rep->margin = margin;
        rep->heldout_mae = (float)(mae / nh);
        rep->heldout_max_over = maxOver;
        rep->heldout_misses = misses;
        rep->heldout_car_clear = (float)clear / nh;
        rep->train_ms = ms;
    }
    return RSB_OK;
}

// ------------------------------------------------------------------ state ring

extern "C" {

rsb_status rsb_ring_default_config(rsb_ring_config* out) {
    if (!out) return RSB_ERR_INVALID;
    out->depth = 10;
    out->capture_every = 3;
    out->restore_fraction = 0.05f;
    out->max_arenas_per_restore = 64;
    out->fuzz_pos = 25.f;
    out->fuzz_vel = 80.f;
    out->lookback_slots = 7;
    out->seed = 0xA5A5A5A5u;
    return RSB_OK;
}

rsb_status rsb_ring_configure(rsb_handle* h, const rsb_ring_config* cfg) {
    if (!h || !cfg) return fail(h, RSB_ERR_INVALID, "rsb_ring_configure: null argument");
    RSB_CUDA(cudaSetDevice(h->device));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    auto& R = h->ring;
    cudaFree(R.dSlots);
    R.dSlots = nullptr;
    R.enabled = false;
    R.filled = R.writeIdx = R.stepsSinceCapture = 0;
    if (cfg->depth <= 0 || h->N <= 0) return RSB_OK;
    R.cfg = *cfg;
    R.cfg.depth = std::max(2, cfg->depth);
    R.cfg.capture_every = std::max(1, cfg->capture_every);
    R.cfg.lookback_slots = std::max(1, std::min(cfg->lookback_slots, R.cfg.depth - 1));
    R.cfg.restore_fraction =
        std::max(0.01f, std::min(0.05f, cfg->restore_fraction > 0.f ? cfg->restore_fraction : 0.05f));
    R.cfg.max_arenas_per_restore = std::max(1, cfg->max_arenas_per_restore > 0 ? cfg->max_arenas_per_restore : 64);
    R.rng = cfg->seed ? cfg->seed : 0xA5A5A5A5u;
    R.slotWords = (size_t)W_BALL * h->N + (size_t)W_CAR * MAX_CARS * h->N + (size_t)W_PAD * NUM_PADS * h->N;
    const size_t bytes = (size_t)R.cfg.depth * R.slotWords * sizeof(uint32_t);
    if (cudaMalloc(&R.dSlots, bytes) != cudaSuccess) {
        R.dSlots = nullptr;
        cudaGetLastError();
        return fail(h, RSB_ERR_NOMEM, "rsb_ring_configure: cannot allocate " + std::to_string(bytes) + " bytes of slots");
    }
    R.enabled = true;
    return RSB_OK;
}

rsb_status rsb_ring_capture(rsb_handle* h, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    auto& R = h->ring;
    if (!R.enabled) return RSB_OK;
    RSB_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    uint32_t* slot = R.dSlots + (size_t)R.writeIdx * R.slotWords;
    const size_t nb = (size_t)W_BALL * h->N, nc = (size_t)W_CAR * MAX_CARS * h->N, np = (size_t)W_PAD * NUM_PADS * h->N;
    RSB_CUDA(cudaMemcpyAsync(slot, h->dBall, nb * 4, cudaMemcpyDeviceToDevice, st));
    RSB_CUDA(cudaMemcpyAsync(slot + nb, h->dCar, nc * 4, cudaMemcpyDeviceToDevice, st));
    RSB_CUDA(cudaMemcpyAsync(slot + nb + nc, h->dPad, np * 4, cudaMemcpyDeviceToDevice, st));
    R.writeIdx = (R.writeIdx + 1) % R.cfg.depth;
    if (R.filled < R.cfg.depth) R.filled++;
    R.captures++;
    return RSB_OK;
}

rsb_status rsb_ring_maybe_capture(rsb_handle* h, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    auto& R = h->ring;
    if (!R.enabled) return RSB_OK;
    if (++R.stepsSinceCapture < R.cfg.capture_every) return RSB_OK;
    R.stepsSinceCapture = 0;
    return rsb_ring_capture(h, stream);
}

rsb_status rsb_ring_restore(rsb_handle* h, float restore_fraction, int32_t lookback_slots, float fuzz_scale,
                            int32_t max_arenas, int32_t* restored, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    if (restored) *restored = 0;
    auto& R = h->ring;
    if (!R.enabled || R.replayDisabled || R.filled < 2) return RSB_OK;
    const int N = h->N;
    float frac = restore_fraction >= 0.f ? restore_fraction : R.cfg.restore_fraction;
    frac = std::max(0.01f, std::min(0.05f, frac));
    int lookback = lookback_slots >= 0 ? lookback_slots : R.cfg.lookback_slots;
    lookback = std::max(1, std::min(lookback, R.filled - 1));
    int lastWritten = R.writeIdx - 1;
    if (lastWritten < 0) lastWritten = R.cfg.depth - 1;
    int slot = lastWritten - lookback;
    while (slot < 0) slot += R.cfg.depth;
    int cap = max_arenas > 0 ? max_arenas : R.cfg.max_arenas_per_restore;
    if (cap <= 0) cap = 64;
    const int fivePct = std::max(1, (int)std::lround(0.05 * (double)N));
    cap = std::min(cap, fivePct);
    int nRestore = std::max(1, (int)std::lround(frac * (double)N));
    nRestore = std::min(nRestore, N);
    nRestore = std::min(nRestore, cap);
    // partial Fisher-Yates over the arena indices, then each arena's jitter draws in order
    std::vector<int> order((size_t)N);
    for (int i = 0; i < N; i++) order[(size_t)i] = i;
    for (int i = 0; i < nRestore; i++) {
        int j = i + (int)(ringRand01(R.rng) * (N - i));
        if (j >= N) j = N - 1;
        std::swap(order[(size_t)i], order[(size_t)j]);
    }
    const float fp = R.cfg.fuzz_pos * fuzz_scale;
    const float fv = R.cfg.fuzz_vel * fuzz_scale;
    const int drawsPerBody = (fp > 0.f ? 3 : 0) + (fv > 0.f ? 3 : 0);
    R.jobs.resize(2 * (size_t)nRestore);
    for (int i = 0; i < nRestore; i++) {
        const int a = order[(size_t)i];
        R.jobs[2 * (size_t)i] = (uint32_t)a;
        R.jobs[2 * (size_t)i + 1] = R.rng;
        const int draws = (2 * h->teamSize[(size_t)a] + 1) * drawsPerBody;
        for (int k = 0; k < draws; k++) ringRand01(R.rng);
    }
    RSB_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    if (R.jobCap < nRestore) {
        if (R.dJobs) {
            RSB_CUDA(cudaStreamSynchronize(st));
            cudaFree(R.dJobs);
            R.dJobs = nullptr;
        }
        R.jobCap = 0;
        const int capJobs = std::max(nRestore, 64);
        RSB_CUDA(cudaMalloc(&R.dJobs, 2 * sizeof(uint32_t) * (size_t)capJobs));
        R.jobCap = capJobs;
    }
    RSB_CUDA(cudaMemcpyAsync(R.dJobs, R.jobs.data(), R.jobs.size() * 4, cudaMemcpyHostToDevice, st));
    const uint32_t* sBall = R.dSlots + (size_t)slot * R.slotWords;
    const uint32_t* sCar = sBall + (size_t)W_BALL * N;
    const uint32_t* sPad = sCar + (size_t)W_CAR * MAX_CARS * N;
    ringRestoreKernel<<<(nRestore + 63) / 64, 64, 0, st>>>(h->dBall, h->dCar, h->dPad, h->dArena, h->dTeamSize, sBall,
                                                            sCar, sPad, R.dJobs, nRestore, N, fp, fv,
                                                            h->P.goalBaseY + h->P.ballRadiusUu);
    RSB_CUDA(cudaGetLastError());
    R.restores += (uint64_t)nRestore;
    R.restoreCalls++;
    // the reference's tripwire: far more restores than captures turns replay off
    if (R.restoreCalls > 32 && R.captures > 0 && R.restoreCalls > R.captures * 4) R.replayDisabled = true;
    if (restored) *restored = nRestore;
    return RSB_OK;
}

rsb_status rsb_ring_stats_get(rsb_handle* h, rsb_ring_stats* out) {
    if (!h || !out) return RSB_ERR_INVALID;
    const auto& R = h->ring;
    out->depth = R.enabled ? R.cfg.depth : 0;
    out->filled = R.filled;
    out->write_idx = R.writeIdx;
    out->replay_disabled = R.replayDisabled ? 1 : 0;
    out->captures = R.captures;
    out->restores = R.restores;
    out->restore_calls = R.restoreCalls;
    return RSB_OK;
}

}  // extern "C"

namespace rsb {
// Message of a failed call that has no handle (rsb_last_error with h == NULL returns it).
void setGlobalError(const std::string& msg) { g_createError = msg; }
}  // namespace rsb

extern "C" {

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
        case RSB_BUF_BALL_PRED: *out = h->dPred; return RSB_OK;
        case RSB_BUF_VANTA_OBS: *out = h->dVantaRows; return RSB_OK;
        default: return fail(h, RSB_ERR_INVALID, "unknown buffer");
    }
}

rsb_status rsb_reset_arenas(rsb_handle* h, const int32_t* idx, int32_t n, uint64_t seed, int32_t mode) {
    if (!h || n < 0 || (n > 0 && !idx) || n > h->N) return fail(h, RSB_ERR_INVALID, "bad reset arena list");
    if (mode < RSB_RESET_KICKOFF || mode > RSB_RESET_CURRICULUM) return fail(h, RSB_ERR_INVALID, "unknown reset mode");
    for (int i = 0; i < n; i++)
        if (idx[i] < 0 || idx[i] >= h->N) return fail(h, RSB_ERR_INVALID, "arena index out of range");
    if (n == 0) return RSB_OK;
    RSB_CUDA(cudaSetDevice(h->device));
    RSB_CUDA(cudaMemcpyAsync(h->dResetIdx, idx, 4 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
    resetKernel<<<(n + 127) / 128, 128, 0, h->stream>>>(envView(h), h->tables, h->curriculum, h->dResetIdx, n, seed,
                                                         mode, false);
    RSB_CUDA(cudaGetLastError());
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_reset_all(rsb_handle* h, uint64_t seed, int32_t mode) {
    if (!h) return RSB_ERR_INVALID;
    if (mode < RSB_RESET_KICKOFF || mode > RSB_RESET_CURRICULUM) return fail(h, RSB_ERR_INVALID, "unknown reset mode");
    RSB_CUDA(cudaSetDevice(h->device));
    resetKernel<<<(h->N + 127) / 128, 128, 0, h->stream>>>(envView(h), h->tables, h->curriculum, nullptr, h->N, seed,
                                                            mode, false);
    RSB_CUDA(cudaGetLastError());
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_reset_done(rsb_handle* h, uint64_t seed, int32_t mode, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    if (mode < RSB_RESET_KICKOFF || mode > RSB_RESET_CURRICULUM) return fail(h, RSB_ERR_INVALID, "unknown reset mode");
    RSB_CUDA(cudaSetDevice(h->device));
    resetKernel<<<(h->N + 127) / 128, 128, 0, pick(h, stream)>>>(envView(h), h->tables, h->curriculum, nullptr, h->N,
                                                                  seed, mode, true);
    RSB_CUDA(cudaGetLastError());
    return RSB_OK;
}

static rsb_status copyOut(rsb_handle* h, void* out, const void* dev, size_t count, size_t expect, size_t elem,
                          const char* what);

rsb_status rsb_vanta_default_config(rsb_vanta_config* cfg) {
    if (!cfg) return RSB_ERR_INVALID;
    *cfg = rsb_vanta_config{};
    cfg->tick_skip = 8;
    cfg->dodge_deadzone = 0.5f;
    cfg->only_closest_opp = 0;
    cfg->predict_ball = 1;
    return RSB_OK;
}

rsb_status rsb_vanta_configure(rsb_handle* h, const rsb_vanta_config* cfg) {
    if (!h || !cfg || cfg->tick_skip <= 0 || !(cfg->dodge_deadzone >= 0.f))
        return fail(h, RSB_ERR_INVALID, "bad VantaObs configuration");
    RSB_CUDA(cudaSetDevice(h->device));
    const size_t N = h->N;
    if (!h->dVA) {
        if (cudaMalloc((void**)&h->dVA, (size_t)VA_WORDS * N * 4) != cudaSuccess ||
            cudaMalloc((void**)&h->dVT, (size_t)VT_WORDS * MAX_CARS * N * 4) != cudaSuccess ||
            cudaMalloc((void**)&h->dVantaPred, N * 3 * sizeof(rsb_ball_state)) != cudaSuccess ||
            cudaMalloc((void**)&h->dVantaRows, std::max<size_t>(1, h->numCars) * VANTA_ROW * 4) != cudaSuccess) {
            cudaFree(h->dVA); cudaFree(h->dVT); cudaFree(h->dVantaPred); cudaFree(h->dVantaRows);
            h->dVA = h->dVT = nullptr;
            h->dVantaPred = nullptr;
            h->dVantaRows = nullptr;
            return fail(h, RSB_ERR_NOMEM, "VantaObs state allocation failed");
        }
    }
    // a (re)configured builder starts from its default state, as after a reset
    RSB_CUDA(cudaMemsetAsync(h->dVA, 0, (size_t)VA_WORDS * N * 4, h->stream));
    RSB_CUDA(cudaMemsetAsync(h->dVT, 0, (size_t)VT_WORDS * MAX_CARS * N * 4, h->stream));
    RSB_CUDA(cudaMemsetAsync(h->dVantaRows, 0, std::max<size_t>(1, h->numCars) * VANTA_ROW * 4, h->stream));
    // pad tables in RLGym order (the AdvancedObs pad map), z of the pad table, and the
    // x-mirror permutation: the first pad at (-x, y, z) within 1 uu (RocketSimCudaHostUtils.cuh:66-86)
    VantaTables& T = h->vantaTables;
    for (int i = 0; i < NUM_PADS; i++) {
        const PadLoc& l = PAD_LOCS_HOST[h->tables.padMap[i]];
        T.x[i] = l.x;
        T.y[i] = l.y;
        T.z[i] = l.z;
        T.pad[i] = (uint8_t)h->tables.padMap[i];
    }
    for (int i = 0; i < NUM_PADS; i++) {
        int m = i;
        for (int j = 0; j < NUM_PADS; j++)
            if (std::fabs(T.x[j] + T.x[i]) < 1.f && std::fabs(T.y[j] - T.y[i]) < 1.f && std::fabs(T.z[j] - T.z[i]) < 1.f) {
                m = j;
                break;
            }
        T.mirror[i] = (uint8_t)m;
    }
    h->vanta = *cfg;
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_build_vanta_obs(rsb_handle* h, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    if (!h->dVA) return fail(h, RSB_ERR_STATE, "VantaObs is not configured (rsb_vanta_configure)");
    RSB_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = pick(h, stream);
    VantaView V{};
    V.arena = h->dVA;
    V.car = h->dVT;
    V.rows = h->dVantaRows;
    V.dt = (float)h->vanta.tick_skip / 120.f;
    V.deadzone = h->vanta.dodge_deadzone;
    V.onlyClosestOpp = h->vanta.only_closest_opp;
    if (h->vanta.predict_ball) {
        // the ball-only rollout of BallPredTracker, slices at 1, 2 and 3 s
        PredSlices ps{};
        ps.n = 3;
        ps.t[0] = 120;
        ps.t[1] = 240;
        ps.t[2] = 360;
        predictBallKernel<<<(h->N + 127) / 128, 128, 0, st>>>(devView(h), ps, h->dVantaPred);
        RSB_CUDA(cudaGetLastError());
        V.pred = h->dVantaPred;
    }
    const EnvView E = envView(h);
    vantaArenaKernel<<<(h->N + 127) / 128, 128, 0, st>>>(E, V, h->vantaTables);
    RSB_CUDA(cudaGetLastError());
    if (h->numCars > 0) {
        vantaRowKernel<<<(h->numCars + VANTA_THREADS - 1) / VANTA_THREADS, VANTA_THREADS, 0, st>>>(
            E, V, h->vantaTables, h->numCars);
        RSB_CUDA(cudaGetLastError());
    }
    return RSB_OK;
}

rsb_status rsb_copy_vanta_obs(rsb_handle* h, float* out, size_t n) {
    if (h && !h->dVantaRows) return fail(h, RSB_ERR_STATE, "VantaObs is not configured (rsb_vanta_configure)");
    return copyOut(h, out, h ? h->dVantaRows : nullptr, n, h ? (size_t)h->numCars * VANTA_ROW : 0, 4, "vanta obs");
}

rsb_status rsb_pad_locations(float* xyz) {
    if (!xyz) return RSB_ERR_INVALID;
    for (int p = 0; p < NUM_PADS; p++) {
        xyz[3 * p + 0] = PAD_LOCS_HOST[p].x;
        xyz[3 * p + 1] = PAD_LOCS_HOST[p].y;
        xyz[3 * p + 2] = PAD_LOCS_HOST[p].z;
    }
    return RSB_OK;
}

rsb_status rsb_env_graph_capture(rsb_handle* h, const int32_t* d_actions, int32_t tick_skip, int32_t reset_mode,
                                 uint64_t seed) {
    if (!h || !d_actions || tick_skip <= 0) return fail(h, RSB_ERR_INVALID, "bad graph capture arguments");
    if (reset_mode < RSB_RESET_KICKOFF || reset_mode > RSB_RESET_CURRICULUM)
        return fail(h, RSB_ERR_INVALID, "unknown reset mode");
    if (!h->dLut) return fail(h, RSB_ERR_STATE, "no action table uploaded");
    if (!h->hasRewards) return fail(h, RSB_ERR_STATE, "no reward configuration at create");
    RSB_CUDA(cudaSetDevice(h->device));
    if (h->envGraph) {
        cudaGraphExecDestroy(h->envGraph);
        h->envGraph = nullptr;
    }
    if (!h->dGraphSeed && cudaMalloc((void**)&h->dGraphSeed, sizeof(uint64_t)) != cudaSuccess)
        return fail(h, RSB_ERR_NOMEM, "graph seed allocation failed");
    RSB_CUDA(cudaMemcpy(h->dGraphSeed, &seed, sizeof seed, cudaMemcpyHostToDevice));
    const uint64_t ticksBefore = h->stats.ticks_simulated;
    RSB_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    rsb_status st = rsb_set_actions_device(h, d_actions, h->numCars, h->stream);
    if (st == RSB_OK) st = rsb_step(h, tick_skip, h->stream);
    if (st == RSB_OK) st = rsb_build_obs(h, h->stream);
    if (st == RSB_OK) st = rsb_build_rewards_terminals(h, tick_skip, h->stream);
    if (st == RSB_OK) {
        resetKernel<<<(h->N + 127) / 128, 128, 0, h->stream>>>(envView(h), h->tables, h->curriculum, nullptr, h->N,
                                                               0, reset_mode, true, h->dGraphSeed);
        advanceSeedKernel<<<1, 1, 0, h->stream>>>(h->dGraphSeed);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->stats.ticks_simulated = ticksBefore;
    if (st != RSB_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cudaFail(h, "cudaStreamEndCapture", e);
    const cudaError_t ie = cudaGraphInstantiate(&h->envGraph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        h->envGraph = nullptr;
        return cudaFail(h, "cudaGraphInstantiate", ie);
    }
    h->graphTicks = tick_skip;
    return RSB_OK;
}

rsb_status rsb_env_graph_launch(rsb_handle* h, void* stream) {
    if (!h) return RSB_ERR_INVALID;
    if (!h->envGraph) return fail(h, RSB_ERR_STATE, "no env step captured");
    RSB_CUDA(cudaSetDevice(h->device));
    RSB_CUDA(cudaGraphLaunch(h->envGraph, pick(h, stream)));
    h->stats.ticks_simulated += (uint64_t)h->N * h->graphTicks;
    return RSB_OK;
}

rsb_status rsb_set_reset_curriculum(rsb_handle* h, float kickoff_w, float fuzzed_w, float aerial_w, float chase_w) {
    if (!h) return RSB_ERR_INVALID;
    auto clampW = [](float w) { return (w >= 0.f && w <= 1e6f) ? w : 0.f; };
    float* w = h->curriculum.w;
    w[0] = clampW(kickoff_w);
    w[1] = clampW(fuzzed_w);
    w[2] = clampW(aerial_w);
    w[3] = clampW(chase_w);
    if (w[0] + w[1] + w[2] + w[3] <= 0.f) w[0] = 1.f;
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
    obsKernel<<<(h->N + OBS_ARENAS - 1) / OBS_ARENAS, OBS_THREADS, 0, pick(h, stream)>>>(envView(h), h->tables);
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

rsb_status rsb_copy_outputs(rsb_handle* h, float* obs, uint8_t* masks, float* rewards, uint8_t* terminals) {
    if (!h) return RSB_ERR_INVALID;
    RSB_CUDA(cudaSetDevice(h->device));
    if (obs)
        RSB_CUDA(cudaMemcpyAsync(obs, h->dObs, (size_t)h->numCars * h->obsStride * 4, cudaMemcpyDeviceToHost,
                                 h->stream));
    if (masks)
        RSB_CUDA(cudaMemcpyAsync(masks, h->dMasks, (size_t)h->numCars * RSB_NUM_ACTIONS, cudaMemcpyDeviceToHost,
                                 h->stream));
    if (rewards)
        RSB_CUDA(cudaMemcpyAsync(rewards, h->dRewards, (size_t)h->numCars * 4, cudaMemcpyDeviceToHost, h->stream));
    if (terminals)
        RSB_CUDA(cudaMemcpyAsync(terminals, h->dTerminals, (size_t)h->N, cudaMemcpyDeviceToHost, h->stream));
    RSB_CUDA(cudaStreamSynchronize(h->stream));
    return RSB_OK;
}

rsb_status rsb_host_register(void* ptr, size_t bytes) {
    if (!ptr || bytes == 0) return RSB_ERR_INVALID;
    const cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        g_createError = std::string("rsb_host_register: ") + cudaGetErrorString(e);
        return RSB_ERR_CUDA;
    }
    return RSB_OK;
}

rsb_status rsb_host_unregister(void* ptr) {
    if (!ptr) return RSB_ERR_INVALID;
    const cudaError_t e = cudaHostUnregister(ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        g_createError = std::string("rsb_host_unregister: ") + cudaGetErrorString(e);
        return RSB_ERR_CUDA;
    }
    return RSB_OK;
}

}  // extern "C"
