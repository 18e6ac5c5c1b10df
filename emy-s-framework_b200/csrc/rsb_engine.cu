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
#include "phys/engine_core.h"

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

using EngineDev = EngineView;

}  // namespace

struct rsb_handle {
    int device = 0;
    int N = 0;
    int numCars = 0;
    int maxCars = 0;
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

__global__ void __launch_bounds__(128) stepKernel(EngineDev D, int ticks) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= D.N) return;
    ArenaSim A;
    stepArena(D, a, ticks, A);
}

__global__ void expandActionsKernel(const int32_t* idx, const rsb_controls* lut, int lutCount, rsb_controls* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = idx[i];
    k = k < 0 ? 0 : (k >= lutCount ? lutCount - 1 : k);
    out[i] = lut[k];
}

// ------------------------------------------------------------------ host helpers

static void computeParams(const rsb_mutators& m, WorldParams& P) {
    P = WorldParams{};
    P.dt = 1.f / 120.f;
    P.gravity = V3{m.gravity.x, m.gravity.y, m.gravity.z} * kUuToBt;
    P.ballRadius = m.ball_radius * kUuToBt;
    P.ballMargin = P.ballRadius;
    P.ballAabbExt = P.ballMargin + 0.08f;
    // btCollisionShape::getBoundingSphere adds 0.08 (a double literal) to the sphere radius
    P.ballCbt = (float)((double)P.ballRadius + 0.08) * 0.02f;
    P.ballInvMass = 1.f / m.ball_mass;
    P.ballGrav = P.gravity * (1.f / P.ballInvMass);
    float inert = 0.4f * m.ball_mass * P.ballMargin * P.ballMargin;
    P.ballInvInertia = V3{1.f / inert, 1.f / inert, 1.f / inert};
    float drag = m.ball_drag < 0.f ? 0.f : (m.ball_drag > 1.f ? 1.f : m.ball_drag);
    P.ballLinDampFactor = powf(1.f - drag, P.dt);
    P.ballFriction = m.ball_world_friction;
    P.ballRestitution = m.ball_world_restitution;
    P.ballMaxSpeedBt = m.ball_max_speed * kUuToBt;
    P.goalBaseY = m.goal_base_threshold_y;
    P.ballRadiusUu = m.ball_radius;
}

static void initialCell(const ArenaStatic& S, V3 mn, int32_t& cell, int32_t& ci, int32_t& cj, int32_t& ck) {
    int i, j, k;
    bpCellIndices(S.bp, mn, i, j, k);
    ci = i; cj = j; ck = k;
    cell = i * S.bp.cellsY * S.bp.cellsZ + j * S.bp.cellsZ + k;
}

static M3 basisFromRot(const rsb_rotmat& r) {
    // RocketSim RotMat is column-major (forward, right, up are the basis columns)
    return m3(r.forward.x, r.right.x, r.up.x, r.forward.y, r.right.y, r.up.y, r.forward.z, r.right.z, r.up.z);
}
static rsb_rotmat rotFromBasis(const float* rot) {
    rsb_rotmat r;
    r.forward = rsb_vec3{rot[0], rot[3], rot[6]};
    r.right = rsb_vec3{rot[1], rot[4], rot[7]};
    r.up = rsb_vec3{rot[2], rot[5], rot[8]};
    return r;
}

template <class T>
static void planesToHost(const std::vector<uint32_t>& planes, int stride, int idx, T& rec) {
    loadPlanes(rec, planes.data(), idx, stride);
}
template <class T>
static void hostToPlanes(std::vector<uint32_t>& planes, int stride, int idx, const T& rec) {
    storePlanes(rec, planes.data(), idx, stride);
}

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

static EngineDev devView(rsb_handle* h) {
    EngineDev D;
    D.S = h->stat->view;
    D.P = h->P;
    D.N = h->N;
    D.teamSize = h->dTeamSize;
    D.carOffset = h->dCarOffset;
    D.ball = h->dBall;
    D.car = h->dCar;
    D.pad = h->dPad;
    D.arena = h->dArena;
    D.controls = h->dControls;
    return D;
}

static cudaStream_t pick(rsb_handle* h, void* s) { return s ? (cudaStream_t)s : h->stream; }

// ------------------------------------------------------------------ C ABI

extern "C" {

rsb_status rsb_default_mutators(rsb_mutators* m) {
    if (!m) return RSB_ERR_INVALID;
    *m = rsb_mutators{};
    m->gravity = rsb_vec3{0, 0, GRAVITY_Z};
    m->car_mass = CAR_MASS_BT;
    m->car_world_friction = CARWORLD_COLLISION_FRICTION;
    m->car_world_restitution = CARWORLD_COLLISION_RESTITUTION;
    m->ball_mass = BALL_MASS_BT;
    m->ball_max_speed = BALL_MAX_SPEED;
    m->ball_drag = BALL_DRAG;
    m->ball_world_friction = BALL_FRICTION;
    m->ball_world_restitution = BALL_RESTITUTION;
    m->jump_accel = JUMP_ACCEL;
    m->jump_immediate_force = JUMP_IMMEDIATE_FORCE;
    m->boost_accel_ground = BOOST_ACCEL_GROUND;
    m->boost_accel_air = BOOST_ACCEL_AIR;
    m->boost_used_per_second = BOOST_USED_PER_SECOND;
    m->respawn_delay = DEMO_RESPAWN_TIME;
    m->bump_cooldown_time = BUMP_COOLDOWN_TIME;
    m->boost_pad_cooldown_big = PAD_COOLDOWN_BIG;
    m->boost_pad_cooldown_small = PAD_COOLDOWN_SMALL;
    m->car_spawn_boost_amount = BOOST_SPAWN_AMOUNT;
    m->ball_hit_extra_force_scale = 1.f;
    m->bump_force_scale = 1.f;
    m->ball_radius = BALL_COLLISION_RADIUS_SOCCAR;
    m->goal_base_threshold_y = SOCCAR_GOAL_SCORE_BASE_THRESHOLD_Y;
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
    h->carOffset.push_back(0);
    for (int a = 0; a < h->N; a++) {
        int ts = cfg->team_sizes ? cfg->team_sizes[a] : cfg->team_size;
        if (ts < 0 || ts > RSB_MAX_TEAM_SIZE) return fail(nullptr, RSB_ERR_INVALID, "team size must be 0..3");
        if (ts > 0) return fail(nullptr, RSB_ERR_UNSUPPORTED, "cars are not built into this library yet");
        h->teamSize.push_back(ts);
        h->carOffset.push_back(h->carOffset.back() + 2 * ts);
        h->maxCars = std::max(h->maxCars, 2 * ts);
    }
    h->numCars = h->carOffset.back();
    if (cfg->mutators) h->mut = *cfg->mutators;
    else rsb_default_mutators(&h->mut);
    computeParams(h->mut, h->P);

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
        // per-thread stack limit cover its frame (the default limit is 1 KB)
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, stepKernel) != cudaSuccess)
            return fail(nullptr, RSB_ERR_CUDA, "cudaFuncGetAttributes failed");
        size_t need = ((fa.localSizeBytes + 4096) + 1023) / 1024 * 1024, cur = 0;
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
        !dalloc(h->dActions, std::max<size_t>(1, h->numCars) * 4))
        return fail(nullptr, RSB_ERR_NOMEM, "device allocation failed");
    cudaMemcpy(h->dTeamSize, h->teamSize.data(), N * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(h->dCarOffset, h->carOffset.data(), (N + 1) * 4, cudaMemcpyHostToDevice);

    // initial state: RocketSim's Arena constructor (ball at rest at its kickoff height,
    // active pads) with the broadphase cells of the creation transforms
    {
        const ArenaStatic& S = h->stat->view;
        std::vector<uint32_t> ball((size_t)W_BALL * N), arena((size_t)W_ARENA * N), pads((size_t)W_PAD * NUM_PADS * N);
        BallP bp{};
        Xf x{m3identity(), V3{0, 0, BALL_REST_Z} * kUuToBt};
        xfToP(x, bp.pos, bp.rot);
        V3 mn, mx;
        Xf x0{m3identity(), V3{0, 0, h->P.ballRadius}};
        ballAabb(h->P, x0, mn, mx);
        initialCell(S, mn, bp.cell, bp.ci, bp.cj, bp.ck);
        bp.regStamp = 0;
        ArenaP ap{};
        ap.goalTeam = -1;
        PadP pp{};
        pp.bits = 1;
        for (size_t a = 0; a < N; a++) {
            hostToPlanes(ball, (int)N, (int)a, bp);
            hostToPlanes(arena, (int)N, (int)a, ap);
            for (int p = 0; p < NUM_PADS; p++) hostToPlanes(pads, (int)(N * NUM_PADS), (int)(p * N + a), pp);
        }
        cudaMemcpy(h->dBall, ball.data(), ball.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(h->dArena, arena.data(), arena.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(h->dPad, pads.data(), pads.size() * 4, cudaMemcpyHostToDevice);
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
    EngineDev D = devView(h);
    int block = 128, grid = (h->N + block - 1) / block;
    stepKernel<<<grid, block, 0, pick(h, stream)>>>(D, ticks);
    RSB_CUDA(cudaGetLastError());
    h->stats.ticks_simulated += (uint64_t)h->N * ticks;
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

rsb_status rsb_get_balls(rsb_handle* h, rsb_ball_state* out, int32_t n) {
    if (!h || !out || n != h->N) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dBall, planes, (size_t)W_BALL * h->N);
    if (st) return st;
    for (int a = 0; a < n; a++) {
        BallP p;
        planesToHost(planes, h->N, a, p);
        rsb_ball_state& o = out[a];
        o.pos = rsb_vec3{p.pos[0] * kBtToUu, p.pos[1] * kBtToUu, p.pos[2] * kBtToUu};
        o.rot = rotFromBasis(p.rot);
        o.vel = rsb_vec3{p.lin[0] * kBtToUu, p.lin[1] * kBtToUu, p.lin[2] * kBtToUu};
        o.ang_vel = rsb_vec3{p.ang[0], p.ang[1], p.ang[2]};
    }
    return RSB_OK;
}

rsb_status rsb_set_balls(rsb_handle* h, const rsb_ball_state* in, int32_t n) {
    if (!h || !in || n != h->N) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dBall, planes, (size_t)W_BALL * h->N);
    if (st) return st;
    for (int a = 0; a < n; a++) {
        BallP p;
        planesToHost(planes, h->N, a, p);
        const rsb_ball_state& s = in[a];
        Xf x{basisFromRot(s.rot), V3{s.pos.x, s.pos.y, s.pos.z} * kUuToBt};
        xfToP(x, p.pos, p.rot);
        V3 v = V3{s.vel.x, s.vel.y, s.vel.z} * kUuToBt;
        p.lin[0] = v.x; p.lin[1] = v.y; p.lin[2] = v.z;
        p.ang[0] = s.ang_vel.x; p.ang[1] = s.ang_vel.y; p.ang[2] = s.ang_vel.z;
        hostToPlanes(planes, h->N, a, p);
    }
    return upload(h, h->dBall, planes);
}

rsb_status rsb_get_cars(rsb_handle* h, rsb_car_state* out, int32_t n) {
    if (!h || (n > 0 && !out) || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    return RSB_OK;
}

rsb_status rsb_set_cars(rsb_handle* h, const rsb_car_state* in, int32_t n) {
    if (!h || (n > 0 && !in) || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    return RSB_OK;
}

rsb_status rsb_get_pads(rsb_handle* h, rsb_pad_state* out, int32_t n) {
    if (!h || !out || n != h->N * RSB_NUM_PADS) return fail(h, RSB_ERR_INVALID, "pad count must equal num_arenas*34");
    std::vector<uint32_t> planes;
    rsb_status st = download(h, h->dPad, planes, (size_t)W_PAD * NUM_PADS * h->N);
    if (st) return st;
    for (int a = 0; a < h->N; a++)
        for (int p = 0; p < NUM_PADS; p++) {
            PadP pp;
            planesToHost(planes, h->N * NUM_PADS, p * h->N + a, pp);
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
            hostToPlanes(planes, h->N * NUM_PADS, p * h->N + a, pp);
        }
    return upload(h, h->dPad, planes);
}

rsb_status rsb_get_arena_info(rsb_handle* h, rsb_arena_info* out, int32_t n) {
    if (!h || !out || n != h->N) return fail(h, RSB_ERR_INVALID, "info count must equal num_arenas");
    std::vector<uint32_t> planes, balls;
    rsb_status st = download(h, h->dArena, planes, (size_t)W_ARENA * h->N);
    if (st) return st;
    st = download(h, h->dBall, balls, (size_t)W_BALL * h->N);
    if (st) return st;
    for (int a = 0; a < n; a++) {
        ArenaP ap;
        planesToHost(planes, h->N, a, ap);
        BallP bp;
        planesToHost(balls, h->N, a, bp);
        rsb_arena_info& o = out[a];
        o = rsb_arena_info{};
        o.tick_count = (uint64_t)ap.tick[0] | ((uint64_t)ap.tick[1] << 32);
        o.num_cars = 2 * h->teamSize[a];
        o.team_size = h->teamSize[a];
        float y = bp.pos[1] * kBtToUu;
        bool scored = fabsf(y) > (h->mut.goal_base_threshold_y + h->mut.ball_radius);
        o.goal_scored = scored;
        o.goal_team = scored ? (y > 0 ? 0 : 1) : -1;
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
        case RSB_BUF_CONTROLS: *out = h->dControls; return RSB_OK;
        case RSB_BUF_ACTIONS: *out = h->dActions; return RSB_OK;
        default: return fail(h, RSB_ERR_UNSUPPORTED, "buffer not built into this library yet");
    }
}

rsb_status rsb_reset_all(rsb_handle* h, uint64_t, int32_t) {
    return fail(h, RSB_ERR_UNSUPPORTED, "resets are not built into this library yet");
}
rsb_status rsb_reset_arenas(rsb_handle* h, const int32_t*, int32_t, uint64_t, int32_t) {
    return fail(h, RSB_ERR_UNSUPPORTED, "resets are not built into this library yet");
}
rsb_status rsb_default_action_lut(rsb_controls*, int32_t) { return RSB_ERR_UNSUPPORTED; }
rsb_status rsb_snapshot(rsb_handle* h, void*) { return fail(h, RSB_ERR_UNSUPPORTED, "not built yet"); }
rsb_status rsb_build_obs(rsb_handle* h, void*) { return fail(h, RSB_ERR_UNSUPPORTED, "not built yet"); }
rsb_status rsb_build_rewards_terminals(rsb_handle* h, int32_t, void*) { return fail(h, RSB_ERR_UNSUPPORTED, "not built yet"); }
rsb_status rsb_copy_obs(rsb_handle* h, float*, size_t) { return fail(h, RSB_ERR_UNSUPPORTED, "not built yet"); }
rsb_status rsb_copy_masks(rsb_handle* h, uint8_t*, size_t) { return fail(h, RSB_ERR_UNSUPPORTED, "not built yet"); }
rsb_status rsb_copy_rewards(rsb_handle* h, float*, size_t) { return fail(h, RSB_ERR_UNSUPPORTED, "not built yet"); }
rsb_status rsb_copy_terminals(rsb_handle* h, uint8_t*, size_t) { return fail(h, RSB_ERR_UNSUPPORTED, "not built yet"); }

}  // extern "C"
