// Host build of the engine's per-arena code behind part of the C ABI (include/rsb.h).
//
// Test infrastructure only: the physics headers under emy-s-framework_b200/csrc/phys are
// written once for host and device (phys/hd.h); this file compiles them with g++ and runs
// stepArena() on host copies of the word-plane records, so that tests can compare the
// restated algorithm with the reference on the CPU, tick by tick and byte by byte, without
// a GPU.  On the host, rsqrtEstimate() executes the CPU's rsqrtss and the sin / cos / atan2
// / asin restatements equal the C library's results, so any difference this build shows
// against the reference is a difference in the restated algorithm itself.
//
// Entry points: rsb_default_mutators, rsb_create, rsb_destroy, rsb_layout, rsb_obs_stride,
// rsb_last_error, rsb_set_controls, rsb_set_action_lut, rsb_set_actions_host, rsb_step,
// rsb_get/set_cars, rsb_get/set_balls, rsb_get/set_pads, rsb_get_arena_info,
// rsb_host_register / rsb_host_unregister (no-ops), and rsb_host_rsqrt_table (the host
// CPU's rsqrtss table).  Everything else is absent.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "arena_build.h"
#include "engine_host.h"

using namespace rsb;

namespace {
std::string g_error;
}

struct rsb_handle {
    int N = 0, numCars = 0, maxCars = 0, threads = 1;
    uint64_t seed = 0;
    std::vector<int32_t> teamSize, carOffset;
    WorldParams P{};
    ArenaStaticHost S;
    std::vector<uint32_t> ball, car, pad, arena;
    std::vector<rsb_controls> controls, lut;
    std::string err;
};

static rsb_status fail(rsb_handle* h, rsb_status code, const std::string& msg) {
    (h ? h->err : g_error) = msg;
    return code;
}

extern "C" {

rsb_status rsb_default_mutators(rsb_mutators* m) {
    if (!m) return RSB_ERR_INVALID;
    defaultMutators(m);
    return RSB_OK;
}

rsb_status rsb_last_error(const rsb_handle* h, char* buf, size_t n) {
    if (!buf || !n) return RSB_ERR_INVALID;
    const std::string& s = h ? h->err : g_error;
    std::snprintf(buf, n, "%s", s.c_str());
    return RSB_OK;
}

rsb_status rsb_create(const rsb_config* cfg, rsb_handle** out) {
    if (!cfg || !out) return fail(nullptr, RSB_ERR_INVALID, "null config or output");
    *out = nullptr;
    if (cfg->num_arenas <= 0) return fail(nullptr, RSB_ERR_INVALID, "num_arenas must be > 0");
    if (!cfg->meshes_path) return fail(nullptr, RSB_ERR_MESH, "meshes_path is required");
    std::unique_ptr<rsb_handle> h(new rsb_handle());
    h->N = cfg->num_arenas;
    h->seed = cfg->seed;
    h->threads = cfg->threads > 0 ? cfg->threads : (int)std::max(1u, std::thread::hardware_concurrency());
    h->carOffset.push_back(0);
    for (int a = 0; a < h->N; a++) {
        const int ts = cfg->team_sizes ? cfg->team_sizes[a] : cfg->team_size;
        if (ts < 0 || ts > RSB_MAX_TEAM_SIZE) return fail(nullptr, RSB_ERR_INVALID, "team size must be 0..3");
        h->teamSize.push_back(ts);
        h->carOffset.push_back(h->carOffset.back() + 2 * ts);
        h->maxCars = std::max(h->maxCars, 2 * ts);
    }
    h->numCars = h->carOffset.back();
    rsb_mutators m;
    if (cfg->mutators) m = *cfg->mutators;
    else defaultMutators(&m);
    computeParams(m, h->P);
    if (!buildArenaStatic(cfg->meshes_path, h->S)) return fail(nullptr, RSB_ERR_MESH, h->S.error);
    HostRecords R;
    initRecords(h->S.view, h->P, h->teamSize, R);
    h->ball = R.ball;
    h->car = R.car;
    h->pad = R.pad;
    h->arena = R.arena;
    h->controls.assign(std::max(1, h->numCars), rsb_controls{});
    *out = h.release();
    return RSB_OK;
}

rsb_status rsb_destroy(rsb_handle* h) {
    if (!h) return RSB_ERR_INVALID;
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

// The rsqrtss table the CUDA engine would upload on this host (phys/refmath.h); returns 1 when
// the CPU's estimate has the table's form, 0 when the table holds exact values instead.
int32_t rsb_host_rsqrt_table(uint32_t* out) { return sampleRsqrtTable(out) ? 1 : 0; }

// rsqrtss through the table the engine samples and uploads (the device's lookup, on the host).
static float rsqrtEstimateTable(float x) {
    static uint32_t table[kRsqrtTableSize];
    static const bool filled = (sampleRsqrtTable(table), true);
    (void)filled;
    return rsqrtFromTable(table, x);
}

// The host C library's sinf / cosf / asinf / atan2f(x, y) and the CPU's rsqrtss on n inputs
// (fn as rsb_eval_refmath), the values the device restatements must reproduce.
int32_t rsb_host_libm(int32_t fn, const float* x, const float* y, float* out, int64_t n) {
    for (int64_t i = 0; i < n; i++) {
        switch (fn) {
            case RSB_MATH_RSQRT_EST: out[i] = _mm_cvtss_f32(_mm_rsqrt_ss(_mm_set_ss(x[i]))); break;
            case RSB_MATH_SIN: out[i] = sinf(x[i]); break;
            case RSB_MATH_COS: out[i] = cosf(x[i]); break;
            case RSB_MATH_ASIN: out[i] = asinf(x[i]); break;
            case RSB_MATH_ATAN2: out[i] = atan2f(x[i], y[i]); break;
            default: return RSB_ERR_INVALID;
        }
    }
    return RSB_OK;
}

// Compares the restatements of phys/refmath.h (host build) with the C library on the floats
// with bit patterns offset, offset + stride, ... (all of them below 2^32), on `threads`
// threads; sin / cos inputs are limited to |x| < 120.  atan2f is checked on pairs of those
// floats with a second operand drawn from a fixed xorshift stream.  Returns the mismatches.
int64_t rsb_host_refmath_check(int32_t fn, uint32_t stride, uint32_t offset, int32_t threads, int64_t* tested) {
    std::vector<int64_t> bad(threads, 0), cnt(threads, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back([&, t] {
            uint32_t rng = 0x9E3779B9u ^ (uint32_t)t;
            for (uint64_t u = (uint64_t)offset + (uint64_t)t * stride; u < (1ull << 32); u += (uint64_t)stride * threads) {
                const float x = u2f((uint32_t)u);
                if (!std::isfinite(x)) continue;
                float a, b;
                switch (fn) {
                    case RSB_MATH_RSQRT_EST: a = _mm_cvtss_f32(_mm_rsqrt_ss(_mm_set_ss(x))); b = rsqrtEstimateTable(x); break;
                    case RSB_MATH_SIN: if (!(fabsf(x) < 120.f)) continue; a = sinf(x); b = rsSinf(x); break;
                    case RSB_MATH_COS: if (!(fabsf(x) < 120.f)) continue; a = cosf(x); b = rsCosf(x); break;
                    case RSB_MATH_ASIN: a = asinf(x); b = rsAsinf(x); break;
                    default: {
                        rng ^= rng << 13; rng ^= rng >> 17; rng ^= rng << 5;
                        const float y = u2f(rng);
                        if (!std::isfinite(y)) continue;
                        a = atan2f(x, y);
                        b = rsAtan2f(x, y);
                    }
                }
                cnt[t]++;
                if (f2u(a) != f2u(b) && !(std::isnan(a) && std::isnan(b))) bad[t]++;
            }
        });
    for (auto& th : pool) th.join();
    int64_t nb = 0, nc = 0;
    for (int t = 0; t < threads; t++) { nb += bad[t]; nc += cnt[t]; }
    if (tested) *tested = nc;
    return nb;
}

// The voxel distance bound (ArenaStatic::occDist, uu) of the handle's static data at n points
// (uu, 3 floats each): 0 off the grid.
int32_t rsb_host_voxel_bound(const rsb_handle* h, const float* pts, int64_t n, float* out) {
    if (!h || !pts || !out) return RSB_ERR_INVALID;
    const ArenaStatic& S = h->S.view;
    for (int64_t i = 0; i < n; i++) {
        const int x = (int)std::floor((pts[3 * i] * kUuToBt - S.occMin.x) * S.occInvCell);
        const int y = (int)std::floor((pts[3 * i + 1] * kUuToBt - S.occMin.y) * S.occInvCell);
        const int z = (int)std::floor((pts[3 * i + 2] * kUuToBt - S.occMin.z) * S.occInvCell);
        const bool in = x >= 0 && y >= 0 && z >= 0 && x < S.occX && y < S.occY && z < S.occZ;
        out[i] = in ? (float)S.occDist[((size_t)x * S.occY + y) * S.occZ + z] : 0.f;
    }
    return RSB_OK;
}

rsb_status rsb_host_register(void*, size_t) { return RSB_OK; }
rsb_status rsb_host_unregister(void*) { return RSB_OK; }

rsb_status rsb_set_controls(rsb_handle* h, const rsb_controls* c, int32_t n) {
    if (!h || !c || n != h->numCars) return fail(h, RSB_ERR_INVALID, "controls count must equal num_cars");
    std::copy(c, c + n, h->controls.begin());
    return RSB_OK;
}

rsb_status rsb_set_action_lut(rsb_handle* h, const rsb_controls* lut, int32_t count) {
    if (!h || !lut || count <= 0) return fail(h, RSB_ERR_INVALID, "empty action table");
    h->lut.assign(lut, lut + count);
    return RSB_OK;
}

rsb_status rsb_set_actions_host(rsb_handle* h, const int32_t* idx, int32_t n) {
    if (!h || !idx || n != h->numCars) return fail(h, RSB_ERR_INVALID, "action count must equal num_cars");
    if (h->lut.empty()) return fail(h, RSB_ERR_STATE, "no action table uploaded");
    const int c = (int)h->lut.size();
    for (int i = 0; i < n; i++) h->controls[i] = h->lut[std::min(std::max(idx[i], 0), c - 1)];
    return RSB_OK;
}

rsb_status rsb_step(rsb_handle* h, int32_t ticks, void*) {
    if (!h || ticks < 0) return fail(h, RSB_ERR_INVALID, "bad tick count");
    EngineView D;
    D.S = h->S.view;
    D.P = h->P;
    D.N = h->N;
    D.teamSize = h->teamSize.data();
    D.carOffset = h->carOffset.data();
    D.ball = h->ball.data();
    D.car = h->car.data();
    D.pad = h->pad.data();
    D.arena = h->arena.data();
    D.controls = reinterpret_cast<const CtlRec*>(h->controls.data());
    D.seed = (uint32_t)(h->seed ^ (h->seed >> 32));
    D.cull = nullptr;
    D.cullAudit = 0;
    D.counters = nullptr;
    D.work = nullptr;
    const int T = std::min(h->threads, h->N);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++)
        pool.emplace_back([&, t] {
            std::unique_ptr<ArenaSim> A(new ArenaSim());
            std::unique_ptr<EpaWork> epa(new EpaWork());
            for (int a = t; a < h->N; a += T) {
                A->W.epa = epa.get();
                stepArena(D, a, ticks, *A);
            }
        });
    for (auto& th : pool) th.join();
    return RSB_OK;
}

rsb_status rsb_get_balls(rsb_handle* h, rsb_ball_state* out, int32_t n) {
    if (!h || !out || n != h->N) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    for (int a = 0; a < n; a++) {
        BallP p;
        loadPlanes(p, h->ball.data(), a, h->N);
        out[a] = ballStateOf(p);
    }
    return RSB_OK;
}

rsb_status rsb_set_balls(rsb_handle* h, const rsb_ball_state* in, int32_t n) {
    if (!h || !in || n != h->N) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    for (int a = 0; a < n; a++) {
        BallP p;
        loadPlanes(p, h->ball.data(), a, h->N);
        applyBallState(p, in[a]);
        storePlanes(p, h->ball.data(), a, h->N);
        ArenaP ap;
        loadPlanes(ap, h->arena.data(), a, h->N);
        const float y = p.pos[1] * kBtToUu;
        ap.scored = fabsf(y) > (h->P.goalBaseY + h->P.ballRadiusUu) ? (p.pos[1] > 0 ? 1 : 2) : 0;
        storePlanes(ap, h->arena.data(), a, h->N);
    }
    return RSB_OK;
}

rsb_status rsb_get_cars(rsb_handle* h, rsb_car_state* out, int32_t n) {
    if (!h || (n > 0 && !out) || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    for (int a = 0; a < h->N; a++)
        for (int s = 0; s < 2 * h->teamSize[a]; s++) {
            CarP p;
            loadPlanes(p, h->car.data(), s * h->N + a, MAX_CARS * h->N);
            out[h->carOffset[a] + s] = carStateOf(p, (uint32_t)s + 1u);
        }
    return RSB_OK;
}

rsb_status rsb_set_cars(rsb_handle* h, const rsb_car_state* in, int32_t n) {
    if (!h || (n > 0 && !in) || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    for (int a = 0; a < h->N; a++)
        for (int s = 0; s < 2 * h->teamSize[a]; s++) {
            CarP p;
            loadPlanes(p, h->car.data(), s * h->N + a, MAX_CARS * h->N);
            applyCarState(p, in[h->carOffset[a] + s]);
            storePlanes(p, h->car.data(), s * h->N + a, MAX_CARS * h->N);
        }
    return RSB_OK;
}

rsb_status rsb_get_pads(rsb_handle* h, rsb_pad_state* out, int32_t n) {
    if (!h || !out || n != h->N * RSB_NUM_PADS) return fail(h, RSB_ERR_INVALID, "pad count must equal num_arenas*34");
    for (int a = 0; a < h->N; a++)
        for (int p = 0; p < NUM_PADS; p++) {
            PadP pp;
            loadPlanes(pp, h->pad.data(), p * h->N + a, h->N * NUM_PADS);
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
    for (int a = 0; a < h->N; a++)
        for (int p = 0; p < NUM_PADS; p++) {
            const rsb_pad_state& s = in[a * NUM_PADS + p];
            PadP pp;
            pp.cooldown = s.cooldown;
            pp.bits = (s.is_active ? 1u : 0u) | (s.prev_locked_car_id << 8);
            storePlanes(pp, h->pad.data(), p * h->N + a, h->N * NUM_PADS);
        }
    return RSB_OK;
}

rsb_status rsb_get_arena_info(rsb_handle* h, rsb_arena_info* out, int32_t n) {
    if (!h || !out || n != h->N) return fail(h, RSB_ERR_INVALID, "info count must equal num_arenas");
    for (int a = 0; a < n; a++) {
        ArenaP ap;
        loadPlanes(ap, h->arena.data(), a, h->N);
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

}  // extern "C"
