// ORACLE — test infrastructure only.  Puts the reference CPU RocketSim
// (GigaLearnCPP/RLGymCPP/RocketSim, built from the reference's own sources by
// oracle/Makefile) behind the engine's C ABI (include/rsb.h), so that every test
// and the CPU-baseline leg of the benchmark can drive the reference and the CUDA
// engine through identical calls.  Nothing in the product links this file.
//
// Reference behaviour followed:
//   - RocketSim::InitFromMem            RocketSim.cpp:102-212 (meshes fed in mesh_0..mesh_15
//                                       numeric order, so that the collision-object order,
//                                       and hence Bullet's pair/manifold order, is fixed
//                                       instead of following directory_iterator order)
//   - Arena::Create / AddCar / Step     Arena.cpp:48-60, 716-812
//   - Car::GetState / SetState          Car.cpp:9-35
//   - Ball::GetState / SetState         Ball.cpp:27-49
//   - BoostPad::GetState / SetState     BoostPad.h:45-46
//   - Arena::IsBallScored               Arena.cpp:949-957
//   - the collector's env step          RLGymCPP EnvSet.cpp:117-260, 392-424 (GameState,
//                                       AdvancedObs, DefaultAction masks, the four stub
//                                       rewards, ZeroSumReward, terminal conditions,
//                                       kickoff / RandomState resets), run with
//                                       RLGymCPP's own classes
#include "rsb.h"

#include "RocketSim.h"
#include "RLGymCPP/ActionParsers/DefaultAction.h"
#include "RLGymCPP/Gamestates/GameState.h"
#include "RLGymCPP/ObsBuilders/AdvancedObs.h"
#include "RLGymCPP/RewardCore/CommonRewards.h"
#include "RLGymCPP/RewardCore/RuntimeRewardRegistry.h"
#include "RLGymCPP/RewardCore/ZeroSumReward.h"
#include "RLGymCPP/StateSetters/RandomState.h"
#include "RLGymCPP/TerminalConditions/GoalScoreCondition.h"
#include "RLGymCPP/TerminalConditions/NoTouchCondition.h"

#include <xmmintrin.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace RocketSim;

// Env state of one arena: what EnvSet keeps per arena for the collector's path
// (EnvSet.cpp:117-260): the reward list (each optionally wrapped in ZeroSumReward) and
// the terminal conditions, plus the actions of the last step for the observations.
struct OracleEnv {
    std::vector<std::pair<RLGC::Reward*, float>> rewards;
    std::vector<RLGC::TerminalCondition*> terminals;
};

// Truncation after a fixed number of ticks since the last reset (the learner's episode cap).
struct EpisodeTickLimit : RLGC::TerminalCondition {
    const int32_t* ticks;
    int32_t limit;
    EpisodeTickLimit(const int32_t* t, int32_t l) : ticks(t), limit(l) {}
    bool IsTerminal(const RLGC::GameState&) override { return *ticks >= limit; }
    bool IsTruncation() override { return true; }
};

struct rsb_handle {
    std::vector<Arena*> arenas;
    std::vector<std::vector<Car*>> cars;  // per arena, blue first then orange
    std::vector<int32_t> teamSize;
    std::vector<int32_t> carOffset;
    std::vector<rsb_controls> lut;
    std::vector<rsb_controls> controls;
    std::vector<int32_t> episodeTicks;
    MutatorConfig mut = MutatorConfig(GameMode::SOCCAR);
    std::vector<Arena*> predArenas;  // ball-only arenas of the ball prediction (BallPredTracker)
    int32_t numCars = 0;
    int32_t threads = 1;
    std::string err;
    rsb_stats stats{};
    // env layer
    bool hasRewards = false;
    rsb_reward_config rewardCfg{};
    std::vector<OracleEnv> env;
    std::vector<float> obs, rewardsOut;
    std::vector<uint8_t> masks, terminalsOut;
    // state ring: CudaEnvSet's host-side ring (CudaEnvSet.h:148-170), slots of public states
    struct ArenaSnap {
        std::vector<CarState> cars;
        BallState ball;
        std::vector<BoostPadState> pads;
        bool valid = false;
    };
    struct Ring {
        bool enabled = false, replayDisabled = false;
        rsb_ring_config cfg{};
        uint32_t rng = 0xA5A5A5A5u;
        std::vector<std::vector<ArenaSnap>> slots;
        int writeIdx = 0, filled = 0, stepsSinceCapture = 0;
        uint64_t captures = 0, restores = 0, restoreCalls = 0;
    } ring;
};

static std::string g_createError;
static void buildEnv(rsb_handle* h);
static void freeEnv(rsb_handle* h);
static std::mutex g_initMutex;
static bool g_inited = false;

static rsb_status fail(rsb_handle* h, rsb_status code, const std::string& msg) {
    if (h) h->err = msg; else g_createError = msg;
    return code;
}

static bool initMeshes(const char* path, std::string& err) {
    std::lock_guard<std::mutex> lock(g_initMutex);
    if (g_inited) return true;
    std::vector<FileData> files;
    for (int i = 0; i < 64; i++) {
        std::filesystem::path p = std::filesystem::path(path) / "soccar" / ("mesh_" + std::to_string(i) + ".cmf");
        if (!std::filesystem::exists(p)) break;
        std::ifstream f(p, std::ios::binary);
        FileData d((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        files.push_back(std::move(d));
    }
    if (files.empty()) {
        err = std::string("no soccar/mesh_<i>.cmf under ") + path;
        return false;
    }
    std::map<GameMode, std::vector<FileData>> m;
    m[GameMode::SOCCAR] = files;
    RocketSim::InitFromMem(m, true);
    g_inited = true;
    return true;
}

static Vec toVec(const rsb_vec3& v) { return Vec(v.x, v.y, v.z); }
static rsb_vec3 fromVec(const Vec& v) { return rsb_vec3{v.x, v.y, v.z}; }

static CarControls toControls(const rsb_controls& c) {
    CarControls r;
    r.throttle = c.throttle; r.steer = c.steer; r.pitch = c.pitch; r.yaw = c.yaw; r.roll = c.roll;
    r.jump = c.jump != 0; r.boost = c.boost != 0; r.handbrake = c.handbrake != 0;
    return r;
}
static rsb_controls fromControls(const CarControls& c) {
    rsb_controls r{};
    r.throttle = c.throttle; r.steer = c.steer; r.pitch = c.pitch; r.yaw = c.yaw; r.roll = c.roll;
    r.jump = c.jump; r.boost = c.boost; r.handbrake = c.handbrake;
    return r;
}

static rsb_car_state fromCarState(const CarState& s, Team team, uint32_t id) {
    rsb_car_state o{};
    o.pos = fromVec(s.pos);
    o.rot.forward = fromVec(s.rotMat.forward);
    o.rot.right = fromVec(s.rotMat.right);
    o.rot.up = fromVec(s.rotMat.up);
    o.vel = fromVec(s.vel);
    o.ang_vel = fromVec(s.angVel);
    o.boost = s.boost;
    o.time_spent_boosting = s.timeSpentBoosting;
    o.jump_time = s.jumpTime; o.flip_time = s.flipTime;
    o.air_time = s.airTime; o.air_time_since_jump = s.airTimeSinceJump;
    o.supersonic_time = s.supersonicTime; o.handbrake_val = s.handbrakeVal;
    o.auto_flip_timer = s.autoFlipTimer; o.auto_flip_torque_scale = s.autoFlipTorqueScale;
    o.demo_respawn_timer = s.demoRespawnTimer;
    o.car_contact_cooldown = s.carContact.cooldownTimer;
    o.flip_rel_torque = fromVec(s.flipRelTorque);
    o.world_contact_normal = fromVec(s.worldContact.contactNormal);
    o.car_contact_other_id = s.carContact.otherCarID;
    o.is_on_ground = s.isOnGround; o.has_jumped = s.hasJumped;
    o.has_double_jumped = s.hasDoubleJumped; o.has_flipped = s.hasFlipped;
    o.is_flipping = s.isFlipping; o.is_jumping = s.isJumping;
    o.is_supersonic = s.isSupersonic; o.is_auto_flipping = s.isAutoFlipping;
    o.is_demoed = s.isDemoed; o.world_contact = s.worldContact.hasContact;
    o.ball_hit_valid = s.ballHitInfo.isValid;
    o.team = (team == Team::BLUE) ? 0 : 1;
    for (int i = 0; i < 4; i++) o.wheels_with_contact[i] = s.wheelsWithContact[i];
    o.ball_hit_tick = s.ballHitInfo.tickCountWhenHit;
    o.ball_hit_extra_tick = s.ballHitInfo.tickCountWhenExtraImpulseApplied;
    o.ball_hit_rel_pos = fromVec(s.ballHitInfo.relativePosOnBall);
    o.ball_hit_ball_pos = fromVec(s.ballHitInfo.ballPos);
    o.ball_hit_extra_vel = fromVec(s.ballHitInfo.extraHitVel);
    o.last_controls = fromControls(s.lastControls);
    o.id = id;
    return o;
}

static CarState toCarState(const rsb_car_state& o) {
    CarState s;
    s.pos = toVec(o.pos);
    s.rotMat = RotMat(toVec(o.rot.forward), toVec(o.rot.right), toVec(o.rot.up));
    s.vel = toVec(o.vel);
    s.angVel = toVec(o.ang_vel);
    s.boost = o.boost;
    s.timeSpentBoosting = o.time_spent_boosting;
    s.jumpTime = o.jump_time; s.flipTime = o.flip_time;
    s.airTime = o.air_time; s.airTimeSinceJump = o.air_time_since_jump;
    s.supersonicTime = o.supersonic_time; s.handbrakeVal = o.handbrake_val;
    s.autoFlipTimer = o.auto_flip_timer; s.autoFlipTorqueScale = o.auto_flip_torque_scale;
    s.demoRespawnTimer = o.demo_respawn_timer;
    s.carContact.cooldownTimer = o.car_contact_cooldown;
    s.flipRelTorque = toVec(o.flip_rel_torque);
    s.worldContact.contactNormal = toVec(o.world_contact_normal);
    s.carContact.otherCarID = o.car_contact_other_id;
    s.isOnGround = o.is_on_ground; s.hasJumped = o.has_jumped;
    s.hasDoubleJumped = o.has_double_jumped; s.hasFlipped = o.has_flipped;
    s.isFlipping = o.is_flipping; s.isJumping = o.is_jumping;
    s.isSupersonic = o.is_supersonic; s.isAutoFlipping = o.is_auto_flipping;
    s.isDemoed = o.is_demoed; s.worldContact.hasContact = o.world_contact;
    s.ballHitInfo.isValid = o.ball_hit_valid;
    for (int i = 0; i < 4; i++) s.wheelsWithContact[i] = o.wheels_with_contact[i];
    s.ballHitInfo.tickCountWhenHit = o.ball_hit_tick;
    s.ballHitInfo.tickCountWhenExtraImpulseApplied = o.ball_hit_extra_tick;
    s.ballHitInfo.relativePosOnBall = toVec(o.ball_hit_rel_pos);
    s.ballHitInfo.ballPos = toVec(o.ball_hit_ball_pos);
    s.ballHitInfo.extraHitVel = toVec(o.ball_hit_extra_vel);
    s.lastControls = toControls(o.last_controls);
    return s;
}

// Runs fn(a) for every arena on the handle's host threads (EnvSet runs its per-arena
// work on a thread pool in the same way, EnvSet.cpp:113-260).
template <class Fn>
static void forArenas(rsb_handle* h, Fn fn) {
    int n = (int)h->arenas.size();
    int t = std::min(h->threads, n);
    if (t <= 1) {
        for (int a = 0; a < n; a++) fn(a);
        return;
    }
    std::vector<std::thread> pool;
    std::atomic<int> next{0};
    const int chunk = 4;
    for (int i = 0; i < t; i++)
        pool.emplace_back([&] {
            for (;;) {
                int a0 = next.fetch_add(chunk);
                if (a0 >= n) break;
                for (int a = a0; a < std::min(n, a0 + chunk); a++) fn(a);
            }
        });
    for (auto& th : pool) th.join();
}

extern "C" {

rsb_status rsb_default_mutators(rsb_mutators* m) {
    if (!m) return RSB_ERR_INVALID;
    MutatorConfig d(GameMode::SOCCAR);
    m->gravity = fromVec(d.gravity);
    m->car_mass = d.carMass; m->car_world_friction = d.carWorldFriction;
    m->car_world_restitution = d.carWorldRestitution;
    m->ball_mass = d.ballMass; m->ball_max_speed = d.ballMaxSpeed; m->ball_drag = d.ballDrag;
    m->ball_world_friction = d.ballWorldFriction; m->ball_world_restitution = d.ballWorldRestitution;
    m->jump_accel = d.jumpAccel; m->jump_immediate_force = d.jumpImmediateForce;
    m->boost_accel_ground = d.boostAccelGround; m->boost_accel_air = d.boostAccelAir;
    m->boost_used_per_second = d.boostUsedPerSecond;
    m->respawn_delay = d.respawnDelay; m->bump_cooldown_time = d.bumpCooldownTime;
    m->boost_pad_cooldown_big = d.boostPadCooldown_Big;
    m->boost_pad_cooldown_small = d.boostPadCooldown_Small;
    m->car_spawn_boost_amount = d.carSpawnBoostAmount;
    m->ball_hit_extra_force_scale = d.ballHitExtraForceScale;
    m->bump_force_scale = d.bumpForceScale; m->ball_radius = d.ballRadius;
    m->unlimited_flips = d.unlimitedFlips; m->unlimited_double_jumps = d.unlimitedDoubleJumps;
    m->demo_mode = (uint8_t)d.demoMode; m->enable_team_demos = d.enableTeamDemos;
    m->goal_base_threshold_y = d.goalBaseThresholdY;
    return RSB_OK;
}

static MutatorConfig toMutators(const rsb_mutators& m) {
    MutatorConfig d(GameMode::SOCCAR);
    d.gravity = toVec(m.gravity);
    d.carMass = m.car_mass; d.carWorldFriction = m.car_world_friction;
    d.carWorldRestitution = m.car_world_restitution;
    d.ballMass = m.ball_mass; d.ballMaxSpeed = m.ball_max_speed; d.ballDrag = m.ball_drag;
    d.ballWorldFriction = m.ball_world_friction; d.ballWorldRestitution = m.ball_world_restitution;
    d.jumpAccel = m.jump_accel; d.jumpImmediateForce = m.jump_immediate_force;
    d.boostAccelGround = m.boost_accel_ground; d.boostAccelAir = m.boost_accel_air;
    d.boostUsedPerSecond = m.boost_used_per_second;
    d.respawnDelay = m.respawn_delay; d.bumpCooldownTime = m.bump_cooldown_time;
    d.boostPadCooldown_Big = m.boost_pad_cooldown_big;
    d.boostPadCooldown_Small = m.boost_pad_cooldown_small;
    d.carSpawnBoostAmount = m.car_spawn_boost_amount;
    d.ballHitExtraForceScale = m.ball_hit_extra_force_scale;
    d.bumpForceScale = m.bump_force_scale; d.ballRadius = m.ball_radius;
    d.unlimitedFlips = m.unlimited_flips; d.unlimitedDoubleJumps = m.unlimited_double_jumps;
    d.demoMode = (DemoMode)m.demo_mode; d.enableTeamDemos = m.enable_team_demos;
    d.goalBaseThresholdY = m.goal_base_threshold_y;
    return d;
}

rsb_status rsb_create(const rsb_config* cfg, rsb_handle** out) {
    if (!cfg || !out) return fail(nullptr, RSB_ERR_INVALID, "null config or output");
    *out = nullptr;
    if (cfg->num_arenas <= 0) return fail(nullptr, RSB_ERR_INVALID, "num_arenas must be > 0");
    if (!cfg->meshes_path) return fail(nullptr, RSB_ERR_MESH, "meshes_path is required");
    if (cfg->tick_rate != 120.f) return fail(nullptr, RSB_ERR_UNSUPPORTED, "tick_rate must be 120");
    std::string err;
    if (!initMeshes(cfg->meshes_path, err)) return fail(nullptr, RSB_ERR_MESH, err);

    rsb_handle* h = new rsb_handle();
    h->threads = cfg->threads > 0 ? cfg->threads : (int)std::max(1u, std::thread::hardware_concurrency());
    h->carOffset.push_back(0);
    for (int a = 0; a < cfg->num_arenas; a++) {
        int ts = cfg->team_sizes ? cfg->team_sizes[a] : cfg->team_size;
        if (ts < 0 || ts > RSB_MAX_TEAM_SIZE) {
            delete h;
            return fail(nullptr, RSB_ERR_INVALID, "team size must be 0..3");
        }
        h->teamSize.push_back(ts);
        h->carOffset.push_back(h->carOffset.back() + 2 * ts);
    }
    h->numCars = h->carOffset.back();
    MutatorConfig mut(GameMode::SOCCAR);
    if (cfg->mutators) mut = toMutators(*cfg->mutators);
    h->mut = mut;
    h->arenas.resize(cfg->num_arenas);
    h->cars.resize(cfg->num_arenas);
    for (int a = 0; a < cfg->num_arenas; a++) {
        Arena* arena = Arena::Create(GameMode::SOCCAR);
        arena->SetMutatorConfig(mut);
        for (int t = 0; t < 2; t++)
            for (int i = 0; i < h->teamSize[a]; i++)
                h->cars[a].push_back(arena->AddCar(t == 0 ? Team::BLUE : Team::ORANGE));
        h->arenas[a] = arena;
    }
    h->controls.assign(h->numCars, rsb_controls{});
    h->episodeTicks.assign(cfg->num_arenas, 0);
    if (cfg->rewards) {
        h->hasRewards = true;
        h->rewardCfg = *cfg->rewards;
        buildEnv(h);
    }
    *out = h;
    return RSB_OK;
}

rsb_status rsb_destroy(rsb_handle* h) {
    if (!h) return RSB_ERR_INVALID;
    freeEnv(h);
    for (Arena* a : h->arenas) delete a;
    for (Arena* a : h->predArenas) delete a;
    delete h;
    return RSB_OK;
}

rsb_status rsb_layout(const rsb_handle* h, int32_t* num_arenas, int32_t* num_cars,
                      int32_t* car_offset, int32_t* team_size) {
    if (!h) return RSB_ERR_INVALID;
    if (num_arenas) *num_arenas = (int32_t)h->arenas.size();
    if (num_cars) *num_cars = h->numCars;
    if (car_offset) std::memcpy(car_offset, h->carOffset.data(), h->carOffset.size() * sizeof(int32_t));
    if (team_size) std::memcpy(team_size, h->teamSize.data(), h->teamSize.size() * sizeof(int32_t));
    return RSB_OK;
}

rsb_status rsb_set_controls(rsb_handle* h, const rsb_controls* c, int32_t n) {
    if (!h || !c || n != h->numCars) return fail(h, RSB_ERR_INVALID, "controls count must equal num_cars");
    std::memcpy(h->controls.data(), c, sizeof(rsb_controls) * n);
    return RSB_OK;
}

rsb_status rsb_set_action_lut(rsb_handle* h, const rsb_controls* lut, int32_t count) {
    if (!h || !lut || count <= 0) return fail(h, RSB_ERR_INVALID, "bad action table");
    h->lut.assign(lut, lut + count);
    return RSB_OK;
}

rsb_status rsb_set_actions_host(rsb_handle* h, const int32_t* idx, int32_t n) {
    if (!h || !idx || n != h->numCars) return fail(h, RSB_ERR_INVALID, "action count must equal num_cars");
    if (h->lut.empty()) return fail(h, RSB_ERR_STATE, "no action table");
    int last = (int)h->lut.size() - 1;
    for (int i = 0; i < n; i++) {
        int k = idx[i] < 0 ? 0 : (idx[i] > last ? last : idx[i]);
        h->controls[i] = h->lut[k];
    }
    return RSB_OK;
}

// CPU implementation: no device staging exists, so this equals rsb_set_actions_host.
rsb_status rsb_set_actions_host_static(rsb_handle* h, const int32_t* idx, int32_t n) {
    if (n > RSB_STATIC_ACTIONS_MAX) return fail(h, RSB_ERR_INVALID, "more than RSB_STATIC_ACTIONS_MAX actions");
    return rsb_set_actions_host(h, idx, n);
}

static void stepRange(rsb_handle* h, int a0, int a1, int ticks) {
    for (int a = a0; a < a1; a++) {
        auto& cars = h->cars[a];
        for (size_t c = 0; c < cars.size(); c++)
            cars[c]->controls = toControls(h->controls[h->carOffset[a] + c]);
        h->arenas[a]->Step(ticks);
        h->episodeTicks[a] += ticks;
    }
}

rsb_status rsb_step(rsb_handle* h, int32_t ticks, void*) {
    if (!h || ticks < 0) return fail(h, RSB_ERR_INVALID, "bad tick count");
    forArenas(h, [&](int a) { stepRange(h, a, a + 1, ticks); });
    h->stats.ticks_simulated += (uint64_t)h->arenas.size() * ticks;
    return RSB_OK;
}

rsb_status rsb_get_cars(rsb_handle* h, rsb_car_state* out, int32_t n) {
    if (!h || !out || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    for (size_t a = 0; a < h->arenas.size(); a++)
        for (size_t c = 0; c < h->cars[a].size(); c++) {
            Car* car = h->cars[a][c];
            out[h->carOffset[a] + c] = fromCarState(car->GetState(), car->team, car->id);
        }
    return RSB_OK;
}

rsb_status rsb_set_cars(rsb_handle* h, const rsb_car_state* in, int32_t n) {
    if (!h || !in || n != h->numCars) return fail(h, RSB_ERR_INVALID, "car count must equal num_cars");
    for (size_t a = 0; a < h->arenas.size(); a++)
        for (size_t c = 0; c < h->cars[a].size(); c++)
            h->cars[a][c]->SetState(toCarState(in[h->carOffset[a] + c]));
    return RSB_OK;
}

static rsb_ball_state ballOut(const BallState& s) {
    rsb_ball_state o{};
    o.pos = fromVec(s.pos);
    o.rot.forward = fromVec(s.rotMat.forward);
    o.rot.right = fromVec(s.rotMat.right);
    o.rot.up = fromVec(s.rotMat.up);
    o.vel = fromVec(s.vel);
    o.ang_vel = fromVec(s.angVel);
    return o;
}

// BallPredTracker (BallPredTracker.cpp:3-10, 80-88): one ball-only arena per arena, made once
// with the batch's mutators; each prediction sets the arena's ball into it and steps one tick
// at a time, recording the ball after each slice's tick count.
rsb_status rsb_predict_ball(rsb_handle* h, const int32_t* slice_ticks, int32_t n_slices, rsb_ball_state* out,
                            size_t out_count, void*) {
    if (!h || !slice_ticks || n_slices < 1 || n_slices > RSB_MAX_PRED_SLICES)
        return fail(h, RSB_ERR_INVALID, "rsb_predict_ball: 1..8 slice ticks are required");
    for (int k = 0; k < n_slices; k++) {
        const int32_t prev = k ? slice_ticks[k - 1] : 0;
        if (slice_ticks[k] <= prev || slice_ticks[k] > RSB_MAX_PRED_TICKS)
            return fail(h, RSB_ERR_INVALID, "rsb_predict_ball: slice ticks must rise, from 1 to 4096");
    }
    const size_t n = h->arenas.size();
    if (!out || out_count != n * (size_t)n_slices)
        return fail(h, RSB_ERR_INVALID, "rsb_predict_ball: the oracle needs a host out of num_arenas * n_slices");
    if (h->predArenas.empty()) {
        for (size_t a = 0; a < n; a++) {
            Arena* p = Arena::Create(GameMode::SOCCAR);
            p->SetMutatorConfig(h->mut);
            h->predArenas.push_back(p);
        }
    }
    forArenas(h, [&](int a) {
        Arena* p = h->predArenas[a];
        p->ball->SetState(h->arenas[a]->ball->GetState());
        int t = 0;
        for (int k = 0; k < n_slices; k++) {
            for (; t < slice_ticks[k]; t++) p->Step(1);
            out[(size_t)a * n_slices + k] = ballOut(p->ball->GetState());
        }
    });
    return RSB_OK;
}

rsb_status rsb_get_balls(rsb_handle* h, rsb_ball_state* out, int32_t n) {
    if (!h || !out || n != (int32_t)h->arenas.size()) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    for (int a = 0; a < n; a++) out[a] = ballOut(h->arenas[a]->ball->GetState());
    return RSB_OK;
}

rsb_status rsb_set_balls(rsb_handle* h, const rsb_ball_state* in, int32_t n) {
    if (!h || !in || n != (int32_t)h->arenas.size()) return fail(h, RSB_ERR_INVALID, "ball count must equal num_arenas");
    for (int a = 0; a < n; a++) {
        BallState s;
        s.pos = toVec(in[a].pos);
        s.rotMat = RotMat(toVec(in[a].rot.forward), toVec(in[a].rot.right), toVec(in[a].rot.up));
        s.vel = toVec(in[a].vel);
        s.angVel = toVec(in[a].ang_vel);
        h->arenas[a]->ball->SetState(s);
    }
    return RSB_OK;
}

rsb_status rsb_get_pads(rsb_handle* h, rsb_pad_state* out, int32_t n) {
    if (!h || !out || n != (int32_t)h->arenas.size() * RSB_NUM_PADS) return fail(h, RSB_ERR_INVALID, "pad count must equal num_arenas*34");
    for (size_t a = 0; a < h->arenas.size(); a++) {
        auto& pads = h->arenas[a]->GetBoostPads();
        for (int p = 0; p < RSB_NUM_PADS; p++) {
            BoostPadState s = pads[p]->GetState();
            rsb_pad_state& o = out[a * RSB_NUM_PADS + p];
            o = rsb_pad_state{};
            o.is_active = s.isActive;
            o.cooldown = s.cooldown;
            o.prev_locked_car_id = s.prevLockedCarID;
        }
    }
    return RSB_OK;
}

rsb_status rsb_set_pads(rsb_handle* h, const rsb_pad_state* in, int32_t n) {
    if (!h || !in || n != (int32_t)h->arenas.size() * RSB_NUM_PADS) return fail(h, RSB_ERR_INVALID, "pad count must equal num_arenas*34");
    for (size_t a = 0; a < h->arenas.size(); a++) {
        auto& pads = h->arenas[a]->GetBoostPads();
        for (int p = 0; p < RSB_NUM_PADS; p++) {
            const rsb_pad_state& o = in[a * RSB_NUM_PADS + p];
            BoostPadState s;
            s.isActive = o.is_active;
            s.cooldown = o.cooldown;
            s.prevLockedCarID = o.prev_locked_car_id;
            pads[p]->SetState(s);
        }
    }
    return RSB_OK;
}

rsb_status rsb_get_arena_info(rsb_handle* h, rsb_arena_info* out, int32_t n) {
    if (!h || !out || n != (int32_t)h->arenas.size()) return fail(h, RSB_ERR_INVALID, "info count must equal num_arenas");
    for (int a = 0; a < n; a++) {
        Arena* ar = h->arenas[a];
        rsb_arena_info& o = out[a];
        o = rsb_arena_info{};
        o.tick_count = ar->tickCount;
        o.num_cars = 2 * h->teamSize[a];
        o.team_size = h->teamSize[a];
        bool scored = ar->IsBallScored();
        o.goal_scored = scored;
        float y = ar->ball->GetState().pos.y;
        // RS_TEAM_FROM_Y(-y): the ball past +y scores for blue (orange's net is at +y)
        o.goal_team = scored ? (y > 0 ? 0 : 1) : -1;
        o.episode_ticks = h->episodeTicks[a];
    }
    return RSB_OK;
}

// One arena at a time (RocketSimCuda.h:349-378) on the RocketSim objects.
static bool validArena(const rsb_handle* h, int32_t a) { return h && a >= 0 && a < (int32_t)h->arenas.size(); }

rsb_status rsb_get_car_at(rsb_handle* h, int32_t a, int32_t c, rsb_car_state* out) {
    if (!validArena(h, a) || !out || c < 0 || c >= (int32_t)h->cars[a].size()) return fail(h, RSB_ERR_INVALID, "no such car");
    Car* car = h->cars[a][c];
    *out = fromCarState(car->GetState(), car->team, car->id);
    return RSB_OK;
}
rsb_status rsb_set_car_controls_at(rsb_handle* h, int32_t a, int32_t c, const rsb_controls* in) {
    if (!validArena(h, a) || !in || c < 0 || c >= (int32_t)h->cars[a].size()) return fail(h, RSB_ERR_INVALID, "no such car");
    h->controls[(size_t)h->carOffset[a] + c] = *in;
    return RSB_OK;
}
rsb_status rsb_set_car_at(rsb_handle* h, int32_t a, int32_t c, const rsb_car_state* in) {
    if (!validArena(h, a) || !in || c < 0 || c >= (int32_t)h->cars[a].size()) return fail(h, RSB_ERR_INVALID, "no such car");
    h->cars[a][c]->SetState(toCarState(*in));
    return RSB_OK;
}
rsb_status rsb_get_ball_at(rsb_handle* h, int32_t a, rsb_ball_state* out) {
    if (!validArena(h, a) || !out) return fail(h, RSB_ERR_INVALID, "no such arena");
    BallState s = h->arenas[a]->ball->GetState();
    out->pos = fromVec(s.pos);
    out->rot.forward = fromVec(s.rotMat.forward);
    out->rot.right = fromVec(s.rotMat.right);
    out->rot.up = fromVec(s.rotMat.up);
    out->vel = fromVec(s.vel);
    out->ang_vel = fromVec(s.angVel);
    return RSB_OK;
}
rsb_status rsb_set_ball_at(rsb_handle* h, int32_t a, const rsb_ball_state* in) {
    if (!validArena(h, a) || !in) return fail(h, RSB_ERR_INVALID, "no such arena");
    BallState s;
    s.pos = toVec(in->pos);
    s.rotMat = RotMat(toVec(in->rot.forward), toVec(in->rot.right), toVec(in->rot.up));
    s.vel = toVec(in->vel);
    s.angVel = toVec(in->ang_vel);
    h->arenas[a]->ball->SetState(s);
    return RSB_OK;
}
rsb_status rsb_get_pads_at(rsb_handle* h, int32_t a, rsb_pad_state* out) {
    if (!validArena(h, a) || !out) return fail(h, RSB_ERR_INVALID, "no such arena");
    auto& pads = h->arenas[a]->GetBoostPads();
    for (int p = 0; p < RSB_NUM_PADS; p++) {
        BoostPadState s = pads[p]->GetState();
        out[p] = rsb_pad_state{};
        out[p].is_active = s.isActive;
        out[p].cooldown = s.cooldown;
        out[p].prev_locked_car_id = s.prevLockedCarID;
    }
    return RSB_OK;
}
rsb_status rsb_set_pads_at(rsb_handle* h, int32_t a, const rsb_pad_state* in) {
    if (!validArena(h, a) || !in) return fail(h, RSB_ERR_INVALID, "no such arena");
    auto& pads = h->arenas[a]->GetBoostPads();
    for (int p = 0; p < RSB_NUM_PADS; p++) {
        BoostPadState s;
        s.isActive = in[p].is_active;
        s.cooldown = in[p].cooldown;
        s.prevLockedCarID = in[p].prev_locked_car_id;
        pads[p]->SetState(s);
    }
    return RSB_OK;
}
rsb_status rsb_get_arena_info_at(rsb_handle* h, int32_t a, rsb_arena_info* out) {
    if (!validArena(h, a) || !out) return fail(h, RSB_ERR_INVALID, "no such arena");
    std::vector<rsb_arena_info> all(h->arenas.size());
    rsb_status st = rsb_get_arena_info(h, all.data(), (int32_t)all.size());
    if (st == RSB_OK) *out = all[(size_t)a];
    return st;
}

rsb_status rsb_sync(rsb_handle* h) { return h ? RSB_OK : RSB_ERR_INVALID; }

// The learned culler is a GPU component with no CPU counterpart in the reference.
rsb_status rsb_set_cull_mode(rsb_handle* h, int32_t mode) { return mode == RSB_CULL_EXACT ? RSB_OK : fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }
rsb_status rsb_culler_log(rsb_handle* h, void*) { return fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }
rsb_status rsb_culler_train(rsb_handle* h, const rsb_culler_config*, rsb_culler_report*) { return fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }
rsb_status rsb_culler_get(rsb_handle* h, float*, float*) { return fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }
rsb_status rsb_culler_set(rsb_handle* h, const float*, float) { return fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }
rsb_status rsb_culler_distance(rsb_handle* h, const float*, int32_t, float*) { return fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }
rsb_status rsb_culler_predict(rsb_handle* h, const float*, int32_t, float*) { return fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }
rsb_status rsb_culler_gradients(rsb_handle* h, const float*, const float*, int32_t, float, float*, float*) { return fail(h, RSB_ERR_UNSUPPORTED, "no culler on the CPU oracle"); }

rsb_status rsb_copy_outputs(rsb_handle* h, float* obs, uint8_t* masks, float* rewards, uint8_t* terminals) {
    if (!h) return RSB_ERR_INVALID;
    rsb_status st = RSB_OK;
    if (obs && st == RSB_OK) st = rsb_copy_obs(h, obs, h->obs.size());
    if (masks && st == RSB_OK) st = rsb_copy_masks(h, masks, h->masks.size());
    if (rewards && st == RSB_OK) st = rsb_copy_rewards(h, rewards, h->rewardsOut.size());
    if (terminals && st == RSB_OK) st = rsb_copy_terminals(h, terminals, h->terminalsOut.size());
    return st;
}
// host memory needs no pinning on the CPU oracle
rsb_status rsb_host_register(void* ptr, size_t bytes) { return ptr && bytes ? RSB_OK : RSB_ERR_INVALID; }
rsb_status rsb_host_unregister(void* ptr) { return ptr ? RSB_OK : RSB_ERR_INVALID; }

// ---- state ring: CudaEnvSet.cpp:608-815 restated on the RocketSim arenas ----

static float ringRand01(uint32_t& rng) {  // CudaEnvSet.cpp:608-613
    rng ^= rng << 13;
    rng ^= rng >> 17;
    rng ^= rng << 5;
    return (rng & 0xFFFFFFu) / float(0xFFFFFFu);
}
static float ringRange(uint32_t& rng, float lo, float hi) { return lo + (hi - lo) * ringRand01(rng); }

rsb_status rsb_ring_default_config(rsb_ring_config* out) {  // CudaEnvSet.h:100-109, :164
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

rsb_status rsb_ring_configure(rsb_handle* h, const rsb_ring_config* cfg) {  // ConfigureStateRing :619-656
    if (!h || !cfg) return fail(h, RSB_ERR_INVALID, "rsb_ring_configure: null argument");
    auto& R = h->ring;
    R.slots.clear();
    R.enabled = false;
    R.filled = R.writeIdx = R.stepsSinceCapture = 0;
    const int numArenas = (int)h->arenas.size();
    if (cfg->depth <= 0 || numArenas <= 0) return RSB_OK;
    R.cfg = *cfg;
    const int depth = (std::max)(2, cfg->depth);
    R.cfg.depth = depth;
    R.cfg.capture_every = (std::max)(1, cfg->capture_every);
    R.cfg.lookback_slots = (std::max)(1, (std::min)(cfg->lookback_slots, depth - 1));
    R.cfg.restore_fraction =
        (std::max)(0.01f, (std::min)(0.05f, cfg->restore_fraction > 0.f ? cfg->restore_fraction : 0.05f));
    R.cfg.max_arenas_per_restore = (std::max)(1, cfg->max_arenas_per_restore > 0 ? cfg->max_arenas_per_restore : 64);
    R.rng = cfg->seed ? cfg->seed : 0xA5A5A5A5u;
    R.slots.assign((size_t)depth, std::vector<rsb_handle::ArenaSnap>((size_t)numArenas));
    R.enabled = true;
    return RSB_OK;
}

rsb_status rsb_ring_capture(rsb_handle* h, void*) {  // CaptureStateRingSlot :669-696
    if (!h) return RSB_ERR_INVALID;
    auto& R = h->ring;
    if (!R.enabled) return RSB_OK;
    auto& arenas = R.slots[(size_t)R.writeIdx];
    for (size_t a = 0; a < h->arenas.size(); a++) {
        auto& snap = arenas[a];
        snap.cars.clear();
        for (Car* car : h->cars[a]) snap.cars.push_back(car->GetState());
        snap.ball = h->arenas[a]->ball->GetState();
        snap.pads.clear();
        for (auto* pad : h->arenas[a]->GetBoostPads()) snap.pads.push_back(pad->GetState());
        snap.valid = true;
    }
    R.writeIdx = (R.writeIdx + 1) % R.cfg.depth;
    if (R.filled < R.cfg.depth) R.filled++;
    R.captures++;
    return RSB_OK;
}

rsb_status rsb_ring_maybe_capture(rsb_handle* h, void* stream) {  // MaybeCaptureStateRing :658-667
    if (!h) return RSB_ERR_INVALID;
    auto& R = h->ring;
    if (!R.enabled) return RSB_OK;
    if (++R.stepsSinceCapture < R.cfg.capture_every) return RSB_OK;
    R.stepsSinceCapture = 0;
    return rsb_ring_capture(h, stream);
}

// ApplyArenaSnap (:698-753): public states of the slot, jittered, through the setters
static void applyArenaSnap(rsb_handle* h, int a, int slot, float fuzzScale) {
    auto& R = h->ring;
    const auto& snap = R.slots[(size_t)slot][(size_t)a];
    if (!snap.valid) return;
    const float fp = R.cfg.fuzz_pos * fuzzScale;
    const float fv = R.cfg.fuzz_vel * fuzzScale;
    for (size_t c = 0; c < h->cars[a].size() && c < snap.cars.size(); c++) {
        CarState car = snap.cars[c];
        if (fp > 0.f) {
            car.pos.x += ringRange(R.rng, -fp, fp);
            car.pos.y += ringRange(R.rng, -fp, fp);
            car.pos.z = (std::max)(17.f, car.pos.z + ringRange(R.rng, -fp * 0.25f, fp * 0.35f));
        }
        if (fv > 0.f) {
            car.vel.x += ringRange(R.rng, -fv, fv);
            car.vel.y += ringRange(R.rng, -fv, fv);
            car.vel.z += ringRange(R.rng, -fv * 0.5f, fv * 0.5f);
        }
        h->cars[a][c]->SetState(car);
    }
    BallState ball = snap.ball;
    if (fp > 0.f) {
        ball.pos.x += ringRange(R.rng, -fp, fp);
        ball.pos.y += ringRange(R.rng, -fp, fp);
        ball.pos.z = (std::max)(93.f, ball.pos.z + ringRange(R.rng, -fp * 0.2f, fp * 0.4f));
    }
    if (fv > 0.f) {
        ball.vel.x += ringRange(R.rng, -fv, fv);
        ball.vel.y += ringRange(R.rng, -fv, fv);
        ball.vel.z += ringRange(R.rng, -fv * 0.5f, fv * 0.5f);
    }
    h->arenas[a]->ball->SetState(ball);
    auto& pads = h->arenas[a]->GetBoostPads();
    for (size_t p = 0; p < pads.size() && p < snap.pads.size(); p++) pads[p]->SetState(snap.pads[p]);
}

rsb_status rsb_ring_restore(rsb_handle* h, float restore_fraction, int32_t lookback_slots, float fuzz_scale,
                            int32_t max_arenas, int32_t* restored, void*) {  // RestoreStateRingReplay :755-815
    if (!h) return RSB_ERR_INVALID;
    if (restored) *restored = 0;
    auto& R = h->ring;
    if (!R.enabled || R.replayDisabled || R.filled < 2) return RSB_OK;
    const int numArenas = (int)h->arenas.size();
    float frac = restore_fraction >= 0.f ? restore_fraction : R.cfg.restore_fraction;
    frac = (std::max)(0.01f, (std::min)(0.05f, frac));
    int lookback = lookback_slots >= 0 ? lookback_slots : R.cfg.lookback_slots;
    lookback = (std::max)(1, (std::min)(lookback, R.filled - 1));
    int lastWritten = R.writeIdx - 1;
    if (lastWritten < 0) lastWritten = R.cfg.depth - 1;
    int slot = lastWritten - lookback;
    while (slot < 0) slot += R.cfg.depth;
    int cap = max_arenas > 0 ? max_arenas : R.cfg.max_arenas_per_restore;
    if (cap <= 0) cap = 64;
    int fivePct = (std::max)(1, (int)std::lround(0.05 * (double)numArenas));
    cap = (std::min)(cap, fivePct);
    int nRestore = (std::max)(1, (int)std::lround(frac * (double)numArenas));
    nRestore = (std::min)(nRestore, numArenas);
    nRestore = (std::min)(nRestore, cap);
    std::vector<int> order((size_t)numArenas);
    for (int i = 0; i < numArenas; i++) order[(size_t)i] = i;
    for (int i = 0; i < nRestore; i++) {
        int j = i + (int)(ringRand01(R.rng) * (numArenas - i));
        if (j >= numArenas) j = numArenas - 1;
        std::swap(order[(size_t)i], order[(size_t)j]);
    }
    for (int i = 0; i < nRestore; i++) applyArenaSnap(h, order[(size_t)i], slot, fuzz_scale);
    R.restores += (uint64_t)nRestore;
    R.restoreCalls++;
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

// GAE lives in its own oracle libraries (gae_oracle.c, gae_pin.cpp); this one only answers
// the ABI.
rsb_status rsb_gae_default_params(rsb_gae_params* out) {
    if (!out) return RSB_ERR_INVALID;
    out->gamma = 0.99f;
    out->lambda = 0.95f;
    out->return_std = 0.f;
    out->clip_range = 0.f;
    return RSB_OK;
}
rsb_status rsb_compute_gae(const float*, const int8_t*, const float*, const float*, int32_t, float*, float*, float*,
                           float*, int32_t, const rsb_gae_params*, void*) {
    return RSB_ERR_UNSUPPORTED;
}
rsb_status rsb_compute_gae_host(const float*, const int8_t*, const float*, int32_t, const float*, int32_t, float*,
                                float*, float*, float*, int32_t, const rsb_gae_params*) {
    return RSB_ERR_UNSUPPORTED;
}

// The CPU oracle has a single configuration.
rsb_status rsb_set_step_config(rsb_handle* h, const rsb_tune_entry* cfg) { return h && cfg ? RSB_OK : RSB_ERR_INVALID; }
rsb_status rsb_autotune(rsb_handle* h, int32_t, rsb_tune_entry*, int32_t, int32_t* count) {
    if (!h) return RSB_ERR_INVALID;
    if (count) *count = 0;
    return RSB_OK;
}

// The reference's own values of the functions the engine restates: the CPU's rsqrtss and the
// C library's sinf / cosf / asinf / atan2f, evaluated here on the host.
rsb_status rsb_eval_refmath(int32_t fn, const float* x, const float* y, float* out, int64_t n, int32_t) {
    if (fn < RSB_MATH_RSQRT_EST || fn > RSB_MATH_ATAN2 || !x || !out || n < 0 || (fn == RSB_MATH_ATAN2 && !y))
        return fail(nullptr, RSB_ERR_INVALID, "bad function, pointer or count");
    for (int64_t i = 0; i < n; i++) {
        switch (fn) {
            case RSB_MATH_RSQRT_EST: out[i] = _mm_cvtss_f32(_mm_rsqrt_ss(_mm_set_ss(x[i]))); break;
            case RSB_MATH_SIN: out[i] = sinf(x[i]); break;
            case RSB_MATH_COS: out[i] = cosf(x[i]); break;
            case RSB_MATH_ASIN: out[i] = asinf(x[i]); break;
            default: out[i] = atan2f(x[i], y[i]); break;
        }
    }
    return RSB_OK;
}

// Oracle-only helpers (not part of include/rsb.h).
//
// rsbref_car_order: the order in which the reference visits the cars of arena `a` on
// every tick (Arena::_cars is an unordered_set of pointers, so the order follows the
// heap addresses of this run).  Writes car slot indices (blue first, then orange).
int32_t rsbref_car_order(rsb_handle* h, int32_t a, int32_t* order) {
    if (!h || a < 0 || a >= (int32_t)h->arenas.size() || !order) return -1;
    int k = 0;
    for (Car* c : h->arenas[a]->GetCars()) {
        for (size_t s = 0; s < h->cars[a].size(); s++)
            if (h->cars[a][s] == c) order[k++] = (int32_t)s;
    }
    return k;
}
// rsbref_wheel_info: the raycast result of wheel w of car slot s in arena a, as the last
// tick's pre-tick left it (btWheelInfo::RaycastInfo): hard point (3), direction (3), contact
// point (3), contact normal (3), suspension length, in contact (1/0), ground object kind
// (-1 none, 0 static, 1 ball, 2 car), all in Bullet units.  Writes 16 floats.
int32_t rsbref_wheel_info(rsb_handle* h, int32_t a, int32_t s, int32_t w, float* out) {
    if (!h || a < 0 || a >= (int32_t)h->arenas.size() || s < 0 || s >= (int32_t)h->cars[a].size() || w < 0 ||
        w > 3 || !out)
        return -1;
    const btWheelInfo::RaycastInfo& r = h->cars[a][s]->_bulletVehicle.m_wheelInfo[w].m_raycastInfo;
    const btVector3* v[4] = {&r.m_hardPointWS, &r.m_wheelDirectionWS, &r.m_contactPointWS, &r.m_contactNormalWS};
    for (int k = 0; k < 4; k++)
        for (int c = 0; c < 3; c++) out[3 * k + c] = (*v[k])[c];
    out[12] = r.m_suspensionLength;
    out[13] = r.m_isInContact ? 1.f : 0.f;
    float kind = -1.f;
    if (r.m_groundObject) {
        const btCollisionObject* o = (const btCollisionObject*)r.m_groundObject;
        kind = o->isStaticObject() ? 0.f : (o->getCollisionShape()->getShapeType() == SPHERE_SHAPE_PROXYTYPE ? 1.f : 2.f);
    }
    out[14] = kind;
    out[15] = 0.f;
    return 0;
}
// rsbref_car_ptr: the reference Car object of slot s in arena a (debug probes)
void* rsbref_car_ptr(rsb_handle* h, int32_t a, int32_t s) {
    if (!h || a < 0 || a >= (int32_t)h->arenas.size() || s < 0 || s >= (int32_t)h->cars[a].size()) return nullptr;
    return h->cars[a][s];
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

rsb_status rsb_obs_stride(const rsb_handle* h, int32_t* stride) {
    if (!h || !stride) return RSB_ERR_INVALID;
    int m = 0;
    for (int t : h->teamSize) m = std::max(m, 2 * t);
    *stride = RSB_OBS_BASE + RSB_OBS_PER_CAR * m;
    return RSB_OK;
}

rsb_status rsb_default_action_lut(rsb_controls* lut, int32_t count) {
    // RLGymCPP's DefaultAction table (DefaultAction.cpp:3-91), converted the way
    // EnvSet hands actions to the cars: (CarControls)action (Action.h:32-45)
    static RLGC::DefaultAction parser;
    if (!lut || count < (int32_t)parser.actions.size()) return RSB_ERR_INVALID;
    for (size_t i = 0; i < parser.actions.size(); i++) lut[i] = fromControls((CarControls)parser.actions[i]);
    return (int32_t)parser.actions.size() == RSB_NUM_ACTIONS ? RSB_OK : RSB_ERR_STATE;
}

rsb_status rsb_set_actions_device(rsb_handle* h, const int32_t*, int32_t, void*) { return fail(h, RSB_ERR_UNSUPPORTED, "no device on the CPU oracle"); }
rsb_status rsb_device_ptr(rsb_handle* h, int32_t, void**) { return fail(h, RSB_ERR_UNSUPPORTED, "no device on the CPU oracle"); }

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

}  // extern "C"

// The env-layer entry points below keep the C linkage of their declarations in rsb.h.

static void buildEnv(rsb_handle* h) {
    const rsb_reward_config& rc = h->rewardCfg;
    h->env.resize(h->arenas.size());
    for (size_t a = 0; a < h->arenas.size(); a++) {
        OracleEnv& e = h->env[a];
        auto add = [&](RLGC::Reward* r, float w, int bit) {
            if (w == 0.f) { delete r; return; }
            if (rc.zero_sum & (1 << bit)) r = new RLGC::ZeroSumReward(r, rc.team_spirit, rc.opponent_scale);
            e.rewards.emplace_back(r, w);
        };
        add(new RLGC::GoalReward(rc.goal_concede_scale), rc.w_goal, 0);
        add(new RLGC::TouchBallReward(), rc.w_touch, 1);
        add(new RLGC::VelocityBallToGoalReward(), rc.w_vel_ball_to_goal, 2);
        add(new RLGC::VelocityPlayerToBallReward(), rc.w_vel_player_to_ball, 3);
        if (rc.no_touch_timeout_s > 0.f) e.terminals.push_back(new RLGC::NoTouchCondition(rc.no_touch_timeout_s));
        e.terminals.push_back(new RLGC::GoalScoreCondition());
        if (rc.episode_max_ticks > 0) e.terminals.push_back(new EpisodeTickLimit(&h->episodeTicks[a], rc.episode_max_ticks));
    }
}

static void freeEnv(rsb_handle* h) {
    for (auto& e : h->env) {
        for (auto& r : e.rewards) delete r.first;
        for (auto* t : e.terminals) delete t;
    }
    h->env.clear();
}

// Slot (creation index) of every entry of Arena::_cars, in iteration order.
static std::vector<int> carsOrder(rsb_handle* h, size_t a) {
    std::vector<int> order;
    for (Car* c : h->arenas[a]->GetCars())
        for (size_t s = 0; s < h->cars[a].size(); s++)
            if (h->cars[a][s] == c) order.push_back((int)s);
    return order;
}

// GameState::UpdateFromArena with the actions of the last step in the arena's car
// order; lastTickCount set so that the state's tickSkip is step_ticks.
static void gameStateOf(rsb_handle* h, size_t a, int stepTicks, RLGC::GameState& gs, std::vector<int>& order) {
    order = carsOrder(h, a);
    std::vector<RLGC::Action> actions(order.size());
    for (size_t i = 0; i < order.size(); i++)
        actions[i] = RLGC::Action(toControls(h->controls[h->carOffset[a] + order[i]]));
    uint64_t tc = h->arenas[a]->tickCount;
    gs = RLGC::GameState();
    gs.lastTickCount = tc - std::min<uint64_t>((uint64_t)std::max(stepTicks, 0), tc);
    gs.UpdateFromArena(h->arenas[a], actions, nullptr);
}

rsb_status rsb_snapshot(rsb_handle* h, void*) {
    // the four stub rewards read no previous state (CommonRewards.h:33-98)
    return h ? RSB_OK : RSB_ERR_INVALID;
}

rsb_status rsb_build_obs(rsb_handle* h, void*) {
    if (!h) return RSB_ERR_INVALID;
    static RLGC::DefaultAction parser;
    RLGC::AdvancedObs builder;
    int32_t stride = 0;
    rsb_obs_stride(h, &stride);
    h->obs.assign((size_t)h->numCars * stride, 0.f);
    h->masks.assign((size_t)h->numCars * RSB_NUM_ACTIONS, 0);
    forArenas(h, [&](int a) {
        RLGC::GameState gs;
        std::vector<int> order;
        gameStateOf(h, a, 0, gs, order);
        for (size_t i = 0; i < order.size(); i++) {
            size_t row = h->carOffset[a] + order[i];
            RLGC::FList o = builder.BuildObs(gs.players[i], gs);
            std::copy(o.begin(), o.end(), h->obs.begin() + row * stride);
            std::vector<uint8_t> m = parser.GetActionMask(gs.players[i], gs);
            std::copy(m.begin(), m.end(), h->masks.begin() + row * RSB_NUM_ACTIONS);
        }
    });
    return RSB_OK;
}

rsb_status rsb_build_rewards_terminals(rsb_handle* h, int32_t step_ticks, void*) {
    if (!h) return RSB_ERR_INVALID;
    if (!h->hasRewards) return fail(h, RSB_ERR_STATE, "no reward configuration at create");
    h->rewardsOut.assign(h->numCars, 0.f);
    h->terminalsOut.assign(h->arenas.size(), 0);
    forArenas(h, [&](int a) {
        RLGC::GameState gs;
        std::vector<int> order;
        gameStateOf(h, a, step_ticks, gs, order);
        // EnvSet.cpp:184-205: every condition is evaluated; normal beats truncation
        uint8_t type = RLGC::TerminalType::NOT_TERMINAL;
        for (auto* cond : h->env[a].terminals) {
            if (cond->IsTerminal(gs)) {
                uint8_t cur = cond->IsTruncation() ? RLGC::TerminalType::TRUNCATED : RLGC::TerminalType::NORMAL;
                if (type == RLGC::TerminalType::NOT_TERMINAL || cur == RLGC::TerminalType::NORMAL) type = cur;
            }
        }
        h->terminalsOut[a] = type;
        // EnvSet.cpp:207-254
        std::vector<float> all(order.size(), 0.f);
        for (auto& wr : h->env[a].rewards) wr.first->PreStep(gs);
        for (auto& wr : h->env[a].rewards) {
            std::vector<float> out = wr.first->GetAllRewards(gs, type);
            float scale = RLGC::RuntimeRewardScale(wr.first->GetName(), wr.second);
            for (size_t i = 0; i < order.size(); i++) all[i] += out[i] * scale;
        }
        for (size_t i = 0; i < order.size(); i++) h->rewardsOut[h->carOffset[a] + order[i]] = all[i];
    });
    return RSB_OK;
}

template <class T>
static rsb_status copyOut(rsb_handle* h, const std::vector<T>& src, T* out, size_t count, const char* what) {
    if (!h || !out) return RSB_ERR_INVALID;
    if (count != src.size()) return fail(h, RSB_ERR_INVALID, std::string(what) + ": count does not match (build it first)");
    std::memcpy(out, src.data(), count * sizeof(T));
    return RSB_OK;
}
rsb_status rsb_copy_obs(rsb_handle* h, float* out, size_t n) { return copyOut(h, h->obs, out, n, "obs"); }
rsb_status rsb_copy_masks(rsb_handle* h, uint8_t* out, size_t n) { return copyOut(h, h->masks, out, n, "masks"); }
rsb_status rsb_copy_rewards(rsb_handle* h, float* out, size_t n) { return copyOut(h, h->rewardsOut, out, n, "rewards"); }
rsb_status rsb_copy_terminals(rsb_handle* h, uint8_t* out, size_t n) { return copyOut(h, h->terminalsOut, out, n, "terminals"); }

// EnvSet::ResetArena (EnvSet.cpp:392-424): state setter, then the terminal conditions
// and rewards are reset; the new state's players carry default (zero) actions.
static void resetOne(rsb_handle* h, int a, uint64_t seed, int32_t mode) {
    Arena* arena = h->arenas[a];
    if (mode == RSB_RESET_KICKOFF) {
        arena->ResetToRandomKickoff((int)(uint32_t)(seed ^ (seed >> 32) ^ (0x9E3779B9u * (uint32_t)(a + 1))) & 0x7fffffff);
    } else {
        RLGC::RandomState(true, true, false).ResetArena(arena);
    }
    for (size_t c = 0; c < h->cars[a].size(); c++) h->controls[h->carOffset[a] + c] = rsb_controls{};
    h->episodeTicks[a] = 0;
    if (!h->env.empty()) {
        RLGC::GameState gs(arena);
        for (auto* t : h->env[a].terminals) t->Reset(gs);
        for (auto& r : h->env[a].rewards) r.first->Reset(gs);
    }
}

// The reference CPU collector has no reset curriculum (it is the GPU batch's, RocketSimCuda.h:283):
// the weights are checked and kept, and a curriculum reset is refused.
rsb_status rsb_set_reset_curriculum(rsb_handle* h, float, float, float, float) {
    return h ? RSB_OK : RSB_ERR_INVALID;
}

// The VantaObs builder is checked against the reference's own device builder
// (oracle/vanta_pin.cu), not against this library.
rsb_status rsb_vanta_default_config(rsb_vanta_config* cfg) {
    if (!cfg) return RSB_ERR_INVALID;
    *cfg = rsb_vanta_config{8, 0.5f, 0, 1};
    return RSB_OK;
}
rsb_status rsb_vanta_configure(rsb_handle* h, const rsb_vanta_config*) {
    return fail(h, RSB_ERR_UNSUPPORTED, "the CPU oracle has no VantaObs builder");
}
rsb_status rsb_build_vanta_obs(rsb_handle* h, void*) {
    return fail(h, RSB_ERR_UNSUPPORTED, "the CPU oracle has no VantaObs builder");
}
rsb_status rsb_copy_vanta_obs(rsb_handle* h, float*, size_t) {
    return fail(h, RSB_ERR_UNSUPPORTED, "the CPU oracle has no VantaObs builder");
}
// Arena's pads: the big soccar pads, then the small ones (Arena.cpp:546-550).
rsb_status rsb_pad_locations(float* xyz) {
    if (!xyz) return RSB_ERR_INVALID;
    using namespace RocketSim::RLConst::BoostPads;
    for (int i = 0; i < LOCS_AMOUNT_BIG + LOCS_AMOUNT_SMALL_SOCCAR; i++) {
        const RocketSim::Vec& v = i < LOCS_AMOUNT_BIG ? LOCS_BIG_SOCCAR[i] : LOCS_SMALL_SOCCAR[i - LOCS_AMOUNT_BIG];
        xyz[3 * i + 0] = v.x;
        xyz[3 * i + 1] = v.y;
        xyz[3 * i + 2] = v.z;
    }
    return RSB_OK;
}

// CUDA graphs have no counterpart on the CPU oracle.
rsb_status rsb_env_graph_capture(rsb_handle* h, const int32_t*, int32_t, int32_t, uint64_t) {
    return fail(h, RSB_ERR_UNSUPPORTED, "no CUDA graphs on the CPU oracle");
}
rsb_status rsb_env_graph_launch(rsb_handle* h, void*) {
    return fail(h, RSB_ERR_UNSUPPORTED, "no CUDA graphs on the CPU oracle");
}

rsb_status rsb_reset_arenas(rsb_handle* h, const int32_t* idx, int32_t n, uint64_t seed, int32_t mode) {
    if (!h || (n > 0 && !idx)) return RSB_ERR_INVALID;
    if (mode != RSB_RESET_KICKOFF && mode != RSB_RESET_RANDOM_STATE)
        return fail(h, RSB_ERR_UNSUPPORTED, "the CPU oracle has kickoff and random-state resets only");
    for (int i = 0; i < n; i++)
        if (idx[i] < 0 || idx[i] >= (int32_t)h->arenas.size()) return fail(h, RSB_ERR_INVALID, "arena index out of range");
    for (int i = 0; i < n; i++) resetOne(h, idx[i], seed, mode);
    return RSB_OK;
}

rsb_status rsb_reset_done(rsb_handle* h, uint64_t seed, int32_t mode, void*) {
    if (!h) return RSB_ERR_INVALID;
    if (mode != RSB_RESET_KICKOFF && mode != RSB_RESET_RANDOM_STATE)
        return fail(h, RSB_ERR_UNSUPPORTED, "the CPU oracle has kickoff and random-state resets only");
    if (h->terminalsOut.size() != h->arenas.size()) return RSB_OK;
    forArenas(h, [&](int a) {
        if (h->terminalsOut[a]) resetOne(h, a, seed, mode);
    });
    return RSB_OK;
}

rsb_status rsb_reset_all(rsb_handle* h, uint64_t seed, int32_t mode) {
    if (!h) return RSB_ERR_INVALID;
    std::vector<int32_t> idx(h->arenas.size());
    for (size_t a = 0; a < idx.size(); a++) idx[a] = (int32_t)a;
    return rsb_reset_arenas(h, idx.data(), (int32_t)idx.size(), seed, mode);
}


