// Host-side set-up shared by the CUDA engine (rsb_engine.cu) and the host harness that runs
// the same per-arena code on the CPU for debugging: world parameters from the mutator
// settings, the creation-time records of every arena, and the conversions between the C
// ABI's state structs and the word-plane records.
#pragma once
#include <cmath>
#include <vector>

#include "rsb.h"
#include "phys/engine_core.h"

namespace rsb {

// Arena / Car / Ball constants evaluated on the host with the reference's operation order
// (Arena::Arena, Ball::_BulletSetup, Car::_BulletSetup, BoostPadGrid::Add).
inline void computeParams(const rsb_mutators& m, WorldParams& P) {
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

    // ---- car: Octane hitbox and wheels (Car::_BulletSetup)
    CarParams& C = P.car;
    const float U = kUuToBt;
    V3 half = (V3{OCT_HITBOX_X, OCT_HITBOX_Y, OCT_HITBOX_Z} * U) * (1.f / 2.f);
    const float margin0 = 0.04f;  // CONVEX_DISTANCE_MARGIN
    V3 implicit = half - V3{margin0, margin0, margin0};
    int minAxis = half.x < half.y ? (half.x < half.z ? 0 : 2) : (half.y < half.z ? 1 : 2);
    float safe = 0.1f * half[minAxis];
    float margin = margin0;
    // setSafeMargin reaches btConvexInternalShape::setMargin, which RocketSim's Bullet makes
    // non-virtual (btConvexInternalShape.h:88): the margin shrinks, the implicit half
    // extents stay at half - 0.04
    if (safe < margin0) margin = safe;
    C.boxHe = implicit;
    C.boxMargin = margin;
    C.boxHeM = implicit + V3{margin, margin, margin};
    C.childOff = V3{OCT_HITBOX_OFF_X, OCT_HITBOX_OFF_Y, OCT_HITBOX_OFF_Z} * U;
    transformAabbHalf(C.boxHe, C.boxMargin, Xf{m3identity(), C.childOff}, C.cmpMin, C.cmpMax);
    {
        V3 mn, mx;
        transformAabb(C.cmpMin, C.cmpMax, 0.f, xfIdentity(), mn, mx);
        float radius = length(mx - mn) * 0.5f;
        V3 center = (mn + mx) * 0.5f;
        C.cbt = (radius + length(center)) * 0.02f;
    }
    // RocketSim builds every car with RLConst::CAR_MASS_BT (Car::_BulletSetup, Car.cpp:206-209):
    // MutatorConfig::carMass set before the cars exist never reaches them, and the reference
    // batch simulator uses its constant car mass throughout (CarPhysics.cuh:48, Collision.cuh:506)
    const float mass = CAR_MASS_BT;
    (void)m.car_mass;
    C.invMass = 1.f / mass;
    C.mass = 1.f / C.invMass;
    {
        V3 h = C.boxHeM;
        float lx = 2.f * h.x, ly = 2.f * h.y, lz = 2.f * h.z;
        V3 inertia{mass / 12.f * (ly * ly + lz * lz), mass / 12.f * (lx * lx + lz * lz), mass / 12.f * (lx * lx + ly * ly)};
        C.invInertiaLocal = V3{1.f / inertia.x, 1.f / inertia.y, 1.f / inertia.z};
    }
    C.grav = P.gravity * (1.f / C.invMass);
    C.susTravel = ((MAX_SUSPENSION_TRAVEL * U) * 100) / 100;
    for (int i = 0; i < 4; i++) {
        bool front = i < 2, left = (i % 2) != 0;
        float radius = front ? OCT_FRONT_RAD : OCT_BACK_RAD;
        V3 off = front ? V3{OCT_FRONT_OFF_X, OCT_FRONT_OFF_Y, OCT_FRONT_OFF_Z} : V3{OCT_BACK_OFF_X, OCT_BACK_OFF_Y, OCT_BACK_OFF_Z};
        if (left) off.y *= -1;
        float rest = (front ? OCT_FRONT_SUS_REST : OCT_BACK_SUS_REST) - MAX_SUSPENSION_TRAVEL;
        C.wheelConn[i] = off * U;
        C.susRest[i] = rest * U;
        C.wheelRadius[i] = radius * U;
        C.rayLen[i] = ((C.susRest[i] + C.susTravel) + C.wheelRadius[i]) - SUSPENSION_SUBTRACTION;
        C.pushThresh[i] = (C.susRest[i] + C.wheelRadius[i]) - SUSPENSION_SUBTRACTION;
        C.susForceScale[i] = front ? SUSPENSION_FORCE_SCALE_FRONT : SUSPENSION_FORCE_SCALE_BACK;
    }
    C.dodgeDeadzone = OCT_DODGE_DEADZONE;
    C.flipZDamp = powf(1 - FLIP_Z_DAMP_120, P.dt / (1 / 120.f));
    C.jumpAccel = m.jump_accel;
    C.jumpImmediateForce = m.jump_immediate_force;
    C.boostAccelGround = m.boost_accel_ground;
    C.boostAccelAir = m.boost_accel_air;
    C.boostUsedPerSecond = m.boost_used_per_second;
    C.respawnDelay = m.respawn_delay;
    C.bumpCooldown = m.bump_cooldown_time;
    C.padCooldownBig = m.boost_pad_cooldown_big;
    C.padCooldownSmall = m.boost_pad_cooldown_small;
    C.spawnBoost = m.car_spawn_boost_amount;
    C.ballHitExtraScale = m.ball_hit_extra_force_scale;
    C.bumpForceScale = m.bump_force_scale;
    C.worldFriction = m.car_world_friction;
    C.worldRestitution = m.car_world_restitution;
    C.unlimitedFlips = m.unlimited_flips;
    C.unlimitedDoubleJumps = m.unlimited_double_jumps;
    C.demoMode = m.demo_mode;
    C.teamDemos = m.enable_team_demos;

    // BoostPadGrid::Add (BoostPadGrid.cpp:26-40)
    for (int i = 0; i < 80; i++) P.padGrid[i] = -1;
    for (int p = 0; p < NUM_PADS; p++) {
        int ix = (int)(PAD_LOCS_HOST[p].x / 1024.f + 4.f);
        int iy = (int)(PAD_LOCS_HOST[p].y / 1024.f + 5.f);
        P.padGrid[ix * 10 + iy] = (int8_t)p;
    }
}

inline void defaultMutators(rsb_mutators* m) {
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
}

// The collector's 90-entry discrete action table (RLGymCPP DefaultAction.cpp:3-60): 24
// ground actions (throttle x steer x boost x handbrake, boosting only at full throttle,
// yaw follows steer), then 66 aerial ones (pitch x yaw x roll x jump x boost; jumps
// without yaw; throttle follows boost; handbrake on directional jumps).
inline int defaultActionLut(rsb_controls* out, int cap) {
    const float RB[2] = {0, 1}, RF[3] = {-1, 0, 1};
    int n = 0;
    auto put = [&](float throttle, float steer, float pitch, float yaw, float roll, float jump, float boost, float hb) {
        if (n < cap) {
            rsb_controls& c = out[n];
            c = rsb_controls{};
            c.throttle = throttle; c.steer = steer; c.pitch = pitch; c.yaw = yaw; c.roll = roll;
            c.jump = jump != 0; c.boost = boost != 0; c.handbrake = hb != 0;
        }
        n++;
    };
    for (float throttle : RF)
        for (float steer : RF)
            for (float boost : RB)
                for (float handbrake : RB) {
                    if (boost == 1 && throttle != 1) continue;
                    put(throttle, steer, 0, steer, 0, 0, boost, handbrake);
                }
    for (float pitch : RF)
        for (float yaw : RF)
            for (float roll : RF)
                for (float jump : RB)
                    for (float boost : RB) {
                        if (jump == 1 && yaw != 0) continue;
                        if (pitch == roll && roll == jump && jump == 0) continue;
                        float handbrake = (jump == 1) && (pitch != 0 || yaw != 0 || roll != 0);
                        put(boost, yaw, pitch, yaw, roll, jump, boost, handbrake);
                    }
    return n;
}

inline void cellOf(const ArenaStatic& S, V3 mn, int32_t& cell, int32_t& ci, int32_t& cj, int32_t& ck) {
    int i, j, k;
    bpCellIndices(S.bp, mn, i, j, k);
    ci = i;
    cj = j;
    ck = k;
    cell = i * S.bp.cellsY * S.bp.cellsZ + j * S.bp.cellsZ + k;
}

// RocketSim RotMat holds forward, right, up as the basis columns
RSB_HD M3 basisFromRot(const rsb_rotmat& r) {
    return m3(r.forward.x, r.right.x, r.up.x, r.forward.y, r.right.y, r.up.y, r.forward.z, r.right.z, r.up.z);
}
RSB_HD rsb_rotmat rotFromBasis(const float* rot) {
    rsb_rotmat r;
    r.forward = rsb_vec3{rot[0], rot[3], rot[6]};
    r.right = rsb_vec3{rot[1], rot[4], rot[7]};
    r.up = rsb_vec3{rot[2], rot[5], rot[8]};
    return r;
}
RSB_HD void basisToFloats(const M3& b, float* rot) {
    for (int i = 0; i < 3; i++) {
        rot[3 * i + 0] = b.r[i].x;
        rot[3 * i + 1] = b.r[i].y;
        rot[3 * i + 2] = b.r[i].z;
    }
}

// RLGymCPP's boost-pad order (CommonValues.h:48-84), used by its GameState and obs.
constexpr float RLGYM_PAD_XY[NUM_PADS][2] = {
    {0.f, -4240.f}, {-1792.f, -4184.f}, {1792.f, -4184.f}, {-3072.f, -4096.f}, {3072.f, -4096.f},
    {-940.f, -3308.f}, {940.f, -3308.f}, {0.f, -2816.f}, {-3584.f, -2484.f}, {3584.f, -2484.f},
    {-1788.f, -2300.f}, {1788.f, -2300.f}, {-2048.f, -1036.f}, {0.f, -1024.f}, {2048.f, -1036.f},
    {-3584.f, 0.f}, {-1024.f, 0.f}, {1024.f, 0.f}, {3584.f, 0.f}, {-2048.f, 1036.f},
    {0.f, 1024.f}, {2048.f, 1036.f}, {-1788.f, 2300.f}, {1788.f, 2300.f}, {-3584.f, 2484.f},
    {3584.f, 2484.f}, {0.f, 2816.f}, {-940.f, 3310.f}, {940.f, 3308.f}, {-3072.f, 4096.f},
    {3072.f, 4096.f}, {-1792.f, 4184.f}, {1792.f, 4184.f}, {0.f, 4240.f}};

// Kickoff spawns of blue (RLConst.h:297-303: x, y, yaw as float).
constexpr double kPi_d = 3.14159265358979323846;

// Tables of the env kernels: the pad-order map of _BuildBoostPadIndexMap
// (GameState.cpp:10-47, a 2D match within sqrt(10) uu), DefaultAction's four masks
// (DefaultAction.cpp:62-90, over the default 90-entry table), and the kickoff bases
// Angle(yaw, 0, 0).ToRotMat() with the orange yaw computed as `yaw += M_PI` on a float.
// Returns false when a pad cannot be matched.
template <class Tables>
inline bool buildEnvTables(Tables& T) {
    T = Tables{};
    for (int i = 0; i < NUM_PADS; i++) {
        int found = -1;
        for (int j = 0; j < NUM_PADS && found < 0; j++) {
            float dx = PAD_LOCS_HOST[j].x - RLGYM_PAD_XY[i][0], dy = PAD_LOCS_HOST[j].y - RLGYM_PAD_XY[i][1];
            if (dx * dx + dy * dy < 10) found = j;
        }
        if (found < 0) return false;
        T.padMap[i] = found;
    }
    rsb_controls lut[RSB_NUM_ACTIONS];
    int n = defaultActionLut(lut, RSB_NUM_ACTIONS);
    const int numGround = 24;
    for (int i = 0; i < n; i++) {
        const rsb_controls& c = lut[i];
        auto set = [&](uint32_t* m) { m[i >> 5] |= 1u << (i & 31); };
        if (c.jump) set(T.jump);
        if (c.boost) set(T.boost);
        if (i < numGround) set(T.ground);
        if (i > numGround && !c.jump) set(T.air);
        if (i < numGround && c.throttle == (float)c.boost && (float)(c.yaw != 0) == (float)c.handbrake) set(T.air);
    }
    const float yawBlue[NUM_KICKOFF_SPAWNS] = {(float)(kPi_d / 4 * 1), (float)(kPi_d / 4 * 3), (float)(kPi_d / 4 * 2),
                                               (float)(kPi_d / 4 * 2), (float)(kPi_d / 4 * 2)};
    const float xs[NUM_KICKOFF_SPAWNS] = {-2048, 2048, -256, 256, 0}, ys[NUM_KICKOFF_SPAWNS] = {-2560, -2560, -3840, -3840, -4608};
    for (int k = 0; k < NUM_KICKOFF_SPAWNS; k++) {
        T.kickX[k] = xs[k];
        T.kickY[k] = ys[k];
        for (int team = 0; team < 2; team++) {
            float yaw = yawBlue[k];
            if (team) yaw = (float)((double)yaw + kPi_d);
            M3 r = m3fromEulerZYX(-0.f, -0.f, yaw);
            basisToFloats(r, T.kickRot[team][k]);
        }
    }
    return true;
}

// Records of a freshly created arena (Arena::Arena + Arena::AddCar): ball at rest at the
// kickoff height, cars placed at respawn locations, pads active, and the broadphase
// registrations of the creation transforms (ball first, then cars in creation order).
struct HostRecords {
    std::vector<uint32_t> ball, car, pad, arena;
};

inline void initRecords(const ArenaStatic& S, const WorldParams& P, const std::vector<int32_t>& teamSize, HostRecords& R) {
    const size_t N = teamSize.size();
    R.ball.assign((size_t)W_BALL * N, 0);
    R.car.assign((size_t)W_CAR * MAX_CARS * N, 0);
    R.pad.assign((size_t)W_PAD * NUM_PADS * N, 0);
    R.arena.assign((size_t)W_ARENA * N, 0);
    BallP bp{};
    Xf x{m3identity(), V3{0, 0, BALL_REST_Z} * kUuToBt};
    xfToP(x, bp.pos, bp.rot);
    {
        V3 mn, mx;
        ballAabb(P, Xf{m3identity(), V3{0, 0, P.ballRadius}}, mn, mx);
        cellOf(S, mn, bp.cell, bp.ci, bp.cj, bp.ck);
    }
    bp.regStamp = 0;
    ArenaP ap{};
    ap.goalTeam = -1;
    PadP pp{};
    pp.bits = 1;
    // the car proxies are created at the identity transform, before the first placement
    V3 cmn, cmx;
    carCompoundAabb(P.car, xfIdentity(), cmn, cmx);
    for (size_t a = 0; a < N; a++) {
        storePlanes(bp, R.ball.data(), (int)a, (int)N);
        storePlanes(ap, R.arena.data(), (int)a, (int)N);
        for (int p = 0; p < NUM_PADS; p++) storePlanes(pp, R.pad.data(), (int)(p * N + a), (int)(N * NUM_PADS));
        int nc = 2 * teamSize[a];
        for (int s = 0; s < nc; s++) {
            bool orange = s >= teamSize[a];
            CarP c{};
            // Car::Respawn placement: respawn location s % 4, mirrored for orange
            const float xs[4] = {-2304.f, -2688.f, 2304.f, 2688.f};
            V3 pos{xs[s % 4], -4608.f * (orange ? -1.f : 1.f), CAR_RESPAWN_Z};
            float yaw = (float)(3.14159265358979323846 / 2 + (orange ? 3.14159265358979323846 : 0.0));
            M3 rot = m3fromEulerZYX(-0.f, -0.f, yaw);
            Xf cx{rot, pos * kUuToBt};
            xfToP(cx, c.pos, c.rot);
            basisToFloats(rot, c.rotMat);
            c.boost = P.car.spawnBoost;
            c.flags = CF_ON_GROUND | (orange ? CF_TEAM_ORANGE : 0u);
            c.ballHitTick[0] = c.ballHitTick[1] = 0xffffffffu;
            c.ballHitExtraTick[0] = c.ballHitExtraTick[1] = 0xffffffffu;
            cellOf(S, cmn, c.cell, c.ci, c.cj, c.ck);
            c.regStamp = (uint32_t)(1 + s);
            storePlanes(c, R.car.data(), (int)(s * N + a), (int)(MAX_CARS * N));
        }
    }
}

RSB_HD rsb_controls ctlFromRecord(const CarP& p) {
    rsb_controls r{};
    r.throttle = p.lastCtl[0];
    r.steer = p.lastCtl[1];
    r.pitch = p.lastCtl[2];
    r.yaw = p.lastCtl[3];
    r.roll = p.lastCtl[4];
    r.jump = (p.lastCtlBits & 1u) ? 1 : 0;
    r.boost = (p.lastCtlBits & 2u) ? 1 : 0;
    r.handbrake = (p.lastCtlBits & 4u) ? 1 : 0;
    return r;
}

// Car::GetState
RSB_HD rsb_car_state carStateOf(const CarP& p, uint32_t id) {
    rsb_car_state o{};
    V3 pos = V3{p.pos[0], p.pos[1], p.pos[2]} * kBtToUu;
    V3 vel = V3{p.lin[0], p.lin[1], p.lin[2]} * kBtToUu;
    o.pos = rsb_vec3{pos.x, pos.y, pos.z};
    o.rot = rotFromBasis(p.rotMat);
    o.vel = rsb_vec3{vel.x, vel.y, vel.z};
    o.ang_vel = rsb_vec3{p.ang[0], p.ang[1], p.ang[2]};
    o.boost = p.boost;
    o.time_spent_boosting = p.timeSpentBoosting;
    o.jump_time = p.jumpTime;
    o.flip_time = p.flipTime;
    o.air_time = p.airTime;
    o.air_time_since_jump = p.airTimeSinceJump;
    o.supersonic_time = p.supersonicTime;
    o.handbrake_val = p.handbrakeVal;
    o.auto_flip_timer = p.autoFlipTimer;
    o.auto_flip_torque_scale = p.autoFlipTorqueScale;
    o.demo_respawn_timer = p.demoRespawnTimer;
    o.car_contact_cooldown = p.carContactCooldown;
    o.flip_rel_torque = rsb_vec3{p.flipRelTorque[0], p.flipRelTorque[1], p.flipRelTorque[2]};
    o.world_contact_normal = rsb_vec3{p.worldContactNormal[0], p.worldContactNormal[1], p.worldContactNormal[2]};
    o.car_contact_other_id = p.carContactOtherId;
    uint32_t f = p.flags;
    o.is_on_ground = (f & CF_ON_GROUND) != 0;
    o.has_jumped = (f & CF_HAS_JUMPED) != 0;
    o.has_double_jumped = (f & CF_HAS_DOUBLE_JUMPED) != 0;
    o.has_flipped = (f & CF_HAS_FLIPPED) != 0;
    o.is_flipping = (f & CF_IS_FLIPPING) != 0;
    o.is_jumping = (f & CF_IS_JUMPING) != 0;
    o.is_supersonic = (f & CF_SUPERSONIC) != 0;
    o.is_auto_flipping = (f & CF_AUTO_FLIPPING) != 0;
    o.is_demoed = (f & CF_DEMOED) != 0;
    o.world_contact = (f & CF_WORLD_CONTACT) != 0;
    o.ball_hit_valid = (f & CF_BALL_HIT_VALID) != 0;
    o.team = (f & CF_TEAM_ORANGE) ? 1 : 0;
    for (int i = 0; i < 4; i++) o.wheels_with_contact[i] = (f & (CF_WHEEL0 << i)) ? 1 : 0;
    o.ball_hit_tick = (uint64_t)p.ballHitTick[0] | ((uint64_t)p.ballHitTick[1] << 32);
    o.ball_hit_extra_tick = (uint64_t)p.ballHitExtraTick[0] | ((uint64_t)p.ballHitExtraTick[1] << 32);
    o.ball_hit_rel_pos = rsb_vec3{p.ballHitRelPos[0], p.ballHitRelPos[1], p.ballHitRelPos[2]};
    o.ball_hit_ball_pos = rsb_vec3{p.ballHitBallPos[0], p.ballHitBallPos[1], p.ballHitBallPos[2]};
    o.ball_hit_extra_vel = rsb_vec3{p.ballHitExtraVel[0], p.ballHitExtraVel[1], p.ballHitExtraVel[2]};
    o.last_controls = ctlFromRecord(p);
    o.id = id;
    return o;
}

// Car::SetState: transform, velocities and the whole CarState replaced; the broadphase
// registration and the vehicle's wheel values are kept (host and device: the state ring's
// restore kernel applies it too)
RSB_HD void applyCarState(CarP& p, const rsb_car_state& s) {
    M3 b = basisFromRot(s.rot);
    Xf x{b, V3{s.pos.x, s.pos.y, s.pos.z} * kUuToBt};
    xfToP(x, p.pos, p.rot);
    basisToFloats(b, p.rotMat);
    V3 v = V3{s.vel.x, s.vel.y, s.vel.z} * kUuToBt;
    p.lin[0] = v.x; p.lin[1] = v.y; p.lin[2] = v.z;
    p.ang[0] = s.ang_vel.x; p.ang[1] = s.ang_vel.y; p.ang[2] = s.ang_vel.z;
    p.boost = s.boost;
    p.timeSpentBoosting = s.time_spent_boosting;
    p.jumpTime = s.jump_time;
    p.flipTime = s.flip_time;
    p.airTime = s.air_time;
    p.airTimeSinceJump = s.air_time_since_jump;
    p.supersonicTime = s.supersonic_time;
    p.handbrakeVal = s.handbrake_val;
    p.autoFlipTimer = s.auto_flip_timer;
    p.autoFlipTorqueScale = s.auto_flip_torque_scale;
    p.demoRespawnTimer = s.demo_respawn_timer;
    p.carContactCooldown = s.car_contact_cooldown;
    p.flipRelTorque[0] = s.flip_rel_torque.x; p.flipRelTorque[1] = s.flip_rel_torque.y; p.flipRelTorque[2] = s.flip_rel_torque.z;
    p.worldContactNormal[0] = s.world_contact_normal.x;
    p.worldContactNormal[1] = s.world_contact_normal.y;
    p.worldContactNormal[2] = s.world_contact_normal.z;
    p.carContactOtherId = s.car_contact_other_id;
    uint32_t f = p.flags & (CF_TEAM_ORANGE | CF_NO_RESPONSE);
    if (s.is_on_ground) f |= CF_ON_GROUND;
    if (s.has_jumped) f |= CF_HAS_JUMPED;
    if (s.has_double_jumped) f |= CF_HAS_DOUBLE_JUMPED;
    if (s.has_flipped) f |= CF_HAS_FLIPPED;
    if (s.is_flipping) f |= CF_IS_FLIPPING;
    if (s.is_jumping) f |= CF_IS_JUMPING;
    if (s.is_supersonic) f |= CF_SUPERSONIC;
    if (s.is_auto_flipping) f |= CF_AUTO_FLIPPING;
    if (s.is_demoed) f |= CF_DEMOED;
    if (s.world_contact) f |= CF_WORLD_CONTACT;
    if (s.ball_hit_valid) f |= CF_BALL_HIT_VALID;
    for (int i = 0; i < 4; i++)
        if (s.wheels_with_contact[i]) f |= CF_WHEEL0 << i;
    p.flags = f;
    p.ballHitTick[0] = (uint32_t)s.ball_hit_tick;
    p.ballHitTick[1] = (uint32_t)(s.ball_hit_tick >> 32);
    p.ballHitExtraTick[0] = (uint32_t)s.ball_hit_extra_tick;
    p.ballHitExtraTick[1] = (uint32_t)(s.ball_hit_extra_tick >> 32);
    p.ballHitRelPos[0] = s.ball_hit_rel_pos.x; p.ballHitRelPos[1] = s.ball_hit_rel_pos.y; p.ballHitRelPos[2] = s.ball_hit_rel_pos.z;
    p.ballHitBallPos[0] = s.ball_hit_ball_pos.x; p.ballHitBallPos[1] = s.ball_hit_ball_pos.y; p.ballHitBallPos[2] = s.ball_hit_ball_pos.z;
    p.ballHitExtraVel[0] = s.ball_hit_extra_vel.x; p.ballHitExtraVel[1] = s.ball_hit_extra_vel.y; p.ballHitExtraVel[2] = s.ball_hit_extra_vel.z;
    const rsb_controls& lc = s.last_controls;
    p.lastCtl[0] = lc.throttle; p.lastCtl[1] = lc.steer; p.lastCtl[2] = lc.pitch; p.lastCtl[3] = lc.yaw; p.lastCtl[4] = lc.roll;
    p.lastCtlBits = (lc.jump ? 1u : 0u) | (lc.boost ? 2u : 0u) | (lc.handbrake ? 4u : 0u);
}

RSB_HD rsb_ball_state ballStateOf(const BallP& p) {
    rsb_ball_state o{};
    V3 pos = V3{p.pos[0], p.pos[1], p.pos[2]} * kBtToUu;
    V3 vel = V3{p.lin[0], p.lin[1], p.lin[2]} * kBtToUu;
    o.pos = rsb_vec3{pos.x, pos.y, pos.z};
    o.rot = rotFromBasis(p.rot);
    o.vel = rsb_vec3{vel.x, vel.y, vel.z};
    o.ang_vel = rsb_vec3{p.ang[0], p.ang[1], p.ang[2]};
    return o;
}

RSB_HD void applyBallState(BallP& p, const rsb_ball_state& s) {
    Xf x{basisFromRot(s.rot), V3{s.pos.x, s.pos.y, s.pos.z} * kUuToBt};
    xfToP(x, p.pos, p.rot);
    V3 v = V3{s.vel.x, s.vel.y, s.vel.z} * kUuToBt;
    p.lin[0] = v.x; p.lin[1] = v.y; p.lin[2] = v.z;
    p.ang[0] = s.ang_vel.x; p.ang[1] = s.ang_vel.y; p.ang[2] = s.ang_vel.z;
}

}  // namespace rsb
