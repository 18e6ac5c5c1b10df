// Game constants of the soccar arena (values as RocketSim's RLConst.h, CarConfig.cpp,
// MutatorConfig.cpp state them; each block names its source).
#pragma once
#include "vecmath.h"

namespace rsb {

// RocketSim src/RLConst.h:11-137
constexpr float GRAVITY_Z = -650.f;
constexpr float ARENA_EXTENT_X = 4096.f, ARENA_EXTENT_Y = 5120.f, ARENA_HEIGHT = 2048.f;
constexpr float CAR_MASS_BT = 180.f;
constexpr float BALL_MASS_BT = CAR_MASS_BT / 6.f;
constexpr float CAR_COLLISION_FRICTION = 0.3f, CAR_COLLISION_RESTITUTION = 0.1f;
constexpr float CARBALL_COLLISION_FRICTION = 2.0f, CARBALL_COLLISION_RESTITUTION = 0.0f;
constexpr float CARWORLD_COLLISION_FRICTION = 0.3f, CARWORLD_COLLISION_RESTITUTION = 0.3f;
constexpr float CARCAR_COLLISION_FRICTION = 0.09f, CARCAR_COLLISION_RESTITUTION = 0.1f;
constexpr float BALL_REST_Z = 93.15f, BALL_MAX_ANG_SPEED = 6.f, BALL_DRAG = 0.03f;
constexpr float BALL_FRICTION = 0.35f, BALL_RESTITUTION = 0.6f;
constexpr float CAR_MAX_SPEED = 2300.f, BALL_MAX_SPEED = 6000.f;
constexpr float BOOST_MAX = 100.f, BOOST_USED_PER_SECOND = BOOST_MAX / 3, BOOST_MIN_TIME = 0.1f;
constexpr float BOOST_ACCEL_GROUND = 2975 / 3.f, BOOST_ACCEL_AIR = 3175 / 3.f, BOOST_SPAWN_AMOUNT = BOOST_MAX / 3;
constexpr float CAR_MAX_ANG_SPEED = 5.5f;
constexpr float SUPERSONIC_START_SPEED = 2200.f, SUPERSONIC_MAINTAIN_MIN_SPEED = SUPERSONIC_START_SPEED - 100.f;
constexpr float SUPERSONIC_MAINTAIN_MAX_TIME = 1.f;
constexpr float POWERSLIDE_RISE_RATE = 5, POWERSLIDE_FALL_RATE = 2;
constexpr float THROTTLE_TORQUE_AMOUNT = CAR_MASS_BT * 400.f;
constexpr float BRAKE_TORQUE_AMOUNT = CAR_MASS_BT * (14.25f + (1.f / 3.f));
constexpr float STOPPING_FORWARD_VEL = 25.f, COASTING_BRAKE_FACTOR = 0.15f;
constexpr float BRAKING_NO_THROTTLE_SPEED_THRESH = 0.01f, THROTTLE_DEADZONE = 0.001f;
constexpr float THROTTLE_AIR_ACCEL = 200 / 3.f;
constexpr float JUMP_ACCEL = 4375.f / 3.f, JUMP_IMMEDIATE_FORCE = 875.f / 3.f;
constexpr float JUMP_MIN_TIME = 0.025f, JUMP_RESET_TIME_PAD = (1 / 40.f), JUMP_MAX_TIME = 0.2f;
constexpr float DOUBLEJUMP_MAX_DELAY = 1.25f;
constexpr float FLIP_Z_DAMP_120 = 0.35f, FLIP_Z_DAMP_START = 0.15f, FLIP_Z_DAMP_END = 0.21f;
constexpr float FLIP_TORQUE_TIME = 0.65f, FLIP_TORQUE_MIN_TIME = 0.41f;
constexpr float FLIP_PITCHLOCK_TIME = 1.f, FLIP_PITCHLOCK_EXTRA_TIME = 0.3f;
constexpr float FLIP_INITIAL_VEL_SCALE = 500.f, FLIP_TORQUE_X = 260.f, FLIP_TORQUE_Y = 224.f;
constexpr float FLIP_FORWARD_IMPULSE_MAX_SPEED_SCALE = 1.f, FLIP_SIDE_IMPULSE_MAX_SPEED_SCALE = 1.9f;
constexpr float FLIP_BACKWARD_IMPULSE_MAX_SPEED_SCALE = 2.5f, FLIP_BACKWARD_IMPULSE_SCALE_X = 16.f / 15.f;
constexpr float BALL_COLLISION_RADIUS_SOCCAR = 91.25f;
constexpr float SOCCAR_GOAL_SCORE_BASE_THRESHOLD_Y = 5124.25f;
// 2 * M_PI / (1 << 16) * 1000, evaluated in double then narrowed as the reference's constexpr does
constexpr float CAR_TORQUE_SCALE = (float)(2 * 3.14159265358979323846 / (1 << 16) * 1000);
constexpr float CAR_AUTOFLIP_IMPULSE = 200, CAR_AUTOFLIP_TORQUE = 50, CAR_AUTOFLIP_TIME = 0.4f;
constexpr float CAR_AUTOFLIP_NORMZ_THRESH = (float)0.70710678118654752440;  // M_SQRT1_2
constexpr float CAR_AUTOFLIP_ROLL_THRESH = 2.8f;
constexpr float CAR_AUTOROLL_FORCE = 100, CAR_AUTOROLL_TORQUE = 80;
constexpr float BALL_CAR_EXTRA_IMPULSE_Z_SCALE = 0.35f, BALL_CAR_EXTRA_IMPULSE_FORWARD_SCALE = 0.65f;
constexpr float BALL_CAR_EXTRA_IMPULSE_MAXDELTAVEL_UU = 4600.f;
constexpr float CAR_SPAWN_REST_Z = 17.f, CAR_RESPAWN_Z = 36.f;
constexpr float BUMP_COOLDOWN_TIME = 0.25f, BUMP_MIN_FORWARD_DIST = 64.5f, DEMO_RESPAWN_TIME = 3.f;

// RLConst::BTVehicle (RLConst.h:137-149)
constexpr float SUSPENSION_FORCE_SCALE_FRONT = 36.f - (1.f / 4.f);
constexpr float SUSPENSION_FORCE_SCALE_BACK = 54.f + (1.f / 4.f) + (1.5f / 100.f);
constexpr float SUSPENSION_STIFFNESS = 500.f, WHEELS_DAMPING_COMPRESSION = 25.f, WHEELS_DAMPING_RELAXATION = 40.f;
constexpr float MAX_SUSPENSION_TRAVEL = 12.f, SUSPENSION_SUBTRACTION = 0.05f;

// RLConst.h:196-198
constexpr float CAR_AIR_CONTROL_TORQUE_X = 130, CAR_AIR_CONTROL_TORQUE_Y = 95, CAR_AIR_CONTROL_TORQUE_Z = 400;
constexpr float CAR_AIR_CONTROL_DAMPING_X = 30, CAR_AIR_CONTROL_DAMPING_Y = 20, CAR_AIR_CONTROL_DAMPING_Z = 50;

// RLConst::BoostPads (RLConst.h:200-260); pad i < 6 is big, RocketSim's arena order (Arena.cpp:540-557)
constexpr float PAD_CYL_HEIGHT = 95, PAD_CYL_RAD_BIG = 208, PAD_CYL_RAD_SMALL = 144;
constexpr float PAD_BOX_HEIGHT = 64, PAD_BOX_RAD_BIG = 160, PAD_BOX_RAD_SMALL = 120;
constexpr float PAD_COOLDOWN_BIG = 10, PAD_COOLDOWN_SMALL = 4;
constexpr float PAD_BOOST_AMOUNT_BIG = 100, PAD_BOOST_AMOUNT_SMALL = 12;
constexpr int NUM_PADS = 34, NUM_BIG_PADS = 6;

// Octane preset (CarConfig.cpp:20-76, index 0)
constexpr float OCT_HITBOX_X = 120.507f, OCT_HITBOX_Y = 86.6994f, OCT_HITBOX_Z = 38.6591f;
constexpr float OCT_HITBOX_OFF_X = (float)13.87566, OCT_HITBOX_OFF_Y = 0, OCT_HITBOX_OFF_Z = 20.755f;
constexpr float OCT_FRONT_RAD = 12.50f, OCT_BACK_RAD = 15.00f;
constexpr float OCT_FRONT_SUS_REST = 38.755f, OCT_BACK_SUS_REST = 37.055f;
constexpr float OCT_FRONT_OFF_X = 51.25f, OCT_FRONT_OFF_Y = 25.90f, OCT_FRONT_OFF_Z = 20.755f;
constexpr float OCT_BACK_OFF_X = -33.75f, OCT_BACK_OFF_Y = 29.50f, OCT_BACK_OFF_Z = 20.755f;
constexpr float OCT_DODGE_DEADZONE = 0.5f;

// Piecewise-linear curves (RLConst.h:327-439), evaluated as LinearPieceCurve::GetOutput
// (Math.cpp:5-31): clamp below the first knot, interpolate between knots, clamp above the last.
struct Curve {
    int n;
    float x[6];
    float y[6];
};

RSB_HD float curveOut(const Curve& c, float input, float def = 1.f) {
    if (c.n == 0) return def;
    if (input <= c.x[0]) return c.y[0];
    for (int i = 1; i < c.n; i++) {
        if (c.x[i] > input) {
            float range = c.x[i] - c.x[i - 1];
            float vdiff = c.y[i] - c.y[i - 1];
            float f = (input - c.x[i - 1]) / range;
            return c.y[i - 1] + vdiff * f;
        }
    }
    return c.y[c.n - 1];
}

// Curves are produced by value (functions usable from host and device code):
// crvSteerAngle = STEER_ANGLE_FROM_SPEED_CURVE, crvPowerslideSteer =
// POWERSLIDE_STEER_ANGLE_FROM_SPEED_CURVE, crvDriveTorque = DRIVE_SPEED_TORQUE_FACTOR_CURVE,
// crvNonSticky = NON_STICKY_FRICTION_FACTOR_CURVE, crvLatFriction / crvLongFriction =
// LAT_ / LONG_FRICTION_CURVE, crvHandbrakeLat / crvHandbrakeLong =
// HANDBRAKE_LAT_ / HANDBRAKE_LONG_FRICTION_FACTOR_CURVE, crvBallCarExtra =
// BALL_CAR_EXTRA_IMPULSE_FACTOR_CURVE, crvBumpGround / crvBumpAir / crvBumpUp =
// BUMP_VEL_AMOUNT_GROUND_ / BUMP_VEL_AMOUNT_AIR_ / BUMP_UPWARD_VEL_AMOUNT_CURVE.
#define RSB_CURVE(fn, ...) \
    RSB_HD Curve fn() { return Curve __VA_ARGS__; }
RSB_CURVE(crvSteerAngle, {6, {0, 500, 1000, 1500, 1750, 3000}, {0.53356f, 0.31930f, 0.18203f, 0.10570f, 0.08507f, 0.03454f}})
RSB_CURVE(crvPowerslideSteer, {2, {0, 2500}, {0.39235f, 0.12610f}})
RSB_CURVE(crvDriveTorque, {3, {0, 1400, 1410}, {1.0f, 0.1f, 0.0f}})
RSB_CURVE(crvNonSticky, {3, {0, 0.7075f, 1}, {0.1f, 0.5f, 1.0f}})
RSB_CURVE(crvLatFriction, {2, {0, 1}, {1.0f, 0.2f}})
RSB_CURVE(crvLongFriction, {0, {}, {}})
RSB_CURVE(crvHandbrakeLat, {1, {0}, {0.1f}})
RSB_CURVE(crvHandbrakeLong, {2, {0, 1}, {0.5f, 0.9f}})
RSB_CURVE(crvBallCarExtra, {4, {0, 500.f, 2300.f, 4600.f}, {0.65f, 0.65f, 0.55f, 0.30f}})
RSB_CURVE(crvBumpGround, {3, {0.f, 1400.f, 2200.f}, {(5.f / 6.f), 1100.f, 1530.f}})
RSB_CURVE(crvBumpAir, {3, {0.f, 1400.f, 2200.f}, {(5.f / 6.f), 1390.f, 1945.f}})
RSB_CURVE(crvBumpUp, {3, {0.f, 1400.f, 2200.f}, {(2.f / 6.f), 278.f, 417.f}})
#undef RSB_CURVE

// Boost pad locations, big pads first (RLConst.h:222-252)
struct PadLoc { float x, y, z; };
#define RSB_PAD_LOCS                                                                     \
    {{-3584.f, 0.f, 73.f}, {3584.f, 0.f, 73.f}, {-3072.f, 4096.f, 73.f},                 \
     {3072.f, 4096.f, 73.f}, {-3072.f, -4096.f, 73.f}, {3072.f, -4096.f, 73.f},          \
     {0.f, -4240.f, 70.f}, {-1792.f, -4184.f, 70.f}, {1792.f, -4184.f, 70.f},           \
     {-940.f, -3308.f, 70.f}, {940.f, -3308.f, 70.f}, {0.f, -2816.f, 70.f},             \
     {-3584.f, -2484.f, 70.f}, {3584.f, -2484.f, 70.f}, {-1788.f, -2300.f, 70.f},       \
     {1788.f, -2300.f, 70.f}, {-2048.f, -1036.f, 70.f}, {0.f, -1024.f, 70.f},           \
     {2048.f, -1036.f, 70.f}, {-1024.f, 0.f, 70.f}, {1024.f, 0.f, 70.f},                \
     {-2048.f, 1036.f, 70.f}, {0.f, 1024.f, 70.f}, {2048.f, 1036.f, 70.f},              \
     {-1788.f, 2300.f, 70.f}, {1788.f, 2300.f, 70.f}, {-3584.f, 2484.f, 70.f},          \
     {3584.f, 2484.f, 70.f}, {0.f, 2816.f, 70.f}, {-940.f, 3308.f, 70.f},               \
     {940.f, 3308.f, 70.f}, {-1792.f, 4184.f, 70.f}, {1792.f, 4184.f, 70.f},            \
     {0.f, 4240.f, 70.f}}
static constexpr PadLoc PAD_LOCS_HOST[NUM_PADS] = RSB_PAD_LOCS;
#if defined(__CUDACC__)
__device__ __constant__ PadLoc PAD_LOCS_DEV[NUM_PADS] = RSB_PAD_LOCS;
#endif
RSB_HD PadLoc padLoc(int p) {
#if defined(__CUDA_ARCH__)
    return PAD_LOCS_DEV[p];
#else
    return PAD_LOCS_HOST[p];
#endif
}

// Car spawn / respawn tables for blue (RLConst.h:278-311); orange is mirrored.
struct SpawnPos { float x, y, yaw; };
constexpr int NUM_KICKOFF_SPAWNS = 5, NUM_RESPAWNS = 4;

}  // namespace rsb
