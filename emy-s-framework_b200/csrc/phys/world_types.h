// Per-arena working state of one simulation tick.
//
// The tick is a restatement of RocketSim's Arena::Step (Arena.cpp:716-812) over Bullet's
// btDiscreteDynamicsWorld::stepSimulation (btDiscreteDynamicsWorld.cpp:320-437).  Object
// numbering follows the reference's collision-object array, which fixes the order of
// broadphase pairs, manifolds and solver rows:
//   0..15  arena meshes (soccar/mesh_0..15)       static, friction 0.6, restitution 0.3
//   16..19 planes: floor, ceiling, -x wall, +x wall  static, same material
//   20     ball
//   21..26 cars, blue first then orange (Arena::AddCar order)
#pragma once
#include "arena_static.h"
#include "consts.h"

namespace rsb {

constexpr int OBJ_BALL = NUM_STATICS;       // 20
constexpr int OBJ_CAR0 = NUM_STATICS + 1;   // 21
constexpr int MAX_CARS = 6;
constexpr int MAX_BODIES = 1 + MAX_CARS;

// btCollisionObject activation states (btCollisionObject.h)
enum : int32_t { ACT_ACTIVE = 1, ACT_SLEEPING = 2, ACT_WANTS_DEACT = 3, ACT_DISABLE_DEACT = 4, ACT_DISABLE_SIM = 5 };

constexpr float STATIC_FRICTION = 0.6f, STATIC_RESTITUTION = 0.3f;

struct Body {
    Xf xf;       // world transform (Bullet units)
    Xf ixf;      // interpolation transform = this tick's predicted transform
    V3 lin, ang; // velocities
    V3 force, torque;
    M3 invIw;    // m_invInertiaTensorWorld
    V3 invIl;    // m_invInertiaLocal
    float invMass;
    V3 grav;     // m_gravity (force)
    float linDampFactor;  // btPow(1 - linearDamping, dt), precomputed on the host
    float friction, restitution;
    int32_t act;
    int32_t noResp;       // CF_NO_CONTACT_RESPONSE
    int32_t islandTag;
    int32_t solverId;
    // broadphase proxy
    V3 bpMin, bpMax;
    int32_t cell, ci, cj, ck;
    int32_t regStamp;     // order of the last (re-)registration in the grid cells
    // special-contact aggregation (btCollisionObject::m_specialResolveInfo)
    int32_t spCount;
    float spFric, spRest, spDist;
    V3 spNormal;
};

// btManifoldPoint fields the pipeline uses
struct MPoint {
    V3 localA, localB, posA, posB, normal;
    float dist, fric, rest;
    int32_t index1;   // triangle index on the B side (-1 when B is not a mesh)
    int32_t special;
};

constexpr int MAX_MANIFOLDS = 64;   // headers, one per processed pair, in creation order
constexpr int MAX_POINTS = 4;       // btPersistentManifold MANIFOLD_CACHE_SIZE
constexpr int MAX_BLOCKS = 16;      // manifolds that hold contacts in one tick

struct Manifold {
    int32_t o0, o1;   // object ids (body0 / body1)
    float cbt;        // contact breaking threshold
    int32_t n;        // number of points
    MPoint* pt;       // point block (4 slots), null until the first contact
};

struct BlockPool {
    int32_t n;
    uint32_t* status;
    MPoint pts[MAX_BLOCKS * MAX_POINTS];
};

// btSolverConstraint fields used by contact and friction rows
struct SRow {
    V3 n1, rc1, angA;  // m_contactNormal1, m_relpos1CrossNormal, m_angularComponentA
    V3 n2, rc2, angB;
    float rhs, rhsPen, cfm, jacInv, lo, hi, friction;
    float applied, appliedPush;
    int16_t bA, bB;   // solver body ids
    int16_t fIdx;     // contact row: first friction row; friction row: its contact row
    int16_t special;
};

struct SBody {
    Xf xf;
    V3 invMassV;
    V3 lin, ang;       // velocities at solve start
    V3 extF, extT;     // m_externalForceImpulse / m_externalTorqueImpulse
    V3 dLin, dAng;     // delta velocities
    V3 push, turn;
    int32_t body;      // index into Arena.bodies, -1 for the fixed body
};

constexpr int MAX_CONTACT_ROWS = 64;
constexpr int MAX_FRICTION_ROWS = 64;
constexpr int MAX_PAIRS = 64;

// Car body, hitbox and wheel constants, evaluated once on the host with the reference's
// operation order (Car::_BulletSetup, Car.cpp:195-277; btBoxShape, btCompoundShape,
// btRigidBody::setMassProps / setGravity) plus the mutator values the car logic reads.
struct CarParams {
    V3 boxHe;            // btBoxShape implicit half extents (without margin)
    float boxMargin;     // setSafeMargin result
    V3 boxHeM;           // half extents with margin
    V3 childOff;         // hitbox offset of the compound's only child
    V3 cmpMin, cmpMax;   // btCompoundShape local AABB
    float cbt;           // contact breaking threshold of the compound shape
    float invMass, mass; // mass = 1 / invMass (btRigidBody::getMass)
    V3 invInertiaLocal;
    V3 grav;             // gravity force (acceleration * (1 / invMass))
    V3 wheelConn[4];     // chassis connection points
    float wheelRadius[4], susRest[4], susForceScale[4];
    float susTravel;     // m_maxSuspensionTravelCm / 100
    float rayLen[4];     // rest + travel + radius - SUSPENSION_SUBTRACTION
    float pushThresh[4]; // rest + radius - SUSPENSION_SUBTRACTION
    float dodgeDeadzone;
    float flipZDamp;     // powf(1 - FLIP_Z_DAMP_120, dt / (1 / 120))
    // mutator values (MutatorConfig)
    float jumpAccel, jumpImmediateForce, boostAccelGround, boostAccelAir, boostUsedPerSecond;
    float respawnDelay, bumpCooldown, padCooldownBig, padCooldownSmall, spawnBoost;
    float ballHitExtraScale, bumpForceScale, worldFriction, worldRestitution;
    int32_t unlimitedFlips, unlimitedDoubleJumps, demoMode, teamDemos;
};

struct WorldParams {
    float dt;                 // 1/120
    V3 gravity;               // Bullet units
    float ballLinDampFactor;  // btPow(1 - ballDrag, dt)
    float ballRadius;         // Bullet units
    float ballMargin;         // sphere margin (= radius)
    float ballAabbExt;        // margin + 0.08f
    float ballCbt;            // contact breaking threshold of the ball shape
    float ballInvMass;
    V3 ballGrav;
    V3 ballInvInertia;
    float ballFriction, ballRestitution;
    float ballMaxSpeedBt;
    float goalBaseY;          // mutator goalBaseThresholdY (uu)
    float ballRadiusUu;
    CarParams car;
    int8_t padGrid[8 * 10];   // BoostPadGrid cells (x * 10 + y) -> pad index, -1 empty
};

// ------------------------------------------------------------------ cars in a tick

// One wheel's btWheelInfoRL raycast and force values of the current tick.
struct WheelTick {
    V3 hardPoint, dirWS, axleWS;
    V3 contactPoint, contactNormal;
    V3 impulse;
    M3 basis;              // m_worldTransform basis (steering applied)
    float suspLen, relVel, clippedInv, susForce;
    int32_t ground;        // collision object hit by the ray, -1 none
    int32_t inContact, withWorld;
};

// Car::_internalState plus the btVehicleRL values that persist between ticks.
struct CarSim {
    float boost, timeSpentBoosting, jumpTime, flipTime, airTime, airTimeSinceJump;
    float supersonicTime, handbrakeVal, autoFlipTimer, autoFlipTorqueScale;
    float demoRespawnTimer, carContactCooldown;
    V3 flipRelTorque, worldContactNormal;
    uint32_t carContactOtherId;
    uint32_t flags;        // CF_* bits
    uint64_t ballHitTick, ballHitExtraTick;
    V3 ballHitRelPos, ballHitBallPos, ballHitExtraVel;
    M3 rotMat;             // CarState::rotMat (basis after the last post-tick update)
    float ctl[5];          // throttle, steer, pitch, yaw, roll
    uint32_t ctlBits;      // jump | boost << 1 | handbrake << 2
    float lastCtl[5];
    uint32_t lastCtlBits;
    float steerAngle, engineForce, brake;
    float latF[4], longF[4], extraPush[4];
    V3 velCache;           // _velocityImpulseCache
    int32_t team;          // 0 blue, 1 orange
    uint32_t id;           // car id (1-based, creation order)
    WheelTick w[4];
};

// CarSim flag bits (shared with the persistent record)
enum : uint32_t {
    CF_ON_GROUND = 1u << 0, CF_HAS_JUMPED = 1u << 1, CF_HAS_DOUBLE_JUMPED = 1u << 2,
    CF_HAS_FLIPPED = 1u << 3, CF_IS_FLIPPING = 1u << 4, CF_IS_JUMPING = 1u << 5,
    CF_SUPERSONIC = 1u << 6, CF_AUTO_FLIPPING = 1u << 7, CF_DEMOED = 1u << 8,
    CF_WORLD_CONTACT = 1u << 9, CF_BALL_HIT_VALID = 1u << 10,
    CF_WHEEL0 = 1u << 11,  // 4 bits: wheelsWithContact
    CF_TEAM_ORANGE = 1u << 15,
    // btCollisionObject::CF_NO_CONTACT_RESPONSE of the car's rigid body: set by the pre-tick of
    // a demoed car, cleared by the pre-tick of a live one (Car.cpp:67-83).  It belongs to the
    // body, so it outlasts the tick (a car that pre-ticks earlier casts its wheel rays past a
    // demoed car, btDefaultVehicleRaycaster.cpp:43) and Car::SetState leaves it alone.  Not
    // part of the public CarState.
    CF_NO_RESPONSE = 1u << 16
};

}  // namespace rsb
