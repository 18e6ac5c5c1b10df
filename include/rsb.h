/*
 * rsb.h — C ABI of the batched RocketSim engine for B200 (sm_100a).
 *
 * One handle owns N independent soccar arenas (ragged 1v1 / 2v2 / 3v3) whose
 * whole state lives in device memory.  The entry points mirror the public
 * methods of the reference batch simulator so that the PPO collector's env
 * layer can switch to this library without changing its call sequence:
 *
 *   reference (RocketSimCuda/include/RocketSimCuda.h)      this ABI
 *   -----------------------------------------------------  ------------------------------
 *   RocketSimCudaBatch::Init            :264               rsb_create
 *   RocketSimCudaBatch::Destroy         :267               rsb_destroy
 *   RocketSimCudaBatch::AddCar          :272               rsb_config.team_sizes (cars are
 *                                                          laid out blue first, then orange)
 *   RocketSimCudaBatch::ResetArena      :275               rsb_reset_arenas
 *   RocketSimCudaBatch::ResetAllArenas  :278               rsb_reset_all
 *   RocketSimCudaBatch::SetResetCurriculum :283            rsb_set_reset_curriculum
 *   RocketSimCudaBatch::UploadDiscreteActionLut :293       rsb_set_action_lut
 *   RocketSimCudaBatch::SetDiscreteActionsFromIndices :297 rsb_set_actions_host
 *   RocketSimCudaBatch::SetDiscreteActionsFromDevice  :300 rsb_set_actions_device
 *   RocketSimCudaBatch::SetAllCarControls :290             rsb_set_controls
 *   RocketSimCudaBatch::Step            :310               rsb_step
 *   RocketSimCudaBatch::BuildAdvancedObsAndDefaultMasks :316 rsb_build_obs
 *   RocketSimCudaBatch::SnapshotTrainingState :334         rsb_snapshot
 *   RocketSimCudaBatch::BuildRewardsAndTerminals :339      rsb_build_rewards_terminals
 *   RocketSimCudaBatch::CopyBuilt*      :342-345           rsb_copy_obs / _masks / _rewards / _terminals
 *   RocketSimCudaBatch::Get*DevicePtr   :387-396           rsb_device_ptr
 *   RocketSimCudaBatch::GetAllCarStates :355               rsb_get_cars
 *   RocketSimCudaBatch::GetAllBallStates :361              rsb_get_balls
 *   RocketSimCudaBatch::GetAllBoostPadStates :365          rsb_get_pads
 *   RocketSimCudaBatch::GetAllArenaInfos :369              rsb_get_arena_info
 *   RocketSimCudaBatch::SetCarState/SetBallState/SetAllBoostPadStates :377-383
 *                                                          rsb_set_cars / rsb_set_balls / rsb_set_pads
 *   RocketSimCudaBatch::Synchronize     :346               rsb_sync
 *   (none: errors were printed and ignored)                rsb_last_error, rsb_stats
 *
 * Conventions
 *   - Every function returns an rsb_status (0 = ok).  On error the handle keeps a
 *     message that rsb_last_error() returns.  Nothing is printed.
 *   - Units are Unreal units (uu) and seconds, as in RocketSim's public states.
 *   - "stream" arguments are a cudaStream_t passed as void*; NULL = the handle's
 *     own stream.  Host-buffer functions synchronise that stream before returning.
 *   - Car c of arena a is global car index car_offset[a] + c.  Within an arena the
 *     first team_size cars are blue, the next team_size orange.  Car ids (used by
 *     boost-pad locks and bump cooldowns) are c + 1, as RocketSim's Arena::AddCar
 *     assigns them in that order.
 *   - Boost pads use RocketSim's arena order (6 big pads first, then 28 small).
 */
#ifndef RSB_H
#define RSB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RSB_MAX_TEAM_SIZE 3
#define RSB_MAX_CARS_PER_ARENA 6
#define RSB_NUM_PADS 34
#define RSB_NUM_ACTIONS 90
#define RSB_OBS_BASE 51
#define RSB_OBS_PER_CAR 29

typedef int32_t rsb_status;
enum {
    RSB_OK = 0,
    RSB_ERR_INVALID = -1,     /* bad argument or size */
    RSB_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    RSB_ERR_NOMEM = -3,       /* allocation failed */
    RSB_ERR_MESH = -4,        /* collision meshes missing or malformed */
    RSB_ERR_STATE = -5,       /* call out of order (e.g. no action table) */
    RSB_ERR_TIMEOUT = -6,     /* a bounded device wait ran out */
    RSB_ERR_UNSUPPORTED = -7  /* option not built into this library */
};

/* Which device buffer rsb_device_ptr returns. */
enum {
    RSB_BUF_OBS = 0,        /* float [num_cars][obs_stride] */
    RSB_BUF_MASKS = 1,      /* uint8 [num_cars][90] */
    RSB_BUF_REWARDS = 2,    /* float [num_cars] */
    RSB_BUF_TERMINALS = 3,  /* uint8 [num_arenas]: RLGymCPP TerminalType: 0 none, 1 normal
                               (goal), 2 truncated (no touch / episode tick limit) */
    RSB_BUF_CONTROLS = 4,   /* rsb_controls [num_cars] */
    RSB_BUF_ACTIONS = 5,    /* int32 [num_cars] */
    RSB_BUF_BALL_PRED = 6,  /* rsb_ball_state [num_arenas][n_slices] of the last rsb_predict_ball */
    RSB_BUF_VANTA_OBS = 7   /* float [num_cars][RSB_VANTA_OBS_SIZE] of the last rsb_build_vanta_obs */
};

/* Arena-narrowphase mode. */
enum {
    RSB_CULL_EXACT = 0,         /* every query runs the exact BVH narrowphase */
    RSB_CULL_LEARNED = 1,       /* a learned distance bound skips the static tests of bodies it
                                   places clear of every static shape for the launch */
    RSB_CULL_LEARNED_AUDIT = 2, /* as LEARNED, but the skipped tests run anyway: whatever they find
                                   counts as a missed contact and reverts the arena to EXACT */
    RSB_CULL_VOXEL = 3,         /* as LEARNED with a bound that is not learned: the distance from the
                                   body's 64 uu voxel to the nearest voxel holding a mesh triangle,
                                   less the voxel diagonal (exact lower bound, needs no training) */
    RSB_CULL_VOXEL_AUDIT = 4    /* as VOXEL, with the skipped tests run and checked */
};

/* Reset modes for rsb_reset_arenas. */
enum {
    RSB_RESET_KICKOFF = 0,      /* RocketSim Arena::ResetToRandomKickoff layout */
    RSB_RESET_RANDOM_STATE = 1, /* RLGymCPP RandomState(true, true, false): uniform random
                                   cars/ball inside the field, half the cars on the ground */
    RSB_RESET_HIGH_CONTACT = 2, /* cars within 300 uu of the ball or each other, 1500-2300
                                   uu/s toward it, half airborne, some on walls / ceiling
                                   (no CPU counterpart in the reference) */
    RSB_RESET_CURRICULUM = 3    /* per arena, one of kickoff / fuzzed kickoff / aerial / ball
                                   chase drawn with the weights of rsb_set_reset_curriculum
                                   (the reference batch's ResetArena, RocketSimCudaApi.cuh:216-442;
                                   GPU-only: the CPU reference has no curriculum) */
};

typedef struct rsb_vec3 { float x, y, z; } rsb_vec3;

/* Rows of RocketSim's RotMat: forward, right, up. */
typedef struct rsb_rotmat { rsb_vec3 forward, right, up; } rsb_rotmat;

/* RocketSim CarControls (Sim/CarControls.h). 24 bytes. */
typedef struct rsb_controls {
    float throttle, steer, pitch, yaw, roll;
    uint8_t jump, boost, handbrake, pad_;
} rsb_controls;

/* RocketSim CarState (Sim/Car/Car.h:15-100) plus BallHitInfo. */
typedef struct rsb_car_state {
    rsb_vec3 pos;
    rsb_rotmat rot;
    rsb_vec3 vel;
    rsb_vec3 ang_vel;          /* rad/s */
    float boost;               /* 0..100 */
    float time_spent_boosting;
    float jump_time, flip_time, air_time, air_time_since_jump;
    float supersonic_time, handbrake_val;
    float auto_flip_timer, auto_flip_torque_scale;
    float demo_respawn_timer;
    float car_contact_cooldown;
    rsb_vec3 flip_rel_torque;
    rsb_vec3 world_contact_normal;
    uint32_t car_contact_other_id;
    uint8_t is_on_ground, has_jumped, has_double_jumped, has_flipped;
    uint8_t is_flipping, is_jumping, is_supersonic, is_auto_flipping;
    uint8_t is_demoed, world_contact, ball_hit_valid, team; /* team: 0 blue, 1 orange */
    uint8_t wheels_with_contact[4];
    uint32_t pad1_;                  /* explicit padding (always 0) */
    uint64_t ball_hit_tick;          /* ~0 when never */
    uint64_t ball_hit_extra_tick;    /* tick of the last extra car-ball impulse, ~0 when never */
    rsb_vec3 ball_hit_rel_pos, ball_hit_ball_pos, ball_hit_extra_vel;
    rsb_controls last_controls;
    uint32_t id;
    uint32_t pad_, pad2_;            /* explicit padding (always 0) */
} rsb_car_state;

/* RocketSim BallState (Sim/Ball/Ball.h:15-45), soccar fields. */
typedef struct rsb_ball_state {
    rsb_vec3 pos;
    rsb_rotmat rot;
    rsb_vec3 vel;
    rsb_vec3 ang_vel;
} rsb_ball_state;

/* RocketSim BoostPadState (Sim/BoostPad/BoostPad.h:21-30). */
typedef struct rsb_pad_state {
    uint8_t is_active;
    uint8_t pad_[3];
    float cooldown;
    uint32_t prev_locked_car_id;  /* 0 = none */
} rsb_pad_state;

typedef struct rsb_arena_info {
    uint64_t tick_count;
    int32_t num_cars;
    int32_t team_size;
    int32_t goal_scored;   /* 1 while the ball is past a goal line (Arena::IsBallScored) */
    int32_t goal_team;     /* team that scored: 0 blue, 1 orange, -1 none */
    int32_t episode_ticks; /* ticks since the last reset, for the timeout terminal */
    int32_t status;        /* per-arena status bits, RSB_ARENA_* */
} rsb_arena_info;

/* Per-arena status bits (rsb_arena_info.status). */
enum {
    RSB_ARENA_NONFINITE = 1,       /* NaN/Inf appeared in the state; arena should be reset */
    RSB_ARENA_ROW_OVERFLOW = 2,    /* a fixed pool (solver rows, manifolds, pairs, the manifold sort's
                                      stack) was full; the extra entries were dropped */
    RSB_ARENA_BVH_OVERFLOW = 4,    /* reserved, never set: the BVH walk is stackless */
    RSB_ARENA_CULL_MISS = 8,       /* the learned culler skipped a query that had a contact */
    RSB_ARENA_EPA_OVERFLOW = 16    /* EPA's horizon walk exceeded its fixed stack; contact dropped */
};

/* RocketSim MutatorConfig (Sim/MutatorConfig/MutatorConfig.h:16-70), soccar defaults when NULL. */
typedef struct rsb_mutators {
    rsb_vec3 gravity;
    float car_mass;            /* accepted and ignored, as in the reference: cars keep RocketSim's
                                  CAR_MASS_BT (Car.cpp:206-209; the batch simulator's CAR_MASS) */
    float car_world_friction, car_world_restitution;
    float ball_mass, ball_max_speed, ball_drag, ball_world_friction, ball_world_restitution;
    float jump_accel, jump_immediate_force;
    float boost_accel_ground, boost_accel_air, boost_used_per_second;
    float respawn_delay, bump_cooldown_time;
    float boost_pad_cooldown_big, boost_pad_cooldown_small, car_spawn_boost_amount;
    float ball_hit_extra_force_scale, bump_force_scale, ball_radius;
    uint8_t unlimited_flips, unlimited_double_jumps, demo_mode, enable_team_demos;
    float goal_base_threshold_y;
} rsb_mutators;

/* The four stub rewards of the collector (CommonRewards.h) plus terminal settings. */
typedef struct rsb_reward_config {
    float w_goal;                 /* GoalReward */
    float w_touch;                /* TouchBallReward */
    float w_vel_ball_to_goal;     /* VelocityBallToGoalReward */
    float w_vel_player_to_ball;   /* VelocityPlayerToBallReward */
    float goal_concede_scale;     /* GoalReward's concedeScale (default -1) */
    float team_spirit;            /* ZeroSumReward teamSpirit */
    float opponent_scale;         /* ZeroSumReward opponentScale */
    int32_t zero_sum;             /* bit k wraps reward k (goal, touch, ball-to-goal velocity,
                                     player-to-ball velocity) in ZeroSumReward */
    int32_t episode_max_ticks;    /* truncation after this many ticks since the arena's
                                     reset (0 = off) */
    float no_touch_timeout_s;     /* NoTouchCondition (0 = off) */
} rsb_reward_config;

typedef struct rsb_config {
    int32_t num_arenas;
    int32_t team_size;              /* used when team_sizes is NULL: 1, 2 or 3 */
    const int32_t* team_sizes;      /* optional [num_arenas], each 1..3 (ragged batches) */
    float tick_rate;                /* must be 120 */
    int32_t tick_skip;              /* env step length in ticks (for rewards), e.g. 8 */
    const char* meshes_path;        /* folder holding soccar/mesh_*.cmf (required) */
    const rsb_mutators* mutators;   /* NULL = soccar defaults */
    const rsb_reward_config* rewards; /* NULL = no rewards / terminals */
    int32_t cull_mode;              /* RSB_CULL_* */
    float cull_margin;              /* uu added to the learned bound before skipping */
    uint64_t seed;
    int32_t device;                 /* CUDA device ordinal */
    int32_t threads;                /* host threads (CPU implementations only; 0 = all) */
} rsb_config;

typedef struct rsb_stats {
    uint64_t ticks_simulated;       /* arena-ticks */
    uint64_t narrowphase_queries;   /* ball/car vs arena-mesh queries */
    uint64_t culled_queries;        /* queries skipped by the learned bound */
    uint64_t missed_contacts;       /* culled queries that had a contact (audited) */
    uint64_t solver_rows;           /* contact rows solved */
    uint64_t arenas_reverted;       /* arenas switched back to the exact path */
    uint64_t status_bits_seen;      /* OR of all rsb_arena_info.status bits */
    uint64_t state_bytes_per_step;  /* persistent state one rsb_step launch reads + writes
                                       (the step kernel's algorithmic HBM traffic); 0 on
                                       CPU implementations */
} rsb_stats;

typedef struct rsb_handle rsb_handle;

/* Fills *m with RocketSim's soccar MutatorConfig defaults. */
rsb_status rsb_default_mutators(rsb_mutators* m);
/* Fills *r with the collector's stub-reward defaults (all weights 1, zero-sum off). */
rsb_status rsb_default_rewards(rsb_reward_config* r);

rsb_status rsb_create(const rsb_config* cfg, rsb_handle** out);
rsb_status rsb_destroy(rsb_handle* h);

/* Layout: car_offset has num_arenas+1 entries, team_size num_arenas. Either may be NULL. */
rsb_status rsb_layout(const rsb_handle* h, int32_t* num_arenas, int32_t* num_cars,
                      int32_t* car_offset, int32_t* team_size);
/* AdvancedObs row stride (floats) of the obs buffer: 51 + 29 * max cars per arena. */
rsb_status rsb_obs_stride(const rsb_handle* h, int32_t* stride);

rsb_status rsb_reset_all(rsb_handle* h, uint64_t seed, int32_t mode);
/* VantaObs v3.5 rows (RocketSimCudaBatch::BuildVantaObs, RocketSimCuda.h:318-321, the device
 * builder VantaObsGpu.cuh): 366 floats per player, packed like the AdvancedObs rows
 * (row = rsb_layout's car offset of the arena + creation slot).  The builder keeps state
 * between builds: boost-pad timers per arena and demo / action timers per player, each
 * updated once per arena tick; an arena reset clears that arena's state
 * (RocketSimCudaApi.cuh:265-275).  With predict_ball the ball block carries the ball-only
 * rollout's positions and velocities at 120 / 240 / 360 ticks (as rsb_predict_ball), else
 * zeros.  Configuring (again) allocates the state once and clears it. */
#define RSB_VANTA_OBS_SIZE 366
typedef struct rsb_vanta_config {
    int32_t tick_skip;        /* the timers' step: tick_skip / 120 s (BatchConfig::vantaTickSkip, 8) */
    float dodge_deadzone;     /* BatchConfig::vantaDodgeDeadzone, 0.5 */
    int32_t only_closest_opp; /* BatchConfig::vantaOnlyClosestOpp, 0 */
    int32_t predict_ball;     /* BatchConfig::vantaPredictBall (default here 1) */
} rsb_vanta_config;
rsb_status rsb_vanta_default_config(rsb_vanta_config* cfg);
rsb_status rsb_vanta_configure(rsb_handle* h, const rsb_vanta_config* cfg);
/* Builds every player's row from the current state, on `stream` (NULL = the handle's). */
rsb_status rsb_build_vanta_obs(rsb_handle* h, void* stream);
/* n = num_cars * RSB_VANTA_OBS_SIZE; synchronises the handle's stream. */
rsb_status rsb_copy_vanta_obs(rsb_handle* h, float* out, size_t n);
/* The 34 boost-pad locations (x, y, z in uu) in the order of rsb_pad_state arrays. */
rsb_status rsb_pad_locations(float* xyz);

/* One collector env step captured as a CUDA graph (the reference launches each kernel of a
 * step separately, RocketSimCudaApi.cuh:551-571; no counterpart there): action expansion from
 * d_actions (device int32 [num_cars], read at every launch, so the caller refills it in
 * place), the (culled) step of tick_skip ticks, observations + masks, rewards + terminals, and
 * the reset of every finished arena with reset_mode.  The k-th launch resets with seed + k, so
 * it equals the eager sequence rsb_set_actions_device, rsb_step, rsb_build_obs,
 * rsb_build_rewards_terminals, rsb_reset_done(seed + k).  The cull mode and the step kernel's
 * launch configuration in force at capture are the ones replayed.  Captured on the handle's
 * stream; a new capture replaces the old one.  Needs an action table and a reward
 * configuration. */
rsb_status rsb_env_graph_capture(rsb_handle* h, const int32_t* d_actions, int32_t tick_skip, int32_t reset_mode,
                                 uint64_t seed);
/* Replays the captured env step on `stream` (NULL = the handle's stream). */
rsb_status rsb_env_graph_launch(rsb_handle* h, void* stream);
/* Weights of the RSB_RESET_CURRICULUM modes (RocketSimCudaBatch::SetResetCurriculum,
 * RocketSimCuda.h:283): relative weights of kickoff, fuzzed kickoff (ball and cars moved a
 * little, mild ball velocity), aerial (ball raised near midfield, one car below it) and ball
 * chase (ball in play, every car near it on the ground facing it).  A negative, non-finite or
 * > 1e6 weight counts as 0; all zero means kickoff only.  A curriculum reset also staggers the
 * no-touch timer over [0, 0.9 x the timeout).  Default: kickoff only. */
rsb_status rsb_set_reset_curriculum(rsb_handle* h, float kickoff_w, float fuzzed_w, float aerial_w, float chase_w);
/* Resets every arena whose terminal flag (from the last rsb_build_rewards_terminals) is
 * set, on the device and stream-ordered, with no host round trip; the flags themselves
 * are left as they are.  Pass a different seed on every call.  No counterpart in the
 * reference: CudaEnvSet::ResetTerminalArenasGpu (CudaEnvSet.cpp:182-200) reads the
 * flags back to the host and calls RocketSimCudaBatch::ResetArena per arena. */
rsb_status rsb_reset_done(rsb_handle* h, uint64_t seed, int32_t mode, void* stream);
rsb_status rsb_reset_arenas(rsb_handle* h, const int32_t* arena_idx, int32_t n,
                            uint64_t seed, int32_t mode);

rsb_status rsb_set_action_lut(rsb_handle* h, const rsb_controls* lut, int32_t count);
/* Fills lut[90] with RLGymCPP's DefaultAction table. */
rsb_status rsb_default_action_lut(rsb_controls* lut, int32_t count);
rsb_status rsb_set_actions_host(rsb_handle* h, const int32_t* idx, int32_t n);
rsb_status rsb_set_actions_device(rsb_handle* h, const int32_t* d_idx, int32_t n, void* stream);
/* Same result as rsb_set_actions_host, for callers that must not allocate device memory
 * on the calling path (e.g. a collector running inside a memory budget fixed before the
 * first step): the host indices are staged in a statically sized device array that is
 * part of the library image instead of a buffer allocated for the handle.  At most
 * RSB_STATIC_ACTIONS_MAX indices per call (larger n returns RSB_ERR_INVALID).  The first
 * call on a device looks up the array's address (no allocation); make that first call
 * before capturing the handle's stream into a graph.  The address is kept for the life of
 * the process: after a cudaDeviceReset (or any new primary context) on that device, do not
 * call this function again in the same process.  The array is shared by every handle on a
 * device: calls from two handles of one device must not overlap in time.  No
 * counterpart in the reference (RocketSimCuda.h has only the allocating variant). */
#define RSB_STATIC_ACTIONS_MAX (65536 * 6)
rsb_status rsb_set_actions_host_static(rsb_handle* h, const int32_t* idx, int32_t n);
rsb_status rsb_set_controls(rsb_handle* h, const rsb_controls* controls, int32_t n);

rsb_status rsb_step(rsb_handle* h, int32_t ticks, void* stream);

rsb_status rsb_snapshot(rsb_handle* h, void* stream);
rsb_status rsb_build_obs(rsb_handle* h, void* stream);
rsb_status rsb_build_rewards_terminals(rsb_handle* h, int32_t step_ticks, void* stream);

rsb_status rsb_copy_obs(rsb_handle* h, float* out, size_t count);
rsb_status rsb_copy_masks(rsb_handle* h, uint8_t* out, size_t count);
rsb_status rsb_copy_rewards(rsb_handle* h, float* out, size_t count);
rsb_status rsb_copy_terminals(rsb_handle* h, uint8_t* out, size_t count);
rsb_status rsb_device_ptr(rsb_handle* h, int32_t which, void** out);

rsb_status rsb_get_cars(rsb_handle* h, rsb_car_state* out, int32_t n);
rsb_status rsb_set_cars(rsb_handle* h, const rsb_car_state* in, int32_t n);
rsb_status rsb_get_balls(rsb_handle* h, rsb_ball_state* out, int32_t n);
rsb_status rsb_set_balls(rsb_handle* h, const rsb_ball_state* in, int32_t n);
rsb_status rsb_get_pads(rsb_handle* h, rsb_pad_state* out, int32_t n);   /* n = arenas * 34 */
rsb_status rsb_set_pads(rsb_handle* h, const rsb_pad_state* in, int32_t n);
rsb_status rsb_get_arena_info(rsb_handle* h, rsb_arena_info* out, int32_t n);

/* One arena at a time (RocketSimCudaBatch::GetCarState / GetBallState / GetBoostPadStates /
 * GetArenaInfo / SetCarState / SetBallState / SetBoostPadStates, RocketSimCuda.h:349-378):
 * car is the slot within the arena (blue first), pads are 34 records in arena order.  The
 * getters gather the one record on the device and copy it (synchronising the handle's
 * stream); the setters launch one small kernel on the handle's stream with the same
 * conversion as the whole-batch setters, so other arenas are not touched. */
rsb_status rsb_get_car_at(rsb_handle* h, int32_t arena, int32_t car, rsb_car_state* out);
/* RocketSimCudaBatch::SetCarControls (RocketSimCuda.h:286): one car's controls, the others
 * unchanged; takes effect at the next rsb_step (ordered on the handle's stream). */
rsb_status rsb_set_car_controls_at(rsb_handle* h, int32_t arena, int32_t car, const rsb_controls* in);
rsb_status rsb_set_car_at(rsb_handle* h, int32_t arena, int32_t car, const rsb_car_state* in);
rsb_status rsb_get_ball_at(rsb_handle* h, int32_t arena, rsb_ball_state* out);
rsb_status rsb_set_ball_at(rsb_handle* h, int32_t arena, const rsb_ball_state* in);
rsb_status rsb_get_pads_at(rsb_handle* h, int32_t arena, rsb_pad_state* out);
rsb_status rsb_set_pads_at(rsb_handle* h, int32_t arena, const rsb_pad_state* in);
rsb_status rsb_get_arena_info_at(rsb_handle* h, int32_t arena, rsb_arena_info* out);

/* Ball prediction: BallPredTracker::ForceUpdateAllPred (RocketSim src/Sim/BallPredTracker/
 * BallPredTracker.cpp:80-88), the ball-only rollout that VantaObs reads at 1, 2 and 3 s
 * (RocketSimCudaObs.cuh:92-112), for every arena in one launch.  Each arena's ball goes through
 * GetState / SetState into a world of its own with no cars, which advances one tick at a time
 * with the batch's physics; out[a * n_slices + k] is the ball after slice_ticks[k] ticks
 * (1..8 slices, rising, at most 4096 ticks).  The arenas are only read.  With out non-null the
 * slices are copied to it (out_count = num_arenas * n_slices) and the stream is synchronised;
 * with out null they stay on the device (rsb_device_ptr, RSB_BUF_BALL_PRED).  The first call
 * allocates the device buffer for RSB_MAX_PRED_SLICES slices of every arena (60 B each), so
 * the RSB_BUF_BALL_PRED pointer stays the same for the life of the handle; each call
 * overwrites its first num_arenas * n_slices entries. */
#define RSB_MAX_PRED_SLICES 8
#define RSB_MAX_PRED_TICKS 4096
rsb_status rsb_predict_ball(rsb_handle* h, const int32_t* slice_ticks, int32_t n_slices, rsb_ball_state* out,
                            size_t out_count, void* stream);

/* One candidate launch configuration of the step kernel and its measured time. */
typedef struct rsb_tune_entry {
    int32_t min_blocks;   /* register budget: at least this many 128-thread blocks per SM */
    int32_t block;        /* threads per block (one arena per thread) */
    float ms;             /* best of two timed launches of `ticks` ticks */
    int32_t persistent;   /* 1: a grid whose warps claim 32 arenas at a time until none are left */
    int32_t warps_per_sm; /* persistent grids: warps resident per SM (0 = as many as fit) */
} rsb_tune_entry;

/* Times every launch configuration of the step kernel on a device copy of the current
 * arena state (the handle's own state is not advanced), keeps the fastest for later
 * rsb_step calls, and reports every candidate in out[0..cap).  Allocates the scratch copy
 * of the state on its first call.  No counterpart in the reference. */
rsb_status rsb_autotune(rsb_handle* h, int32_t ticks, rsb_tune_entry* out, int32_t cap, int32_t* count);
/* Selects a launch configuration (min_blocks, block, persistent as rsb_autotune reports them),
 * e.g. one tuned in an earlier run; RSB_ERR_INVALID if no such configuration exists. */
rsb_status rsb_set_step_config(rsb_handle* h, const rsb_tune_entry* cfg);

/* ---- learned culler (no counterpart in the reference) ----
 * A 3 -> 64 -> 64 -> 1 MLP (BF16 weights, FP32 accumulation) estimates the distance (uu)
 * from a point to the arena meshes; it is trained on the GPU by the library's own forward /
 * backward kernels on positions the simulation visits, and its margin is calibrated so that
 * the estimate minus the margin stays below the exact distance on every held-out point.
 * With cull_mode LEARNED / LEARNED_AUDIT and trained (or set) weights, every rsb_step first
 * marks the bodies whose static tests cannot find anything during the launch. */
#define RSB_CULLER_PARAMS 4481

typedef struct rsb_culler_config {
    int32_t train_points;     /* points the MLP is fitted on (e.g. 4,000,000) */
    int32_t heldout_points;   /* further points that calibrate the margin (e.g. 1,000,000) */
    float logged_fraction;    /* share of points taken from the logged body centres */
    float jitter_fraction;    /* share of logged near-surface centres moved by Gaussian jitter */
    float jitter_sigma;       /* uu (e.g. 150) */
    float near_surface;       /* uu: logged centres closer than this to a mesh get jittered */
    float target_cap;         /* uu: distances beyond this are clamped in the loss */
    int32_t epochs;
    int32_t batch;
    float lr;                 /* Adam, cosine-decayed */
    float over_weight;        /* loss weight of over-estimates (they widen the margin) */
    float margin_slack;       /* uu added to the calibrated margin */
    uint64_t seed;
} rsb_culler_config;

typedef struct rsb_culler_report {
    int32_t train_points, heldout_points, logged_points, epochs, steps;
    float final_loss;         /* mean weighted squared error (km^2) of the last epoch */
    float margin;             /* uu subtracted from the estimate */
    float heldout_mae;        /* uu, mean absolute error (distances capped at target_cap) */
    float heldout_max_over;   /* uu, largest over-estimate before the margin */
    int32_t heldout_misses;   /* held-out points where estimate - margin exceeds the exact distance */
    float heldout_car_clear;  /* share of held-out points whose bound clears a car's 8-tick reach */
    float train_ms;
} rsb_culler_report;

/* Appends the centre of every body (ball, cars) to the training log (up to 8M points). */
rsb_status rsb_culler_log(rsb_handle* h, void* stream);
/* Builds the point set, computes exact distances, trains, calibrates, and turns the bound on. */
rsb_status rsb_culler_train(rsb_handle* h, const rsb_culler_config* cfg, rsb_culler_report* out);
/* Switches between RSB_CULL_EXACT / _LEARNED / _LEARNED_AUDIT for later rsb_step calls. */
rsb_status rsb_set_cull_mode(rsb_handle* h, int32_t mode);
/* FP32 master weights (RSB_CULLER_PARAMS floats) and the calibrated margin (uu). */
rsb_status rsb_culler_get(rsb_handle* h, float* params, float* margin);
rsb_status rsb_culler_set(rsb_handle* h, const float* params, float margin);
/* Host buffers: exact distance to the meshes, the MLP estimate (before the margin), and the
 * loss gradient of the current weights over n points (the training kernel's reduction). */
rsb_status rsb_culler_distance(rsb_handle* h, const float* pts, int32_t n, float* out);
rsb_status rsb_culler_predict(rsb_handle* h, const float* pts, int32_t n, float* out);
rsb_status rsb_culler_gradients(rsb_handle* h, const float* pts, const float* target, int32_t n,
                                float over_weight, float* grad, float* loss);

/* The four CopyBuilt* calls of CudaEnvSet.cpp:163-166 in one: the observation rows, masks,
 * rewards and terminals queued on the handle's stream, then one synchronisation.  A NULL
 * destination is skipped.  Sizes are those of rsb_copy_obs / _masks / _rewards / _terminals. */
rsb_status rsb_copy_outputs(rsb_handle* h, float* obs, uint8_t* masks, float* rewards, uint8_t* terminals);

/* Page-locks (and releases) a caller's host buffer, so that the copies to and from it run at
 * full PCIe speed without staging (cudaHostRegister, portable to every device).  No
 * counterpart in the reference, whose host vectors are pageable.  Register a buffer once,
 * reuse it every step, and unregister it before freeing it. */
rsb_status rsb_host_register(void* ptr, size_t bytes);
rsb_status rsb_host_unregister(void* ptr);

/* ---- state ring: rewind a few arenas to an earlier state ----
 * Replaces the state ring of GGL::CudaEnvSet (GigaLearnCPP/src/public/GigaLearnCPP/Sim/
 * CudaEnvSet.h:100-125, CudaEnvSet.cpp:608-815).  The reference copies every car, ball and
 * pad state to the host at each capture (a device synchronisation plus a full-batch
 * download); here the slots live in device memory and a capture is three device-to-device
 * copies on the stream.  A restore picks the arenas and draws the position / velocity
 * jitter exactly as RestoreStateRingReplay / ApplyArenaSnap do (xorshift32 stream,
 * partial Fisher-Yates over the arena indices, cars then ball), then applies, on the
 * device, what the reference's SetCarState / SetBallState / SetBoostPadStates would: the
 * public state of the slot, jittered, written over the live arena (broadphase registration
 * and wheel values of the live cars are kept, as Car::SetState keeps them).  Arena counters
 * (tick count, episode ticks) are not rewound, as in the reference.  Call rsb_build_obs
 * afterwards if observations are needed (CudaEnvSet.cpp:800-806 does). */
typedef struct rsb_ring_config {
    int32_t depth;                  /* slots, >= 2 (10); 0 turns the ring off and frees it */
    int32_t capture_every;          /* env steps between captures in rsb_ring_maybe_capture (3) */
    float restore_fraction;         /* share of arenas per restore, clamped to [0.01, 0.05] (0.05) */
    int32_t max_arenas_per_restore; /* cap per restore, also <= 5 % of the arenas (64) */
    float fuzz_pos;                 /* uu of position jitter (25) */
    float fuzz_vel;                 /* uu/s of velocity jitter (80) */
    int32_t lookback_slots;         /* slots back from the newest capture, 1 .. depth-1 (7) */
    uint32_t seed;                  /* xorshift32 state of the restore draws (0xA5A5A5A5) */
} rsb_ring_config;

typedef struct rsb_ring_stats {
    int32_t depth, filled, write_idx, replay_disabled;
    uint64_t captures, restores, restore_calls;
} rsb_ring_stats;

/* The reference's defaults (CudaEnvSet.h:100-109, rng CudaEnvSet.h:164). */
rsb_status rsb_ring_default_config(rsb_ring_config* out);
/* ConfigureStateRing (CudaEnvSet.cpp:619-656): clamps the fields as the reference does and
 * allocates depth slots of the batch's car, ball and pad records (2,428 B per 3v3 arena per
 * slot).  Synchronises the handle's stream. */
rsb_status rsb_ring_configure(rsb_handle* h, const rsb_ring_config* cfg);
/* CaptureStateRingSlot (CudaEnvSet.cpp:669-696): the live records into the next slot. */
rsb_status rsb_ring_capture(rsb_handle* h, void* stream);
/* MaybeCaptureStateRing (CudaEnvSet.cpp:658-667): counts env steps, captures every
 * capture_every-th call. */
rsb_status rsb_ring_maybe_capture(rsb_handle* h, void* stream);
/* RestoreStateRingReplay (CudaEnvSet.cpp:755-815): negative restore_fraction / lookback_slots
 * / max_arenas take the configured values; *restored = arenas rewound (0 with fewer than two
 * captures, with the ring off, or once the reference's tripwire - more than 32 calls and
 * more than 4 per capture - has turned replay off). */
rsb_status rsb_ring_restore(rsb_handle* h, float restore_fraction, int32_t lookback_slots, float fuzz_scale,
                            int32_t max_arenas, int32_t* restored, void* stream);
rsb_status rsb_ring_stats_get(rsb_handle* h, rsb_ring_stats* out);

/* ---- GAE over a flat rollout buffer (no handle) ----
 * rsb_compute_gae replaces rsc::ComputeGAEOnDevice (RocketSimCuda/include/
 * RocketSimCudaTraining.h:17-30, RocketSimCuda/src/GAECuda.cu:247-300) with the same
 * arguments in the same order and the same results element for element:
 *   - terminals: 0 running, 1 NORMAL (episode end, bootstrap 0), 2 TRUNCATED (bootstrap from
 *     trunc_val_preds); every nonzero value ends an independent segment;
 *   - the k-th TRUNCATED step counted from the END of the buffer (k = 0 for the last one)
 *     bootstraps from trunc_val_preds[k] (the learner's CPU GAE::Compute,
 *     GigaLearnCPP/src/private/GigaLearnCPP/PPO/GAE.cpp:164, indexes them the other way
 *     round); a num_truncs that does not match the TRUNCATED steps reads nothing out of range
 *     (such a step bootstraps from 0);
 *   - val_preds holds T values, and one more (val_preds[T]) when terminals[T-1] == 0: the
 *     final step then bootstraps from it, as the reference does;
 *   - advantages, returns and target_values (= val_preds + advantages) are written for all T
 *     elements; *rew_clip_portion = (sum|r/std| - sum|clip(r/std)|) / max(sum|r/std|, 1e-7),
 *     summed in another order than the reference's atomics (equal within float rounding).
 * All pointers are device pointers; stream is a cudaStream_t as void* (NULL = legacy default
 * stream).  The library keeps a small per-device scratch (grown on demand, as the
 * reference's is); calls on one device are serialised on the host, and work queued on two
 * streams must not overlap.  Three kernel launches, no host synchronisation. */
typedef struct rsb_gae_params {
    float gamma;       /* 0.99 by default */
    float lambda;      /* 0.95 */
    float return_std;  /* > 0: rewards are divided by it (and clipped to +-clip_range if > 0) */
    float clip_range;
} rsb_gae_params;

rsb_status rsb_gae_default_params(rsb_gae_params* out);
rsb_status rsb_compute_gae(const float* rews, const int8_t* terminals, const float* val_preds,
                           const float* trunc_val_preds, int32_t num_truncs, float* advantages,
                           float* target_values, float* returns, float* rew_clip_portion, int32_t T,
                           const rsb_gae_params* params, void* stream);
/* The same on host buffers (the call site of the learner's CPU GAE::Compute,
 * GAE.h:8-12): copies in, computes on the current device, copies out, synchronises.
 * num_val_preds >= T, and >= T + 1 when terminals[T-1] == 0. */
rsb_status rsb_compute_gae_host(const float* rews, const int8_t* terminals, const float* val_preds,
                                int32_t num_val_preds, const float* trunc_val_preds, int32_t num_truncs,
                                float* advantages, float* target_values, float* returns,
                                float* rew_clip_portion, int32_t T, const rsb_gae_params* params);

/* Diagnostic (no counterpart in the reference): evaluates on device `device` the float
 * functions whose bits the simulation takes from the reference's CPU build, for n inputs:
 *   RSB_MATH_RSQRT_EST  x86 rsqrtss estimate of x (the table sampled from this host's CPU at
 *                       the first rsb_create on the device; RSB_ERR_STATE before that)
 *   RSB_MATH_SIN/COS/ASIN  sinf / cosf / asinf of x as the host C library returns them
 *   RSB_MATH_ATAN2      atan2f(x, y) (x is the y-coordinate, as in the C function)
 * y may be NULL except for RSB_MATH_ATAN2.  Host buffers; synchronous. */
enum { RSB_MATH_RSQRT_EST = 0, RSB_MATH_SIN = 1, RSB_MATH_COS = 2, RSB_MATH_ASIN = 3, RSB_MATH_ATAN2 = 4 };
rsb_status rsb_eval_refmath(int32_t fn, const float* x, const float* y, float* out, int64_t n, int32_t device);

rsb_status rsb_sync(rsb_handle* h);
rsb_status rsb_stats_get(rsb_handle* h, rsb_stats* out);
/* Copies the last error message (NUL-terminated, truncated to n). Safe with h == NULL
   (returns the last rsb_create failure). */
rsb_status rsb_last_error(const rsb_handle* h, char* buf, size_t n);

#ifdef __cplusplus
}
#endif
#endif /* RSB_H */
