"""Python binding of the engine's C ABI (include/rsb.h).

The same binding drives any library that exports the rsb_* symbols: the CUDA
engine (``librsb.so`` in this package) and, in tests and the CPU-baseline leg of
the benchmark, the reference-backed oracle library.  Bulk state I/O goes through
numpy structured arrays whose dtypes mirror the C structs byte for byte.

The class mirrors the reference batch simulator's public methods
(RocketSimCuda/include/RocketSimCuda.h:258-396): ``create`` ~ Init + AddCar,
``reset_all`` ~ ResetAllArenas, ``set_actions`` ~ SetDiscreteActionsFromIndices,
``step`` ~ Step, ``build_obs`` ~ BuildAdvancedObsAndDefaultMasks,
``build_rewards_terminals`` ~ BuildRewardsAndTerminals, ``get_cars`` ~
GetAllCarStates and so on.  Errors raise :class:`RsbError` with the library's
message instead of being printed and ignored.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

RSB_MAX_CARS_PER_ARENA = 6
RSB_NUM_PADS = 34
RSB_NUM_ACTIONS = 90
RSB_STATIC_ACTIONS_MAX = 65536 * 6
RSB_OBS_BASE = 51
RSB_OBS_PER_CAR = 29

(RSB_BUF_OBS, RSB_BUF_MASKS, RSB_BUF_REWARDS, RSB_BUF_TERMINALS, RSB_BUF_CONTROLS, RSB_BUF_ACTIONS, RSB_BUF_BALL_PRED,
 RSB_BUF_VANTA_OBS) = range(8)
RSB_VANTA_OBS_SIZE = 366
RSB_MAX_PRED_SLICES = 8
RSB_MAX_PRED_TICKS = 4096
RSB_CULL_EXACT, RSB_CULL_LEARNED, RSB_CULL_LEARNED_AUDIT, RSB_CULL_VOXEL, RSB_CULL_VOXEL_AUDIT = 0, 1, 2, 3, 4
RSB_CULLER_PARAMS = 4481
RSB_RESET_KICKOFF, RSB_RESET_RANDOM_STATE, RSB_RESET_HIGH_CONTACT, RSB_RESET_CURRICULUM = 0, 1, 2, 3
RSB_MATH_RSQRT_EST, RSB_MATH_SIN, RSB_MATH_COS, RSB_MATH_ASIN, RSB_MATH_ATAN2 = range(5)
RSB_ARENA_NONFINITE, RSB_ARENA_ROW_OVERFLOW, RSB_ARENA_BVH_OVERFLOW, RSB_ARENA_CULL_MISS, RSB_ARENA_EPA_OVERFLOW = (
    1, 2, 4, 8, 16)

_STATUS = {
    -1: "RSB_ERR_INVALID", -2: "RSB_ERR_CUDA", -3: "RSB_ERR_NOMEM", -4: "RSB_ERR_MESH",
    -5: "RSB_ERR_STATE", -6: "RSB_ERR_TIMEOUT", -7: "RSB_ERR_UNSUPPORTED",
}


class RsbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS.get(code, code)}: {msg}")
        self.code = code


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class RotMat(C.Structure):
    _fields_ = [("forward", Vec3), ("right", Vec3), ("up", Vec3)]


class Controls(C.Structure):
    _fields_ = [("throttle", C.c_float), ("steer", C.c_float), ("pitch", C.c_float),
                ("yaw", C.c_float), ("roll", C.c_float), ("jump", C.c_uint8),
                ("boost", C.c_uint8), ("handbrake", C.c_uint8), ("pad_", C.c_uint8)]


class CarState(C.Structure):
    _fields_ = [
        ("pos", Vec3), ("rot", RotMat), ("vel", Vec3), ("ang_vel", Vec3),
        ("boost", C.c_float), ("time_spent_boosting", C.c_float),
        ("jump_time", C.c_float), ("flip_time", C.c_float), ("air_time", C.c_float),
        ("air_time_since_jump", C.c_float), ("supersonic_time", C.c_float),
        ("handbrake_val", C.c_float), ("auto_flip_timer", C.c_float),
        ("auto_flip_torque_scale", C.c_float), ("demo_respawn_timer", C.c_float),
        ("car_contact_cooldown", C.c_float), ("flip_rel_torque", Vec3),
        ("world_contact_normal", Vec3), ("car_contact_other_id", C.c_uint32),
        ("is_on_ground", C.c_uint8), ("has_jumped", C.c_uint8), ("has_double_jumped", C.c_uint8),
        ("has_flipped", C.c_uint8), ("is_flipping", C.c_uint8), ("is_jumping", C.c_uint8),
        ("is_supersonic", C.c_uint8), ("is_auto_flipping", C.c_uint8), ("is_demoed", C.c_uint8),
        ("world_contact", C.c_uint8), ("ball_hit_valid", C.c_uint8), ("team", C.c_uint8),
        ("wheels_with_contact", C.c_uint8 * 4), ("pad1_", C.c_uint32),
        ("ball_hit_tick", C.c_uint64), ("ball_hit_extra_tick", C.c_uint64),
        ("ball_hit_rel_pos", Vec3), ("ball_hit_ball_pos", Vec3), ("ball_hit_extra_vel", Vec3),
        ("last_controls", Controls), ("id", C.c_uint32), ("pad_", C.c_uint32), ("pad2_", C.c_uint32),
    ]


class BallState(C.Structure):
    _fields_ = [("pos", Vec3), ("rot", RotMat), ("vel", Vec3), ("ang_vel", Vec3)]


class PadState(C.Structure):
    _fields_ = [("is_active", C.c_uint8), ("pad_", C.c_uint8 * 3), ("cooldown", C.c_float),
                ("prev_locked_car_id", C.c_uint32)]


class ArenaInfo(C.Structure):
    _fields_ = [("tick_count", C.c_uint64), ("num_cars", C.c_int32), ("team_size", C.c_int32),
                ("goal_scored", C.c_int32), ("goal_team", C.c_int32),
                ("episode_ticks", C.c_int32), ("status", C.c_int32)]


class Mutators(C.Structure):
    _fields_ = [("gravity", Vec3)] + [(n, C.c_float) for n in (
        "car_mass", "car_world_friction", "car_world_restitution", "ball_mass", "ball_max_speed",
        "ball_drag", "ball_world_friction", "ball_world_restitution", "jump_accel",
        "jump_immediate_force", "boost_accel_ground", "boost_accel_air", "boost_used_per_second",
        "respawn_delay", "bump_cooldown_time", "boost_pad_cooldown_big", "boost_pad_cooldown_small",
        "car_spawn_boost_amount", "ball_hit_extra_force_scale", "bump_force_scale", "ball_radius")] + [
        ("unlimited_flips", C.c_uint8), ("unlimited_double_jumps", C.c_uint8),
        ("demo_mode", C.c_uint8), ("enable_team_demos", C.c_uint8),
        ("goal_base_threshold_y", C.c_float)]


class RewardConfig(C.Structure):
    _fields_ = [("w_goal", C.c_float), ("w_touch", C.c_float), ("w_vel_ball_to_goal", C.c_float),
                ("w_vel_player_to_ball", C.c_float), ("goal_concede_scale", C.c_float),
                ("team_spirit", C.c_float), ("opponent_scale", C.c_float), ("zero_sum", C.c_int32),
                ("episode_max_ticks", C.c_int32), ("no_touch_timeout_s", C.c_float)]


class Config(C.Structure):
    _fields_ = [("num_arenas", C.c_int32), ("team_size", C.c_int32),
                ("team_sizes", C.POINTER(C.c_int32)), ("tick_rate", C.c_float),
                ("tick_skip", C.c_int32), ("meshes_path", C.c_char_p),
                ("mutators", C.POINTER(Mutators)), ("rewards", C.POINTER(RewardConfig)),
                ("cull_mode", C.c_int32), ("cull_margin", C.c_float), ("seed", C.c_uint64),
                ("device", C.c_int32), ("threads", C.c_int32)]


class CullerConfig(C.Structure):
    _fields_ = [("train_points", C.c_int32), ("heldout_points", C.c_int32), ("logged_fraction", C.c_float),
                ("jitter_fraction", C.c_float), ("jitter_sigma", C.c_float), ("near_surface", C.c_float),
                ("target_cap", C.c_float), ("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float),
                ("over_weight", C.c_float), ("margin_slack", C.c_float), ("seed", C.c_uint64)]


class CullerReport(C.Structure):
    _fields_ = [("train_points", C.c_int32), ("heldout_points", C.c_int32), ("logged_points", C.c_int32),
                ("epochs", C.c_int32), ("steps", C.c_int32), ("final_loss", C.c_float), ("margin", C.c_float),
                ("heldout_mae", C.c_float), ("heldout_max_over", C.c_float), ("heldout_misses", C.c_int32),
                ("heldout_car_clear", C.c_float), ("train_ms", C.c_float)]


def culler_config(**kw) -> CullerConfig:
    """Defaults of the culler training (4M training and 1M held-out points, 150 uu jitter)."""
    c = CullerConfig(train_points=4_000_000, heldout_points=1_000_000, logged_fraction=0.45,
                     jitter_fraction=0.35, jitter_sigma=150.0, near_surface=600.0, target_cap=2500.0,
                     epochs=30, batch=65536, lr=3e-3, over_weight=4.0, margin_slack=2.0, seed=0x5EED0003)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class TuneEntry(C.Structure):
    _fields_ = [("min_blocks", C.c_int32), ("block", C.c_int32), ("ms", C.c_float), ("persistent", C.c_int32),
                ("warps_per_sm", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "ticks_simulated", "narrowphase_queries", "culled_queries", "missed_contacts",
        "solver_rows", "arenas_reverted", "status_bits_seen", "state_bytes_per_step")]


class VantaConfig(C.Structure):
    _fields_ = [("tick_skip", C.c_int32), ("dodge_deadzone", C.c_float), ("only_closest_opp", C.c_int32),
                ("predict_ball", C.c_int32)]


class RingConfig(C.Structure):
    _fields_ = [("depth", C.c_int32), ("capture_every", C.c_int32), ("restore_fraction", C.c_float),
                ("max_arenas_per_restore", C.c_int32), ("fuzz_pos", C.c_float), ("fuzz_vel", C.c_float),
                ("lookback_slots", C.c_int32), ("seed", C.c_uint32)]


class RingStats(C.Structure):
    _fields_ = [("depth", C.c_int32), ("filled", C.c_int32), ("write_idx", C.c_int32),
                ("replay_disabled", C.c_int32), ("captures", C.c_uint64), ("restores", C.c_uint64),
                ("restore_calls", C.c_uint64)]


class GaeParams(C.Structure):
    _fields_ = [("gamma", C.c_float), ("lam", C.c_float), ("return_std", C.c_float), ("clip_range", C.c_float)]


CAR_DTYPE = np.dtype(CarState)
BALL_DTYPE = np.dtype(BallState)
PAD_DTYPE = np.dtype(PadState)
INFO_DTYPE = np.dtype(ArenaInfo)
CONTROLS_DTYPE = np.dtype(Controls)

_P = C.c_void_p
_SIGS = {
    "rsb_default_mutators": [C.POINTER(Mutators)],
    "rsb_default_rewards": [C.POINTER(RewardConfig)],
    "rsb_create": [C.POINTER(Config), C.POINTER(_P)],
    "rsb_destroy": [_P],
    "rsb_layout": [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _P, _P],
    "rsb_obs_stride": [_P, C.POINTER(C.c_int32)],
    "rsb_reset_all": [_P, C.c_uint64, C.c_int32],
    "rsb_reset_arenas": [_P, _P, C.c_int32, C.c_uint64, C.c_int32],
    "rsb_set_action_lut": [_P, _P, C.c_int32],
    "rsb_default_action_lut": [_P, C.c_int32],
    "rsb_set_actions_host": [_P, _P, C.c_int32],
    "rsb_set_actions_host_static": [_P, _P, C.c_int32],
    "rsb_set_actions_device": [_P, _P, C.c_int32, _P],
    "rsb_set_controls": [_P, _P, C.c_int32],
    "rsb_step": [_P, C.c_int32, _P],
    "rsb_reset_done": [_P, C.c_uint64, C.c_int32, _P],
    "rsb_autotune": [_P, C.c_int32, _P, C.c_int32, _P],
    "rsb_set_step_config": [_P, _P],
    "rsb_culler_log": [_P, _P],
    "rsb_set_cull_mode": [_P, C.c_int32],
    "rsb_culler_train": [_P, _P, _P],
    "rsb_culler_get": [_P, _P, _P],
    "rsb_culler_set": [_P, _P, C.c_float],
    "rsb_culler_distance": [_P, _P, C.c_int32, _P],
    "rsb_culler_predict": [_P, _P, C.c_int32, _P],
    "rsb_culler_gradients": [_P, _P, _P, C.c_int32, C.c_float, _P, _P],
    "rsb_snapshot": [_P, _P],
    "rsb_build_obs": [_P, _P],
    "rsb_build_rewards_terminals": [_P, C.c_int32, _P],
    "rsb_copy_obs": [_P, _P, C.c_size_t],
    "rsb_copy_masks": [_P, _P, C.c_size_t],
    "rsb_copy_rewards": [_P, _P, C.c_size_t],
    "rsb_copy_terminals": [_P, _P, C.c_size_t],
    "rsb_device_ptr": [_P, C.c_int32, C.POINTER(_P)],
    "rsb_get_cars": [_P, _P, C.c_int32],
    "rsb_set_cars": [_P, _P, C.c_int32],
    "rsb_get_balls": [_P, _P, C.c_int32],
    "rsb_set_balls": [_P, _P, C.c_int32],
    "rsb_get_pads": [_P, _P, C.c_int32],
    "rsb_set_pads": [_P, _P, C.c_int32],
    "rsb_get_arena_info": [_P, _P, C.c_int32],
    "rsb_copy_outputs": [_P, _P, _P, _P, _P],
    "rsb_get_car_at": [_P, C.c_int32, C.c_int32, _P],
    "rsb_set_car_controls_at": [_P, C.c_int32, C.c_int32, _P],
    "rsb_set_car_at": [_P, C.c_int32, C.c_int32, _P],
    "rsb_get_ball_at": [_P, C.c_int32, _P],
    "rsb_predict_ball": [_P, _P, C.c_int32, _P, C.c_size_t, _P],
    "rsb_set_ball_at": [_P, C.c_int32, _P],
    "rsb_get_pads_at": [_P, C.c_int32, _P],
    "rsb_set_pads_at": [_P, C.c_int32, _P],
    "rsb_get_arena_info_at": [_P, C.c_int32, _P],
    "rsb_host_register": [_P, C.c_size_t],
    "rsb_host_unregister": [_P],
    "rsb_ring_default_config": [_P],
    "rsb_ring_configure": [_P, _P],
    "rsb_ring_capture": [_P, _P],
    "rsb_ring_maybe_capture": [_P, _P],
    "rsb_ring_restore": [_P, C.c_float, C.c_int32, C.c_float, C.c_int32, C.POINTER(C.c_int32), _P],
    "rsb_ring_stats_get": [_P, _P],
    "rsb_gae_default_params": [_P],
    "rsb_compute_gae": [_P, _P, _P, _P, C.c_int32, _P, _P, _P, _P, C.c_int32, _P, _P],
    "rsb_compute_gae_host": [_P, _P, _P, C.c_int32, _P, C.c_int32, _P, _P, _P, _P, C.c_int32, _P],
    "rsb_sync": [_P],
    "rsb_stats_get": [_P, C.POINTER(Stats)],
    "rsb_last_error": [_P, C.c_char_p, C.c_size_t],
    "rsb_eval_refmath": [C.c_int32, _P, _P, _P, C.c_int64, C.c_int32],
    "rsb_set_reset_curriculum": [_P, C.c_float, C.c_float, C.c_float, C.c_float],
    "rsb_env_graph_capture": [_P, _P, C.c_int32, C.c_int32, C.c_uint64],
    "rsb_vanta_default_config": [C.POINTER(VantaConfig)],
    "rsb_vanta_configure": [_P, C.POINTER(VantaConfig)],
    "rsb_build_vanta_obs": [_P, _P],
    "rsb_copy_vanta_obs": [_P, _P, C.c_size_t],
    "rsb_pad_locations": [_P],
    "rsb_env_graph_launch": [_P, _P],
}

#: every symbol include/rsb.h declares (checked by the ABI tests)
ABI_SYMBOLS = tuple(_SIGS.keys())

_LIBS: dict[str, C.CDLL] = {}


def load_library(path: str) -> C.CDLL:
    """Loads (once) a library exporting the rsb_* ABI and declares its signatures."""
    path = os.path.abspath(path)
    if path in _LIBS:
        return _LIBS[path]
    lib = C.CDLL(path, mode=C.RTLD_LOCAL)
    for name, args in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = C.c_int32
    _LIBS[path] = lib
    return lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def default_mutators(lib: C.CDLL) -> Mutators:
    m = Mutators()
    lib.rsb_default_mutators(C.byref(m))
    return m


def default_rewards(lib: C.CDLL, **overrides) -> RewardConfig:
    """rsb_default_rewards, then the given fields replaced (e.g. zero_sum=0b1111)."""
    r = RewardConfig()
    st = lib.rsb_default_rewards(C.byref(r))
    if st != 0:
        raise RsbError(st, "rsb_default_rewards failed")
    for k, v in overrides.items():
        setattr(r, k, v)
    return r


def pad_locations(lib: C.CDLL) -> np.ndarray:
    """rsb_pad_locations: the 34 pad locations (x, y, z) in the order of the pad-state arrays."""
    out = np.zeros((RSB_NUM_PADS, 3), np.float32)
    st = lib.rsb_pad_locations(_ptr(out))
    if st != 0:
        raise RsbError(st, _global_error(lib))
    return out


def default_action_lut(lib: C.CDLL) -> np.ndarray:
    lut = np.zeros(RSB_NUM_ACTIONS, CONTROLS_DTYPE)
    st = lib.rsb_default_action_lut(_ptr(lut), RSB_NUM_ACTIONS)
    if st != 0:
        raise RsbError(st, "rsb_default_action_lut failed")
    return lut


def gae_params(lib: C.CDLL, gamma: float | None = None, lam: float | None = None, return_std: float | None = None,
               clip_range: float | None = None) -> GaeParams:
    """rsb_gae_default_params (gamma 0.99, lambda 0.95, no standardisation), then overrides."""
    p = GaeParams()
    st = lib.rsb_gae_default_params(C.byref(p))
    if st != 0:
        raise RsbError(st, "rsb_gae_default_params failed")
    for k, v in (("gamma", gamma), ("lam", lam), ("return_std", return_std), ("clip_range", clip_range)):
        if v is not None:
            setattr(p, k, v)
    return p


def compute_gae_device(lib: C.CDLL, rews: int, terminals: int, val_preds: int, trunc_val_preds: int,
                       num_truncs: int, advantages: int, target_values: int, returns: int, rew_clip_portion: int,
                       T: int, params: GaeParams, stream: int = 0):
    """rsb_compute_gae on device pointers (ints), the drop-in for rsc::ComputeGAEOnDevice
    (RocketSimCuda/include/RocketSimCudaTraining.h:17-30): float32 rewards / values, int8
    terminals (1 NORMAL, 2 TRUNCATED), val_preds[T] read when the final step is not terminal."""
    st = lib.rsb_compute_gae(_P(rews or None), _P(terminals or None), _P(val_preds or None),
                             _P(trunc_val_preds or None), num_truncs, _P(advantages or None),
                             _P(target_values or None), _P(returns or None), _P(rew_clip_portion or None), T,
                             C.byref(params), _P(stream or None))
    if st != 0:
        raise RsbError(st, _global_error(lib))


def compute_gae(lib: C.CDLL, rews, terminals, val_preds, trunc_val_preds=None, params: GaeParams | None = None):
    """rsb_compute_gae_host on numpy arrays: (advantages, target_values, returns, rew_clip_portion).
    Same arguments as the learner's GAE::Compute (GigaLearnCPP/src/private/GigaLearnCPP/PPO/GAE.h:8-12)
    but the device function's conventions (truncation values counted from the buffer's end)."""
    r = np.ascontiguousarray(rews, np.float32)
    t = np.ascontiguousarray(terminals, np.int8)
    v = np.ascontiguousarray(val_preds, np.float32)
    tv = np.ascontiguousarray(trunc_val_preds if trunc_val_preds is not None else np.zeros(0), np.float32)
    n = len(r)
    if len(t) != n:
        raise ValueError("rews and terminals differ in length")
    params = params or gae_params(lib)
    adv, tgt, ret = (np.empty(n, np.float32) for _ in range(3))
    clip = np.zeros(1, np.float32)
    st = lib.rsb_compute_gae_host(_ptr(r), _ptr(t), _ptr(v), len(v), _ptr(tv) if len(tv) else None, len(tv),
                                  _ptr(adv), _ptr(tgt), _ptr(ret), _ptr(clip), n, C.byref(params))
    if st != 0:
        raise RsbError(st, _global_error(lib))
    return adv, tgt, ret, float(clip[0])


def eval_refmath(lib: C.CDLL, fn: int, x, y=None, device: int = 0) -> np.ndarray:
    """rsb_eval_refmath on numpy arrays (float32): the device's restated rsqrtss / sinf / cosf /
    asinf / atan2f(x, y)."""
    x = np.ascontiguousarray(x, np.float32)
    yy = None if y is None else np.ascontiguousarray(y, np.float32)
    out = np.empty_like(x)
    st = lib.rsb_eval_refmath(fn, _ptr(x), _ptr(yy) if yy is not None else None, _ptr(out), len(x), device)
    if st != 0:
        raise RsbError(st, _global_error(lib))
    return out


def _global_error(lib: C.CDLL) -> str:
    buf = C.create_string_buffer(512)
    lib.rsb_last_error(None, buf, len(buf))
    return buf.value.decode(errors="replace")


def default_action_table() -> np.ndarray:
    """The collector's 90-entry discrete action table built in Python (same enumeration as
    RLGymCPP DefaultAction.cpp:3-60), for callers that have no engine library loaded."""
    rows = []
    for throttle in (-1, 0, 1):
        for steer in (-1, 0, 1):
            for boost in (0, 1):
                for handbrake in (0, 1):
                    if boost == 1 and throttle != 1:
                        continue
                    rows.append((throttle, steer, 0, steer, 0, 0, boost, handbrake))
    for pitch in (-1, 0, 1):
        for yaw in (-1, 0, 1):
            for roll in (-1, 0, 1):
                for jump in (0, 1):
                    for boost in (0, 1):
                        if jump == 1 and yaw != 0:
                            continue
                        if pitch == roll == jump == 0:
                            continue
                        handbrake = int(jump == 1 and (pitch != 0 or yaw != 0 or roll != 0))
                        rows.append((boost, yaw, pitch, yaw, roll, jump, boost, handbrake))
    lut = np.zeros(len(rows), CONTROLS_DTYPE)
    for i, r in enumerate(rows):
        for f, v in zip(("throttle", "steer", "pitch", "yaw", "roll", "jump", "boost", "handbrake"), r):
            lut[i][f] = v
    return lut


class Batch:
    """N arenas behind one rsb handle."""

    def __init__(self, lib: C.CDLL | str, num_arenas: int, team_size: int | None = 2,
                 team_sizes=None, meshes_path: str = "", tick_skip: int = 8,
                 mutators: Mutators | None = None, rewards: RewardConfig | None = None,
                 cull_mode: int = RSB_CULL_EXACT, cull_margin: float = 0.0, seed: int = 0,
                 device: int = 0, threads: int = 0):
        self.lib = load_library(lib) if isinstance(lib, str) else lib
        self._h = C.c_void_p()
        cfg = Config()
        cfg.num_arenas = num_arenas
        cfg.team_size = team_size or 0
        self._team_sizes = None
        if team_sizes is not None:
            self._team_sizes = np.ascontiguousarray(team_sizes, np.int32)
            cfg.team_sizes = self._team_sizes.ctypes.data_as(C.POINTER(C.c_int32))
        cfg.tick_rate = 120.0
        cfg.tick_skip = tick_skip
        cfg.meshes_path = meshes_path.encode()
        self._mut = mutators
        if mutators is not None:
            cfg.mutators = C.pointer(mutators)
        self._rew = rewards
        if rewards is not None:
            cfg.rewards = C.pointer(rewards)
        cfg.cull_mode = cull_mode
        cfg.cull_margin = cull_margin
        cfg.seed = seed
        cfg.device = device
        cfg.threads = threads
        st = self.lib.rsb_create(C.byref(cfg), C.byref(self._h))
        if st != 0:
            raise RsbError(st, self._error(None))
        na, nc = C.c_int32(), C.c_int32()
        self._check(self.lib.rsb_layout(self._h, C.byref(na), C.byref(nc), None, None))
        self.num_arenas, self.num_cars = na.value, nc.value
        self.car_offset = np.zeros(self.num_arenas + 1, np.int32)
        self.team_size = np.zeros(self.num_arenas, np.int32)
        self._check(self.lib.rsb_layout(self._h, None, None, _ptr(self.car_offset), _ptr(self.team_size)))
        stride = C.c_int32()
        self._check(self.lib.rsb_obs_stride(self._h, C.byref(stride)))
        self.obs_stride = stride.value

    # ---------------------------------------------------------------- plumbing
    def _error(self, h) -> str:
        buf = C.create_string_buffer(512)
        self.lib.rsb_last_error(h, buf, 512)
        return buf.value.decode(errors="replace")

    def _check(self, st: int):
        if st != 0:
            raise RsbError(st, self._error(self._h))

    def close(self):
        for a in getattr(self, "_pinned", []):
            self.lib.rsb_host_unregister(C.c_void_p(a.ctypes.data))
        self._pinned = []
        if self._h:
            self.lib.rsb_destroy(self._h)
            self._h = C.c_void_p()

    def pin(self, a: np.ndarray) -> np.ndarray:
        """Page-locks a host array for fast copies (rsb_host_register); it stays registered
        until the batch is closed."""
        a = np.ascontiguousarray(a)
        self._check_global(self.lib.rsb_host_register(C.c_void_p(a.ctypes.data), a.nbytes))
        if not hasattr(self, "_pinned"):
            self._pinned = []
        self._pinned.append(a)
        return a

    def pinned_outputs(self) -> dict:
        """Page-locked host arrays for the observation rows, masks, rewards and terminals,
        allocated once; copy_outputs() fills them in place every step."""
        return {"obs": self.pin(np.zeros((self.num_cars, self.obs_stride), np.float32)),
                "masks": self.pin(np.zeros((self.num_cars, RSB_NUM_ACTIONS), np.uint8)),
                "rewards": self.pin(np.zeros(max(1, self.num_cars), np.float32)),
                "terminals": self.pin(np.zeros(self.num_arenas, np.uint8))}

    def copy_outputs(self, bufs: dict) -> dict:
        """rsb_copy_outputs: the four output buffers into `bufs` (see pinned_outputs), one
        synchronisation."""
        p = {k: (C.c_void_p(bufs[k].ctypes.data) if k in bufs else None)
             for k in ("obs", "masks", "rewards", "terminals")}
        if "obs" in bufs:
            assert bufs["obs"].size == self.num_cars * self.obs_stride
        self._check(self.lib.rsb_copy_outputs(self._h, p["obs"], p["masks"], p["rewards"], p["terminals"]))
        return bufs

    def _check_global(self, st: int):
        if st != 0:
            raise RsbError(st, _global_error(self.lib))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- control
    def reset_all(self, seed: int, mode: int = RSB_RESET_KICKOFF):
        self._check(self.lib.rsb_reset_all(self._h, seed, mode))

    def reset_arenas(self, idx, seed: int, mode: int = RSB_RESET_KICKOFF):
        a = np.ascontiguousarray(idx, np.int32)
        self._check(self.lib.rsb_reset_arenas(self._h, _ptr(a), len(a), seed, mode))

    def env_graph_capture(self, d_actions: int, tick_skip: int, reset_mode: int, seed: int):
        """rsb_env_graph_capture: one env step (actions from the device buffer d_actions) as a graph."""
        self._check(self.lib.rsb_env_graph_capture(self._h, C.c_void_p(d_actions), tick_skip, reset_mode, seed))

    def env_graph_launch(self, stream: int | None = None):
        self._check(self.lib.rsb_env_graph_launch(self._h, C.c_void_p(stream or 0)))

    def vanta_configure(self, **overrides) -> VantaConfig:
        """rsb_vanta_configure with the reference's defaults (tickSkip 8, dodge deadzone 0.5, all
        three opponents, ball prediction on) and the given fields; clears the builder's state."""
        cfg = VantaConfig()
        self._check_global(self.lib.rsb_vanta_default_config(C.byref(cfg)))
        for k, v in overrides.items():
            setattr(cfg, k, v)
        self._check(self.lib.rsb_vanta_configure(self._h, C.byref(cfg)))
        return cfg

    def build_vanta_obs(self, stream: int | None = None):
        self._check(self.lib.rsb_build_vanta_obs(self._h, C.c_void_p(stream or 0)))

    def copy_vanta_obs(self) -> np.ndarray:
        out = np.zeros((self.num_cars, RSB_VANTA_OBS_SIZE), np.float32)
        self._check(self.lib.rsb_copy_vanta_obs(self._h, _ptr(out), out.size))
        return out

    def set_reset_curriculum(self, kickoff_w: float, fuzzed_w: float, aerial_w: float, chase_w: float = 0.0):
        self._check(self.lib.rsb_set_reset_curriculum(self._h, kickoff_w, fuzzed_w, aerial_w, chase_w))

    def reset_done(self, seed: int, mode: int = RSB_RESET_KICKOFF, stream: int | None = None):
        """Resets the arenas whose terminal flag is set (device-side, stream-ordered)."""
        self._check(self.lib.rsb_reset_done(self._h, seed, mode, C.c_void_p(stream or 0)))

    def set_action_lut(self, lut: np.ndarray):
        lut = np.ascontiguousarray(lut, CONTROLS_DTYPE)
        self._check(self.lib.rsb_set_action_lut(self._h, _ptr(lut), len(lut)))

    def set_actions(self, idx):
        a = np.ascontiguousarray(idx, np.int32)
        self._check(self.lib.rsb_set_actions_host(self._h, _ptr(a), len(a)))

    def set_actions_static(self, idx):
        """rsb_set_actions_host_static: stages the indices in the library's static device
        array (no allocation on this path; see include/rsb.h)."""
        a = np.ascontiguousarray(idx, np.int32)
        self._check(self.lib.rsb_set_actions_host_static(self._h, _ptr(a), len(a)))

    def set_actions_device(self, dev_ptr: int, n: int, stream: int | None = None):
        self._check(self.lib.rsb_set_actions_device(self._h, C.c_void_p(dev_ptr), n, C.c_void_p(stream or 0)))

    def set_controls(self, controls: np.ndarray):
        c = np.ascontiguousarray(controls, CONTROLS_DTYPE)
        self._check(self.lib.rsb_set_controls(self._h, _ptr(c), len(c)))

    def step(self, ticks: int, stream: int | None = None):
        self._check(self.lib.rsb_step(self._h, ticks, C.c_void_p(stream or 0)))

    def snapshot(self, stream: int | None = None):
        self._check(self.lib.rsb_snapshot(self._h, C.c_void_p(stream or 0)))

    def build_obs(self, stream: int | None = None):
        self._check(self.lib.rsb_build_obs(self._h, C.c_void_p(stream or 0)))

    def build_rewards_terminals(self, step_ticks: int, stream: int | None = None):
        self._check(self.lib.rsb_build_rewards_terminals(self._h, step_ticks, C.c_void_p(stream or 0)))

    def autotune(self, ticks: int = 8) -> list[dict]:
        """rsb_autotune: times the step kernel's launch configurations, keeps the fastest."""
        out = (TuneEntry * 64)()
        n = C.c_int32()
        self._check(self.lib.rsb_autotune(self._h, ticks, out, 64, C.byref(n)))
        return [{"min_blocks": e.min_blocks, "block": e.block, "ms": e.ms, "persistent": e.persistent,
                 "warps_per_sm": e.warps_per_sm} for e in out[:min(n.value, 64)]]

    def set_step_config(self, min_blocks: int, block: int, persistent: bool = False, warps_per_sm: int = 0):
        """rsb_set_step_config: pins a launch configuration of the step kernel."""
        e = TuneEntry(min_blocks=min_blocks, block=block, ms=0.0, persistent=1 if persistent else 0,
                      warps_per_sm=warps_per_sm)
        self._check(self.lib.rsb_set_step_config(self._h, C.byref(e)))

    # ---------------------------------------------------------------- learned culler
    def set_cull_mode(self, mode: int):
        self._check(self.lib.rsb_set_cull_mode(self._h, mode))

    def culler_log(self, stream: int | None = None):
        self._check(self.lib.rsb_culler_log(self._h, C.c_void_p(stream or 0)))

    def culler_train(self, cfg: CullerConfig | None = None) -> dict:
        cfg = cfg or culler_config()
        rep = CullerReport()
        self._check(self.lib.rsb_culler_train(self._h, C.byref(cfg), C.byref(rep)))
        return {n: getattr(rep, n) for n, _ in CullerReport._fields_}

    def culler_get(self):
        w = np.zeros(RSB_CULLER_PARAMS, np.float32)
        m = C.c_float()
        self._check(self.lib.rsb_culler_get(self._h, _ptr(w), C.byref(m)))
        return w, m.value

    def culler_set(self, params, margin: float):
        w = np.ascontiguousarray(params, np.float32)
        self._check(self.lib.rsb_culler_set(self._h, _ptr(w), margin))

    def culler_distance(self, pts) -> np.ndarray:
        p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        out = np.zeros(len(p), np.float32)
        self._check(self.lib.rsb_culler_distance(self._h, _ptr(p), len(p), _ptr(out)))
        return out

    def culler_predict(self, pts) -> np.ndarray:
        p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        out = np.zeros(len(p), np.float32)
        self._check(self.lib.rsb_culler_predict(self._h, _ptr(p), len(p), _ptr(out)))
        return out

    def culler_gradients(self, pts, target, over_weight: float = 4.0):
        p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(target, np.float32)
        g = np.zeros(RSB_CULLER_PARAMS, np.float32)
        loss = C.c_float()
        self._check(self.lib.rsb_culler_gradients(self._h, _ptr(p), _ptr(t), len(p), over_weight, _ptr(g),
                                                  C.byref(loss)))
        return g, loss.value

    # ---------------------------------------------------------------- one arena
    def get_car(self, arena: int, car: int) -> np.ndarray:
        out = np.zeros(1, CAR_DTYPE)
        self._check(self.lib.rsb_get_car_at(self._h, arena, car, _ptr(out)))
        return out[0]

    def set_car(self, arena: int, car: int, state):
        a = np.ascontiguousarray(np.asarray(state, CAR_DTYPE).reshape(1))
        self._check(self.lib.rsb_set_car_at(self._h, arena, car, _ptr(a)))

    def get_ball(self, arena: int) -> np.ndarray:
        out = np.zeros(1, BALL_DTYPE)
        self._check(self.lib.rsb_get_ball_at(self._h, arena, _ptr(out)))
        return out[0]

    def set_ball(self, arena: int, state):
        a = np.ascontiguousarray(np.asarray(state, BALL_DTYPE).reshape(1))
        self._check(self.lib.rsb_set_ball_at(self._h, arena, _ptr(a)))

    def get_arena_pads(self, arena: int) -> np.ndarray:
        out = np.zeros(RSB_NUM_PADS, PAD_DTYPE)
        self._check(self.lib.rsb_get_pads_at(self._h, arena, _ptr(out)))
        return out

    def set_arena_pads(self, arena: int, pads):
        a = np.ascontiguousarray(np.asarray(pads, PAD_DTYPE))
        assert a.size == RSB_NUM_PADS
        self._check(self.lib.rsb_set_pads_at(self._h, arena, _ptr(a)))

    def get_arena_info_at(self, arena: int) -> np.ndarray:
        out = np.zeros(1, INFO_DTYPE)
        self._check(self.lib.rsb_get_arena_info_at(self._h, arena, _ptr(out)))
        return out[0]

    # ---------------------------------------------------------------- state ring
    def ring_configure(self, **overrides) -> RingConfig:
        """rsb_ring_configure with the reference's defaults (depth 10, capture every 3 env
        steps, 5 % of the arenas, 25 uu / 80 uu/s jitter, 7 slots back) and the given fields."""
        cfg = RingConfig()
        self._check(self.lib.rsb_ring_default_config(C.byref(cfg)))
        for k, v in overrides.items():
            setattr(cfg, k, v)
        self._ring_cfg = cfg
        self._check(self.lib.rsb_ring_configure(self._h, C.byref(cfg)))
        return cfg

    def ring_capture(self, stream: int | None = None):
        self._check(self.lib.rsb_ring_capture(self._h, C.c_void_p(stream or 0)))

    def ring_maybe_capture(self, stream: int | None = None):
        self._check(self.lib.rsb_ring_maybe_capture(self._h, C.c_void_p(stream or 0)))

    def ring_restore(self, restore_fraction: float = -1.0, lookback_slots: int = -1, fuzz_scale: float = 1.0,
                     max_arenas: int = -1, stream: int | None = None) -> int:
        n = C.c_int32()
        self._check(self.lib.rsb_ring_restore(self._h, restore_fraction, lookback_slots, fuzz_scale, max_arenas,
                                              C.byref(n), C.c_void_p(stream or 0)))
        return n.value

    def ring_stats(self) -> dict:
        st = RingStats()
        self._check(self.lib.rsb_ring_stats_get(self._h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in RingStats._fields_}

    def sync(self):
        self._check(self.lib.rsb_sync(self._h))

    # ---------------------------------------------------------------- buffers
    def copy_obs(self) -> np.ndarray:
        out = np.zeros((self.num_cars, self.obs_stride), np.float32)
        self._check(self.lib.rsb_copy_obs(self._h, _ptr(out), out.size))
        return out

    def copy_masks(self) -> np.ndarray:
        out = np.zeros((self.num_cars, RSB_NUM_ACTIONS), np.uint8)
        self._check(self.lib.rsb_copy_masks(self._h, _ptr(out), out.size))
        return out

    def copy_rewards(self) -> np.ndarray:
        out = np.zeros(self.num_cars, np.float32)
        self._check(self.lib.rsb_copy_rewards(self._h, _ptr(out), out.size))
        return out

    def copy_terminals(self) -> np.ndarray:
        out = np.zeros(self.num_arenas, np.uint8)
        self._check(self.lib.rsb_copy_terminals(self._h, _ptr(out), out.size))
        return out

    def device_ptr(self, which: int) -> int:
        p = C.c_void_p()
        self._check(self.lib.rsb_device_ptr(self._h, which, C.byref(p)))
        return p.value or 0

    # ---------------------------------------------------------------- state
    def get_cars(self) -> np.ndarray:
        out = np.zeros(self.num_cars, CAR_DTYPE)
        self._check(self.lib.rsb_get_cars(self._h, _ptr(out), self.num_cars))
        return out

    def set_cars(self, cars: np.ndarray):
        c = np.ascontiguousarray(cars, CAR_DTYPE)
        self._check(self.lib.rsb_set_cars(self._h, _ptr(c), len(c)))

    def get_balls(self) -> np.ndarray:
        out = np.zeros(self.num_arenas, BALL_DTYPE)
        self._check(self.lib.rsb_get_balls(self._h, _ptr(out), self.num_arenas))
        return out

    def predict_ball(self, slice_ticks=(120, 240, 360), to_host: bool = True, stream=None):
        """BallPredTracker's ball-only rollout of every arena's ball (BallPredTracker.cpp:80-88):
        [num_arenas, len(slice_ticks)] ball states after each slice's tick count.  With
        to_host False the slices stay in the device buffer RSB_BUF_BALL_PRED and None is
        returned (ordered on `stream`, not synchronised)."""
        t = np.ascontiguousarray(slice_ticks, np.int32)
        if not to_host:
            self._check(self.lib.rsb_predict_ball(self._h, _ptr(t), len(t), None, 0, C.c_void_p(stream or 0)))
            return None
        out = np.zeros((self.num_arenas, len(t)), BALL_DTYPE)
        self._check(self.lib.rsb_predict_ball(self._h, _ptr(t), len(t), _ptr(out), out.size, C.c_void_p(stream or 0)))
        return out

    def set_balls(self, balls: np.ndarray):
        b = np.ascontiguousarray(balls, BALL_DTYPE)
        self._check(self.lib.rsb_set_balls(self._h, _ptr(b), len(b)))

    def get_pads(self) -> np.ndarray:
        out = np.zeros(self.num_arenas * RSB_NUM_PADS, PAD_DTYPE)
        self._check(self.lib.rsb_get_pads(self._h, _ptr(out), len(out)))
        return out

    def set_pads(self, pads: np.ndarray):
        p = np.ascontiguousarray(pads, PAD_DTYPE)
        self._check(self.lib.rsb_set_pads(self._h, _ptr(p), len(p)))

    def get_arena_info(self) -> np.ndarray:
        out = np.zeros(self.num_arenas, INFO_DTYPE)
        self._check(self.lib.rsb_get_arena_info(self._h, _ptr(out), self.num_arenas))
        return out

    def stats(self) -> dict:
        s = Stats()
        self._check(self.lib.rsb_stats_get(self._h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in Stats._fields_}
