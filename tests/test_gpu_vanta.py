"""VantaObs rows (rsb_build_vanta_obs) against the reference's own device builder.

The reference tree has no CPU VantaObs; its GPU transcription (RocketSimCuda/src/VantaObsGpu.cuh)
is compiled from the reference tree into oracle/_ref/libvantaref.so (oracle/vanta_pin.cu) and fed
the engine's state after every env step: cars, ball, pads, tick counts and the ball-prediction
slices (the engine's own, pinned separately by tests/test_gpu_ball_pred.py).  Both builders keep
state between builds (pad timers, demo timers, the players' action timers), so the two run side
by side over many env steps, with random actions, random pad states, demoed cars and arena
resets, and every one of the 366 floats of every row must be bit-identical after every step.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PIN = os.path.join(ROOT, "oracle", "_ref", "libvantaref.so")


@pytest.fixture(scope="module")
def pin():
    if not os.path.exists(PIN):
        pytest.fail(f"{PIN} is missing: build the oracle (make -C oracle vanta)")
    lib = C.CDLL(PIN)
    lib.vantaref_create.restype = C.c_void_p
    lib.vantaref_create.argtypes = [C.c_int32, C.c_int32]
    lib.vantaref_destroy.argtypes = [C.c_void_p]
    lib.vantaref_reset.restype = C.c_int32
    lib.vantaref_reset.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.vantaref_build.restype = C.c_int32
    lib.vantaref_build.argtypes = [C.c_void_p] + [C.c_void_p] * 7 + [C.c_int32, C.c_float, C.c_int32, C.c_void_p]
    return lib


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _run(pkg, pin, meshes_dir, n, seed, steps=24, team_size=None, team_sizes=None, predict=1, only_closest=0,
         deadzone=0.5):
    rsb = pkg.rsb
    lib = pkg.engine_library()
    eng = rsb.Batch(lib, n, team_size=team_size, team_sizes=team_sizes, meshes_path=meshes_dir)
    eng.set_action_lut(rsb.default_action_lut(lib))
    eng.reset_all(seed, rsb.RSB_RESET_RANDOM_STATE)
    rng = np.random.default_rng(seed)
    pads = eng.get_pads()
    pads["is_active"] = rng.random(len(pads)) < 0.7
    pads["cooldown"] = np.where(pads["is_active"], 0.0, rng.uniform(0, 10, len(pads))).astype(np.float32)
    eng.set_pads(pads)
    eng.vanta_configure(tick_skip=8, dodge_deadzone=deadzone, only_closest_opp=only_closest, predict_ball=predict)
    max_cars = int(np.diff(eng.car_offset).max())
    h = pin.vantaref_create(n, max_cars)
    assert h
    xyz = np.ascontiguousarray(rsb.pad_locations(lib), np.float32)
    off = np.ascontiguousarray(eng.car_offset, np.int32)
    compared = 0
    try:
        for step in range(steps):
            eng.set_actions(rng.integers(0, rsb.RSB_NUM_ACTIONS, eng.num_cars).astype(np.int32))
            eng.step(8)
            if step % 6 == 3:
                # demo a few cars on both sides (the state both builders read)
                cars = eng.get_cars()
                pick = rng.random(len(cars)) < 0.1
                cars["is_demoed"][pick] = 1
                eng.set_cars(cars)
            if step % 8 == 5:
                idx = np.sort(rng.choice(n, max(1, n // 10), replace=False)).astype(np.int32)
                eng.reset_arenas(idx, seed + step, rsb.RSB_RESET_RANDOM_STATE)
                assert pin.vantaref_reset(h, _ptr(idx), len(idx)) == 0
            eng.build_vanta_obs()
            got = eng.copy_vanta_obs()
            cars, balls, pads = eng.get_cars(), eng.get_balls(), eng.get_pads()
            ticks = np.ascontiguousarray(eng.get_arena_info()["tick_count"], np.uint64)
            pred = np.ascontiguousarray(eng.predict_ball((120, 240, 360))) if predict else None
            want = np.zeros_like(got)
            st = pin.vantaref_build(h, _ptr(cars), _ptr(off), _ptr(balls), _ptr(pads), _ptr(xyz), _ptr(pred),
                                    _ptr(ticks), 8, deadzone, only_closest, _ptr(want))
            assert st == 0, st
            same = got.view(np.uint32) == want.view(np.uint32)
            if not same.all():
                r, c = np.argwhere(~same)[0]
                raise AssertionError(f"step {step}: {int((~same).sum())} values differ; first row {r} column {c}: "
                                     f"{got[r, c]!r} vs reference {want[r, c]!r}")
            compared += got.size
    finally:
        pin.vantaref_destroy(h)
        eng.close()
    return compared


@pytest.mark.parametrize("team_size", [1, 2, 3])
def test_vanta_rows_match_reference_builder(pkg, pin, meshes_dir, team_size):
    assert _run(pkg, pin, meshes_dir, 384, 100 + team_size, team_size=team_size) > 0


def test_vanta_rows_ragged_batch(pkg, pin, meshes_dir):
    ts = np.array([1 + (a * 7) % 3 for a in range(300)], np.int32)
    assert _run(pkg, pin, meshes_dir, 300, 7, team_sizes=ts) > 0


def test_vanta_rows_options(pkg, pin, meshes_dir):
    """No ball prediction (zero slices), only the closest opponent, another dodge deadzone."""
    assert _run(pkg, pin, meshes_dir, 256, 21, steps=16, team_size=3, predict=0, only_closest=1, deadzone=0.3) > 0


def test_vanta_requires_configuration(pkg, meshes_dir):
    rsb = pkg.rsb
    b = rsb.Batch(pkg.engine_library(), 8, team_size=1, meshes_path=meshes_dir)
    with pytest.raises(rsb.RsbError):
        b.build_vanta_obs()
    with pytest.raises(rsb.RsbError):
        b.vanta_configure(tick_skip=0)
    b.vanta_configure()
    b.build_vanta_obs()
    rows = b.copy_vanta_obs()
    assert rows.shape == (b.num_cars, rsb.RSB_VANTA_OBS_SIZE) and np.isfinite(rows).all()
    b.close()
