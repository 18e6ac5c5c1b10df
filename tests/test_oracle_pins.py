"""Pins the oracle (the reference's CPU RocketSim and RLGymCPP env pieces, compiled from the
reference's own sources into oracle/_ref) against the expectations the reference's own
tests state, so that the GPU parity tests, which compare the engine with this oracle,
rest on a checked base.  CPU only.

Sources of the expectations:
  RocketSimCuda/tests/test_physics.cpp:44-50    ball vel.z ~ -5.4167 after one tick from rest
  RocketSimCuda/tests/test_physics.cpp:264-303  kickoff: orange = blue mirrored, both face the centre
  RocketSimCuda/tests/cpu_parity_harness.cpp:117-140, 166-210, 290-345  ballistic flight with
      drag against the closed-form / double-precision recurrence, ball speed clamp, air boost,
      demo respawn after 3 s at z = 36 with 33.3 boost
  RocketSimCuda/tests/reports/cpu_parity_report.txt  obs lengths 109 (1v1) / 167 (2v2)
  RLGymCPP DefaultAction.cpp:3-118              the 90-entry table and its masks
  RLGymCPP AdvancedObs.cpp:4-65                 the observation layout
  RocketSim.cpp:19-28, CollisionMeshFile.cpp:75-99  the 16 soccar mesh hashes

Goal detection follows the CPU (Arena::IsBallScored, Arena.cpp:949-957: |y| beyond the goal
line plus the ball radius, no width or height test); the reference GPU kernel's own
predicate (cpu_parity_harness.cpp:350-370) differs and is not the behaviour followed here.
"""
from __future__ import annotations

import glob
import os
import struct

import numpy as np
import pytest

from conftest import ORACLE_LIB


@pytest.fixture(scope="module")
def rsb(pkg):
    return pkg.rsb


def _batch(rsb, oracle_lib, meshes_dir, n=1, team_size=1, **kw):
    return rsb.Batch(oracle_lib, n, team_size=team_size, meshes_path=meshes_dir, threads=1, **kw)


def _set_identity(arr):
    for k, f in enumerate(("forward", "right", "up")):
        for j, c in enumerate("xyz"):
            arr["rot"][f][c] = 1.0 if k == j else 0.0


def _v(rec, field):
    return np.array([float(rec[field][c]) for c in "xyz"])


def test_ball_drop_one_tick(rsb, oracle_lib, meshes_dir):
    """test_physics.cpp:44-50 drops a ball from rest.  The CPU reference keeps a ball whose
    linear and angular velocities are exactly zero asleep (Arena::Step, Arena.cpp:721-726,
    RL's kickoff freeze), so the drop starts from a tiny downward velocity; a ball at exact
    rest stays put."""
    b = _batch(rsb, oracle_lib, meshes_dir, team_size=0)
    balls = b.get_balls()
    balls["pos"]["x"], balls["pos"]["y"], balls["pos"]["z"] = 0, 0, 500
    for c in "xyz":
        balls["vel"][c] = 0
        balls["ang_vel"][c] = 0
    b.set_balls(balls)
    b.step(1)
    assert b.get_balls()[0]["pos"]["z"] == np.float32(500.0)
    balls["vel"]["z"] = -1e-3
    b.set_balls(balls)
    b.step(1)
    s = b.get_balls()[0]
    assert s["pos"]["z"] < 500 and s["vel"]["z"] < 0
    assert abs(s["vel"]["z"] - (-5.4167)) < 0.1
    b.step(240)
    s = b.get_balls()[0]
    assert 0 < s["pos"]["z"] < 500


def test_ballistic_flight_matches_closed_form(rsb, oracle_lib, meshes_dir):
    """Gravity + linear drag in double precision, in Bullet's order: the damping scales the
    previous velocity (btDiscreteDynamicsWorld::predictUnconstraintMotion), the solver adds
    the gravity impulse, then the position integrates: v = v (1 - drag)^dt + g dt; p += v dt.
    Tolerance 1e-4 relative / 1e-2 uu absolute, as the reference's harness.  (The harness's
    own recurrence, cpu_parity_harness.cpp:131-141, damps after adding gravity, which is
    0.16 uu/s away from the CPU reference after one second.)"""
    b = _batch(rsb, oracle_lib, meshes_dir, team_size=0)
    balls = b.get_balls()
    p0, v0 = np.array([123.0, -45.0, 1500.0]), np.array([200.0, -150.0, 300.0])
    for k, c in enumerate("xyz"):
        balls["pos"][c], balls["vel"][c], balls["ang_vel"][c] = p0[k], v0[k], 0
    b.set_balls(balls)
    p, v = p0.copy(), v0.copy()
    g, dt, damp = np.array([0, 0, -650.0]), 1 / 120, (1 - 0.03) ** (1 / 120)
    for _ in range(120):
        v = v * damp + g * dt
        p = p + v * dt
    b.step(120)
    s = b.get_balls()[0]
    for got, ref in ((_v(s, "pos"), p), (_v(s, "vel"), v)):
        assert np.all(np.abs(got - ref) <= 1e-2 + 1e-4 * np.abs(ref)), (got, ref)


def test_ball_speed_clamp(rsb, oracle_lib, meshes_dir):
    b = _batch(rsb, oracle_lib, meshes_dir, team_size=0)
    balls = b.get_balls()
    for k, c in enumerate("xyz"):
        balls["pos"][c] = (0, 0, 1000)[k]
        balls["vel"][c] = (5000, 4000, 3000)[k]
    b.set_balls(balls)
    b.step(1)
    v = _v(b.get_balls()[0], "vel")
    assert abs(np.linalg.norm(v) - 6000.0) < 1e-2
    d0 = np.array([5000, 4000, 3000.0]) / np.linalg.norm([5000, 4000, 3000.0])
    assert np.dot(v / np.linalg.norm(v), d0) > 0.9999


def test_air_boost(rsb, oracle_lib, meshes_dir):
    b = _batch(rsb, oracle_lib, meshes_dir)
    cars = b.get_cars()
    _set_identity(cars)
    cars["pos"]["x"], cars["pos"]["y"], cars["pos"]["z"] = (0, 2000), (0, 0), (500, 17)
    for c in "xyz":
        cars["vel"][c] = 0
        cars["ang_vel"][c] = 0
    cars["boost"] = 100
    cars["is_on_ground"] = 0
    b.set_cars(cars)
    ctl = np.zeros(2, rsb.CONTROLS_DTYPE)
    ctl["boost"][0] = 1
    b.set_controls(ctl)
    for n_ticks, total in ((30, 30), (90, 120)):
        b.step(n_ticks)
        c = b.get_cars()[0]
        t = total / 120
        assert abs(c["vel"]["x"] - 3175 / 3 * t) <= 1e-2 + 1e-4 * 3175 / 3 * t
        assert abs(c["boost"] - (100 - 100 / 3 * t)) < 1e-3
        assert abs(c["vel"]["y"]) < 1e-3


def test_demo_respawn(rsb, oracle_lib, meshes_dir):
    b = _batch(rsb, oracle_lib, meshes_dir)
    cars = b.get_cars()
    cars["is_demoed"][0] = 1
    cars["demo_respawn_timer"][0] = 3.0
    b.set_cars(cars)
    for t in range(1, 400):
        b.step(1)
        c = b.get_cars()[0]
        if not c["is_demoed"]:
            break
    assert t == 360
    assert abs(c["pos"]["z"] - 36.0) < 1.0 and abs(c["boost"] - 100 / 3) < 1e-3
    assert abs(abs(c["pos"]["y"]) - 4608) < 1e-3 and abs(c["pos"]["x"]) in (2304.0, 2688.0)


@pytest.mark.parametrize("x,y,z,scored,team", [(0, 5220, 100, 1, 0), (0, 5200, 100, 0, -1), (0, -5220, 100, 1, 1),
                                                (0, 5000, 100, 0, -1), (1000, 5300, 100, 1, 0)])
def test_goal_detection_follows_cpu(rsb, oracle_lib, meshes_dir, x, y, z, scored, team):
    b = _batch(rsb, oracle_lib, meshes_dir, team_size=0)
    balls = b.get_balls()
    balls["pos"]["x"], balls["pos"]["y"], balls["pos"]["z"] = x, y, z
    b.set_balls(balls)
    info = b.get_arena_info()[0]
    assert info["goal_scored"] == scored and info["goal_team"] == team


def test_kickoff_orange_mirrors_blue(rsb, oracle_lib, meshes_dir):
    b = _batch(rsb, oracle_lib, meshes_dir, n=16)
    b.reset_all(7, rsb.RSB_RESET_KICKOFF)
    cars = b.get_cars()
    for a in range(16):
        blue, orange = cars[2 * a], cars[2 * a + 1]
        assert orange["pos"]["x"] == -blue["pos"]["x"] and orange["pos"]["y"] == -blue["pos"]["y"]
        fb, fo = _v(blue["rot"], "forward"), _v(orange["rot"], "forward")
        assert abs(fo[0] + fb[0]) < 0.05 and abs(fo[1] + fb[1]) < 0.05
        for c in (blue, orange):
            p, f = _v(c, "pos"), _v(c["rot"], "forward")
            assert -p[0] * f[0] - p[1] * f[1] > 0, "faces the centre"
            assert c["pos"]["z"] == np.float32(17.0) and abs(c["boost"] - 100 / 3) < 1e-4


def test_default_action_table(rsb, oracle_lib, engine_lib):
    ref = rsb.default_action_lut(oracle_lib)   # RLGymCPP DefaultAction, built from its sources
    eng = rsb.default_action_lut(engine_lib)
    assert ref.tobytes() == eng.tobytes()
    py = rsb.default_action_table()
    assert py.tobytes() == ref.tobytes()
    assert len(ref) == 90 and (ref["jump"] == 1).sum() == 18


def _expected_masks(lut, on_ground, boost, flip_or_jump):
    """DefaultAction::GetActionMask restated over the table."""
    n_ground = 24
    idx = np.arange(len(lut))
    ground = idx < n_ground
    air = (idx > n_ground) & (lut["jump"] == 0)
    air |= ground & (lut["throttle"] == lut["boost"].astype(np.float32)) & \
        ((lut["yaw"] != 0).astype(np.float32) == lut["handbrake"].astype(np.float32))
    m = ground.copy() if on_ground else air.copy()
    if boost == 0:
        m &= lut["boost"] == 0
    if flip_or_jump:
        m |= lut["jump"] == 1
    return m.astype(np.uint8)


def test_masks_and_obs_layout(rsb, oracle_lib, meshes_dir):
    lut = rsb.default_action_lut(oracle_lib)
    for ts, length in ((1, 109), (2, 167), (3, 225)):
        b = _batch(rsb, oracle_lib, meshes_dir, n=4, team_size=ts, rewards=rsb.default_rewards(oracle_lib))
        assert b.obs_stride == length
        b.reset_all(3, rsb.RSB_RESET_RANDOM_STATE)
        cars = b.get_cars()
        cars["boost"][0] = 0.0     # one car with an empty tank
        b.set_cars(cars)
        b.build_obs()
        obs, masks = b.copy_obs(), b.copy_masks()
        balls = b.get_balls()
        pads = b.get_pads()
        for a in range(4):
            ball = balls[a]
            for s in range(2 * ts):
                i = b.car_offset[a] + s
                c = cars[i]
                inv = np.array([-1, -1, 1.0]) if c["team"] else np.ones(3)
                row = obs[i]
                f32 = np.float32
                np.testing.assert_allclose(row[0:3], _v(ball, "pos") * inv * f32(1 / 5000), rtol=1e-6, atol=1e-7)
                np.testing.assert_allclose(row[3:6], _v(ball, "vel") * inv * f32(1 / 2300), rtol=1e-6, atol=1e-7)
                np.testing.assert_allclose(row[6:9], _v(ball, "ang_vel") * inv * f32(1 / 3), rtol=1e-6, atol=1e-7)
                assert not row[9:17].any(), "no previous action after a reset"
                assert np.all(row[17:51] == 1.0), "every pad available after a reset"
                assert np.all(pads["is_active"][a * 34:(a + 1) * 34] == 1)
                # own block: position, forward, up, velocity, angular velocity, boost, flags
                blk = row[51:80]
                np.testing.assert_allclose(blk[0:3], _v(c, "pos") * inv / 5000, rtol=1e-5, atol=1e-6)
                np.testing.assert_allclose(blk[3:6], _v(c["rot"], "forward") * inv, rtol=1e-6, atol=1e-7)
                np.testing.assert_allclose(blk[6:9], _v(c["rot"], "up") * inv, rtol=1e-6, atol=1e-7)
                np.testing.assert_allclose(blk[9:12], _v(c, "vel") * inv / 2300, rtol=1e-5, atol=1e-6)
                np.testing.assert_allclose(blk[12:15], _v(c, "ang_vel") * inv / 3, rtol=1e-5, atol=1e-6)
                assert blk[24] == np.float32(c["boost"] / np.float32(100))
                assert blk[25] == c["is_on_ground"] and blk[27] == c["is_demoed"] and blk[28] == c["has_jumped"]
                assert not row[length:].any()
                fj = bool(c["is_on_ground"]) or (not c["has_flipped"] and not c["has_double_jumped"]
                                                  and c["air_time_since_jump"] < 1.25)
                assert blk[26] == fj
                turtled = c["world_contact"] and c["world_contact_normal"]["z"] > 0.9
                exp = _expected_masks(lut, c["is_on_ground"], c["boost"], fj or turtled)
                assert np.array_equal(masks[i], exp), (ts, a, s)


def _mesh_hash(path):
    """CollisionMeshFile::UpdateHash: vertex coordinates converted to uint32 the way x86-64
    converts float to an unsigned 32-bit value (truncate toward zero, keep the low 32 bits)."""
    data = open(path, "rb").read()
    nt, nv = struct.unpack_from("<ii", data, 0)
    tris = np.frombuffer(data, np.int32, 3 * nt, 8).reshape(nt, 3)
    verts = np.frombuffer(data, np.float32, 3 * nv, 8 + 12 * nt).reshape(nv, 3)
    vals = (np.trunc(verts.astype(np.float64)).astype(np.int64) & 0xFFFFFFFF).astype(np.uint64)
    M = 0xFFFFFFFF
    h = (nv + nt * nv) & M
    for t in range(nt):
        for i in range(3):
            for j in range(3):
                cur = int(vals[tris[t, i], j])
                for _ in range(2):
                    cur = (((cur >> 16) ^ cur) * 0x45D9F3B) & M
                cur = (cur >> 16) ^ cur
                h ^= (cur + 0x9E3779B9 + ((h << 6) & M) + (h >> 2)) & M
    return h


def test_soccar_mesh_hashes(meshes_dir):
    expected = {0xA160BAF9, 0x2811EEE8, 0xB81AC8B9, 0x760358D3, 0x73AE4940, 0x918F4A4E, 0x1F8EE550, 0x255BA8C1,
                0x14B84668, 0xEC759EBF, 0x94FB0D5C, 0xDEA07102, 0xBD4FBEA8, 0x39A47F63, 0x3D79D25D, 0xD84C7A68}
    files = sorted(glob.glob(os.path.join(meshes_dir, "soccar", "mesh_*.cmf")))
    assert len(files) == 16
    assert {_mesh_hash(f) for f in files} == expected


def test_oracle_library_is_the_reference_build():
    assert os.path.exists(ORACLE_LIB)


def bounce_invariants(b, ticks=120):
    """Ball thrown down from 1,000 uu at 1,758 uu/s onto the floor (ball_floor_bounce_120t
    in RocketSimCuda/tests/reports/cpu_parity_report.txt): it bounces, does not tunnel through the
    floor (its centre stays above half its radius; Bullet's discrete contact lets it sink about
    11 uu at this speed before pushing it out), and its mechanical energy per unit mass never
    grows by more than 0.1 %."""
    balls = b.get_balls()
    _set_identity(balls)
    for k, c in enumerate("xyz"):
        balls["pos"][c], balls["vel"][c], balls["ang_vel"][c] = (0.0, 0.0, 1000.0)[k], (0.0, 0.0, -1757.84)[k], 0.0
    b.set_balls(balls)
    e0 = 0.5 * 1757.84 ** 2 + 650.0 * 1000.0  # 2.195e6, the report's E0
    min_z, max_e, bounced = 1e9, 0.0, False
    for _ in range(ticks):
        b.step(1)
        s = b.get_balls()[0]
        z, v = float(s["pos"]["z"]), _v(s, "vel")
        min_z = min(min_z, z)
        max_e = max(max_e, 0.5 * float(v @ v) + 650.0 * z)
        bounced |= v[2] > 0
    return bounced, min_z, max_e, e0


def test_ball_floor_bounce_invariants(rsb, oracle_lib, meshes_dir):
    bounced, min_z, max_e, e0 = bounce_invariants(_batch(rsb, oracle_lib, meshes_dir, team_size=0))
    assert bounced and min_z >= 0.5 * 91.25 and max_e <= e0 * 1.001, (bounced, min_z, max_e, e0)
