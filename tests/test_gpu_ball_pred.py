"""Ball prediction on the device (rsb_predict_ball, BallPredTracker::ForceUpdateAllPred,
BallPredTracker.cpp:80-88): against the oracle's ball-only arenas, against the engine's own
ball-only batch, on the device buffer, and at 3v3 x 65,536."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_util import POS_ABS_UU, VEL_ABS_UU, max_excess, random_balls, random_cars, vec

pytestmark = pytest.mark.gpu

SLICES = [1, 120, 240, 360]


class _Dev:
    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": typestr, "version": 3}


def _synced_pair(pkg, oracle_lib, meshes_dir, n, seed):
    rsb = pkg.rsb
    eng = rsb.Batch(pkg.engine_library(), n, team_size=2, meshes_path=meshes_dir)
    ora = rsb.Batch(oracle_lib, n, team_size=2, meshes_path=meshes_dir, threads=8)
    cars = random_cars(rsb, ora.get_cars(), seed)
    balls = random_balls(rsb, n, seed + 1)
    for b in (eng, ora):
        b.set_cars(cars)
        b.set_balls(balls)
    return eng, ora


def test_prediction_matches_oracle(pkg, oracle_lib, meshes_dir):
    n = 512
    eng, ora = _synced_pair(pkg, oracle_lib, meshes_dir, n, 40)
    balls0, cars0 = eng.get_balls(), eng.get_cars()
    pe, po = eng.predict_ball(SLICES), ora.predict_ball(SLICES)
    assert eng.get_balls().tobytes() == balls0.tobytes() and eng.get_cars().tobytes() == cars0.tobytes()
    # one tick: the ball-only tolerances of the tick-by-tick ball test
    a, b = pe[:, 0], po[:, 0]
    assert max_excess(vec(a, "pos"), vec(b, "pos"), POS_ABS_UU) <= 0
    assert max_excess(vec(a, "vel"), vec(b, "vel"), VEL_ABS_UU) <= 0
    for k, t in enumerate(SLICES):
        d = np.linalg.norm(vec(pe[:, k], "pos") - vec(po[:, k], "pos"), axis=1)
        same = (pe[:, k].tobytes() == po[:, k].tobytes())
        print(f"PRED tick {t}: identical={int((d == 0).sum())}/{n} max_pos_diff={d.max():.3g} uu over1uu={int((d > 1).sum())} all_bytes_equal={same}")
        # the device's arithmetic is the reference's: every slice equal byte for byte
        assert same, f"tick {t}: {int((d != 0).sum())} balls differ, the largest by {d.max():.3g} uu"


def test_repeated_predictions_match_oracle(pkg, oracle_lib, meshes_dir):
    """BallPredTracker keeps its ball-only arena between updates (the oracle does too, with its
    Bullet world, tick count and broadphase registration); the engine starts every call from
    a fresh ball-only world.  Three calls in a row on different balls - flying, at rest on the
    floor, rolling, and the balls of a stepped batch - give the oracle's slices byte for byte."""
    rsb = pkg.rsb
    n = 256
    eng, ora = _synced_pair(pkg, oracle_lib, meshes_dir, n, 60)
    rest = random_balls(rsb, n, 61, rest_fraction=0.0)
    rest["pos"]["z"] = 93.15
    for c in "xyz":
        rest["vel"][c] = 0.0
        rest["ang_vel"][c] = 0.0
    rolling = rest.copy()
    rolling["vel"]["x"] = np.random.default_rng(62).uniform(-1500, 1500, n)
    rolling["vel"]["y"] = np.random.default_rng(63).uniform(-1500, 1500, n)
    for call, balls in enumerate((None, rest, rolling, "stepped")):
        if isinstance(balls, np.ndarray):
            for b in (eng, ora):
                b.set_balls(balls)
        elif balls == "stepped":
            # both sides take the stepped balls through the public state (uu): the engine's
            # records and the oracle's Bullet bodies then hold the same values
            ora.step(8)
            stepped = ora.get_balls()
            for b in (eng, ora):
                b.set_balls(stepped)
        pe, po = eng.predict_ball(SLICES), ora.predict_ball(SLICES)
        for k, t in enumerate(SLICES):
            d = np.linalg.norm(vec(pe[:, k], "pos") - vec(po[:, k], "pos"), axis=1)
            assert pe[:, k].tobytes() == po[:, k].tobytes(), (
                f"call {call}, tick {t}: {int((d > 0).sum())} balls differ, largest {d.max():.3g} uu")


def test_prediction_equals_ball_only_batch(pkg, meshes_dir):
    rsb = pkg.rsb
    n = 4096
    eng = rsb.Batch(pkg.engine_library(), n, team_size=3, meshes_path=meshes_dir)
    eng.reset_all(0x5EED0043, rsb.RSB_RESET_RANDOM_STATE)
    eng.set_balls(random_balls(rsb, n, 44))
    solo = rsb.Batch(pkg.engine_library(), n, team_size=0, meshes_path=meshes_dir)
    solo.set_balls(eng.get_balls())
    pred = eng.predict_ball(SLICES)
    t = 0
    for k, s in enumerate(SLICES):
        solo.step(s - t)
        t = s
        assert pred[:, k].tobytes() == solo.get_balls().tobytes(), f"slice {s}"


def test_device_buffer_holds_the_slices(pkg, meshes_dir):
    import torch

    rsb = pkg.rsb
    n = 1000
    eng = rsb.Batch(pkg.engine_library(), n, team_size=1, meshes_path=meshes_dir)
    eng.set_balls(random_balls(rsb, n, 45))
    host = eng.predict_ball([120, 240, 360])
    t = np.ascontiguousarray([120, 240, 360], np.int32)
    st = eng.lib.rsb_predict_ball(eng._h, t.ctypes.data_as(C.c_void_p), 3, None, 0, None)
    assert st == 0
    eng.sync()
    words = rsb.BALL_DTYPE.itemsize // 4
    dev = torch.as_tensor(_Dev(eng.device_ptr(rsb.RSB_BUF_BALL_PRED), (n * 3, words), "<f4"), device="cuda")
    assert dev.cpu().numpy().tobytes() == host.tobytes()


def test_prediction_at_3v3_x_65536(pkg, meshes_dir):
    import torch

    rsb = pkg.rsb
    n = 65536
    eng = rsb.Batch(pkg.engine_library(), n, team_size=3, meshes_path=meshes_dir)
    eng.reset_all(0x5EED0003, rsb.RSB_RESET_RANDOM_STATE)
    eng.predict_ball([120, 240, 360])  # warm-up
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    pred = eng.predict_ball([120, 240, 360])
    end.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    print(f"PRED 3v3 x {n}: 360 ticks in {ms:.1f} ms ({n * 360 / ms / 1e3:.3g} M ball-ticks/s, copy included)")
    for f in ("pos", "vel"):
        assert np.isfinite(vec(pred.reshape(-1), f)).all()
    z = pred["pos"]["z"]
    assert (z > 0.5 * 91.25).all() and (z < 2044 + 91.25).all()
    assert (np.abs(pred["pos"]["x"]) < 4096 + 92).all()
    info = eng.get_arena_info()
    assert (info["status"] == 0).all()
