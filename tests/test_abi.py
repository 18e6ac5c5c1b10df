"""C ABI checks that need no GPU: both libraries load and export every symbol that
include/rsb.h declares; the engine refuses to run without a CUDA device."""
from __future__ import annotations

import os

import numpy as np
import re

import pytest

from conftest import ORACLE_LIB, ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "rsb.h")).read()
    return sorted(set(re.findall(r"^rsb_status\s+(rsb_\w+)\s*\(", text, flags=re.M)))


def test_header_matches_binding(pkg):
    assert header_symbols() == sorted(pkg.rsb.ABI_SYMBOLS)


@pytest.mark.parametrize("which", ["engine", "oracle"])
def test_library_exports_every_symbol(pkg, which):
    lib = pkg.engine_library() if which == "engine" else pkg.rsb.load_library(ORACLE_LIB)
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_engine_without_gpu_fails_loudly(pkg, meshes_dir):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.rsb.RsbError) as e:
        pkg.rsb.Batch(pkg.engine_library(), 2, team_size=0, meshes_path=meshes_dir)
    assert e.value.code == -2  # RSB_ERR_CUDA: no CPU fallback exists


def test_oracle_rejects_bad_config(pkg, oracle_lib, meshes_dir):
    with pytest.raises(pkg.rsb.RsbError):
        pkg.rsb.Batch(oracle_lib, 0, team_size=1, meshes_path=meshes_dir)
    with pytest.raises(pkg.rsb.RsbError):
        pkg.rsb.Batch(oracle_lib, 1, team_size=4, meshes_path=meshes_dir)


def test_default_action_table_matches_engine(pkg):
    """The 90-action table from the engine's C ABI equals the Python enumeration."""
    rsb = pkg.rsb
    a = rsb.default_action_lut(pkg.engine_library())
    b = rsb.default_action_table()
    assert len(a) == rsb.RSB_NUM_ACTIONS == len(b)
    assert a.tobytes() == b.tobytes()


def test_default_action_table_shape(pkg):
    """24 ground actions first (no boost below full throttle), then 66 aerial ones."""
    lut = pkg.rsb.default_action_table()
    ground, air = lut[:24], lut[24:]
    assert (ground["pitch"] == 0).all() and (ground["jump"] == 0).all()
    assert (ground["yaw"] == ground["steer"]).all()
    assert ((ground["boost"] == 0) | (ground["throttle"] == 1)).all()
    assert (air["throttle"] == air["boost"]).all() and (air["steer"] == air["yaw"]).all()
    assert not ((air["jump"] == 1) & (air["yaw"] != 0)).any()
    assert len(np.unique(lut.tobytes())) == 1 and len({r.tobytes() for r in lut}) == 90


def test_pad_locations_match_reference(pkg):
    """The engine's pad order and locations (rsb_pad_locations) are RocketSim's arena pads:
    the big soccar pads, then the small ones (Arena.cpp:546-550), as the oracle reports them."""
    rsb = pkg.rsb
    a = rsb.pad_locations(pkg.engine_library())
    b = rsb.pad_locations(rsb.load_library(ORACLE_LIB))
    assert a.shape == (rsb.RSB_NUM_PADS, 3) and a.tobytes() == b.tobytes()
    assert (a[:6, 2] == 73).all() and (a[6:, 2] == 70).all()


def test_vanta_default_config(pkg):
    """BatchConfig's VantaObs defaults (RocketSimCuda.h:184-189) from both libraries, ball
    prediction on."""
    import ctypes as C

    rsb = pkg.rsb
    for lib in (pkg.engine_library(), rsb.load_library(ORACLE_LIB)):
        cfg = rsb.VantaConfig()
        assert lib.rsb_vanta_default_config(C.byref(cfg)) == 0
        assert (cfg.tick_skip, cfg.dodge_deadzone, cfg.only_closest_opp, cfg.predict_ball) == (8, 0.5, 0, 1)
