"""The engine's physics, compiled for the host, against the reference on the CPU.

The physics headers are built with g++ into a host harness (tests/cpp/host_engine.cpp) and
run beside the oracle (the reference's own RocketSim, oracle/_ref/librsref.so) from identical
seeded states and controls, one tick at a time, free-running for 480 ticks.  Every byte of
every car, ball and boost-pad state must be equal after every tick: this shows that the
restated algorithm is the reference's, operation for operation, including the rsqrtss
estimate and the C library's sin / cos / atan2 / asin (which the host build takes from the
CPU and the library directly; the device reproduces them, see tests/test_refmath.py).

Two things are outside the comparison, both because the reference's own results depend on
the process, not on the simulation's inputs:
  * arenas whose cars the reference visits in another order than the engine (its car set is
    an unordered_set hashed by heap address; gpu_util.reference_reverse_order);
  * an arena after a demolished car respawns in it: RocketSim draws the respawn spot from a
    process-global random engine (Car::Respawn, Car.cpp:43-56).
"""
from __future__ import annotations

import numpy as np
import pytest

from host_util import build_host_engine
from parity_util import run_lockstep

TICKS = 480


@pytest.fixture(scope="module")
def host_lib(pkg):
    return pkg.rsb.load_library(build_host_engine())


@pytest.mark.parametrize("team_size", [1, 2, 3])
def test_host_build_is_bit_exact_over_480_free_ticks(pkg, host_lib, oracle_lib, meshes_dir, team_size):
    compared, differed, respawned, first = run_lockstep(pkg.rsb, pkg, host_lib, oracle_lib, meshes_dir, team_size,
                                                        128, seed=300 + 10 * team_size, ticks=TICKS)
    print(f"team size {team_size}: {compared} arenas compared, {respawned} left out after a respawn, "
          f"{differed} differed")
    assert compared >= 90
    assert differed == 0, f"first difference: arena {first[0]} at tick {first[1]}"


def test_host_build_ragged_batch_is_bit_exact(pkg, host_lib, oracle_lib, meshes_dir):
    sizes = np.array([1, 2, 3] * 32, np.int32)
    compared, differed, respawned, first = run_lockstep(pkg.rsb, pkg, host_lib, oracle_lib, meshes_dir, None,
                                                        len(sizes), seed=77, ticks=240, team_sizes=sizes)
    assert compared >= 80
    assert differed == 0, f"first difference: arena {first[0]} at tick {first[1]}"


def test_refmath_table_form_on_this_cpu(pkg):
    """The engine reproduces rsqrtss from a 2 x 4096 table sampled on the host; its check of
    the CPU's estimate must pass here for the host build to be equal to the device build."""
    import ctypes as C
    lib = C.CDLL(build_host_engine())
    fn = lib.rsb_host_rsqrt_table
    fn.restype = C.c_int32
    fn.argtypes = [C.c_void_p]
    tab = np.zeros(2 * 4096, np.uint32)
    assert fn(tab.ctypes.data) == 1
    # the estimate is within its documented relative error of 1.5 * 2^-12
    x = (1 + np.arange(4096) / 4096.0)
    for p in (0, 1):
        est = tab[p * 4096:(p + 1) * 4096].view(np.float32).astype(np.float64)
        exact = 1 / np.sqrt(x * 2 ** p)
        assert np.abs(est / exact - 1).max() <= 1.5 * 2.0 ** -12
