"""Shared fixtures.

`-m gpu` tests run the CUDA engine on a B200 and compare it with the oracle (the
reference's own CPU RocketSim, built from its sources into oracle/_ref by
oracle/Makefile).  `-m "not gpu"` tests cover the oracle, the host logic and the C ABI
of the built library without a GPU.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "emy-s-framework_b200")
ORACLE_LIB = os.path.join(ROOT, "oracle", "_ref", "librsref.so")


def load_pkg():
    name = "emy_s_framework_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); compares the engine with the oracle")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def meshes_dir(pkg):
    d = pkg.MESHES_DIR
    if not os.path.isdir(os.path.join(d, "soccar")):
        pytest.fail(f"arena meshes are not staged under {d}: run __graft_entry__.build()")
    return d


@pytest.fixture(scope="session")
def oracle_lib(pkg):
    if not os.path.exists(ORACLE_LIB):
        pytest.fail(f"{ORACLE_LIB} missing: run `make -C oracle` (needs the reference sources)")
    return pkg.rsb.load_library(ORACLE_LIB)


@pytest.fixture(scope="session")
def engine_lib(pkg):
    return pkg.engine_library()
