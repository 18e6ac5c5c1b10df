"""B200-native batched RocketSim engine.

The engine itself is the CUDA library ``librsb.so`` (C ABI: include/rsb.h); this package
holds its build recipe and a thin Python binding (``rsb.Batch``) that mirrors the
reference batch simulator's methods.  There is no CPU execution path: creating a batch
without a CUDA device fails with ``RSB_ERR_CUDA``.
"""
from __future__ import annotations

import os

from . import rsb  # noqa: F401
from .rsb import Batch, RsbError, load_library  # noqa: F401

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "librsb.so")
DATA_DIR = os.path.join(PKG_DIR, "_data")
MESHES_DIR = os.path.join(DATA_DIR, "collision_meshes")


def engine_library():
    """Loads the CUDA engine; raises when it has not been built."""
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() (nvcc) first")
    return load_library(LIB_PATH)
