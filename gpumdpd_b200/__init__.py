"""gpumdpd_b200 -- a B200-native DPD timestep engine with the command surface of GPUDPD.

The compute path is libdpd_b200.so (hand-written sm_100a CUDA behind a C ABI,
include/dpd_b200.h); this package is its Python host layer: ctypes bindings
(`capi`), the engine/batch/server mirrors (`engine`, `server`) and the seeded
synthetic inputs (`inputs`).
"""
from .capi import DpdError, load  # noqa: F401
from .engine import Batch, Engine  # noqa: F401
from .server import Server  # noqa: F401

__all__ = ["Engine", "Batch", "Server", "DpdError", "load"]
