"""distbvh_b200 — a B200-native (sm_100a) per-rank element broadphase with distBVH's semantics.

The compute path is libbvhg.so (hand-written CUDA kernels behind the C ABI in include/bvhg.h). This package holds
its build recipe, a ctypes binding used by the tests and the benchmark, the synthetic workload generators, and
the C++ host API (host/include/bvh/*.hpp) that mirrors the reference's collision_world / collision_object.
"""
from ._abi import (  # noqa: F401
    BvhgError, Context, EXPORTS, FILTER_FP32, MEM_DEVICE, MEM_HOST, PLAIN_FP64, REBUILD, REFIT, STAGES, debug_normal,
    lib, LIB_PATH,
)
