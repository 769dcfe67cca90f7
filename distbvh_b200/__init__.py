"""distbvh_b200 — a B200-native (sm_100a) per-rank element broadphase with distBVH's semantics.

The compute path is libbvhg.so (hand-written CUDA kernels behind the C ABI in include/bvhg.h). This package holds
its build recipe, a ctypes binding used by the tests and the benchmark, the synthetic workload generators, and
the C++ host API (host/bvhg/collision_world.hpp) that mirrors the reference's collision_world / collision_object.

The binding is loaded on first use of any of its names (distbvh_b200.Context, distbvh_b200.lib, ...), and that
first use raises ImportError when libbvhg.so is missing. Importing only the mesh generators
(`from distbvh_b200 import meshes`) does not load the CUDA library.
"""
_ABI_NAMES = (
    "OK", "ERR_ARG", "ERR_CUDA", "ERR_OVERFLOW", "ERR_TIMEOUT", "ERR_STATE", "ERR_NOMEM",
    "BvhgError", "Context", "EXPORTS", "FILTER_FP32", "MEM_DEVICE", "MEM_HOST", "PLAIN_FP64", "REBUILD", "REFIT",
    "STAGES", "debug_normal", "lib", "LIB_PATH",
)


def __getattr__(name):
    if name in _ABI_NAMES:
        from . import _abi
        return getattr(_abi, name)
    raise AttributeError(f"module 'distbvh_b200' has no attribute {name!r}")


def __dir__():
    return sorted(list(globals()) + list(_ABI_NAMES))
