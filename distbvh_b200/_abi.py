"""ctypes binding of libbvhg.so (include/bvhg.h) for tests and benchmarks.

This is plumbing over the C ABI, not a second implementation: every call goes to the CUDA library. Importing it
raises when the library is missing, so nothing can silently run without the native code.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbvhg.so")

OK, ERR_ARG, ERR_CUDA, ERR_OVERFLOW, ERR_TIMEOUT, ERR_STATE, ERR_NOMEM = range(7)
PLAIN_FP64, FILTER_FP32 = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1
REBUILD, REFIT = 0, 1
FLAG_STAGE_TIMING = 0x1
STAGES = ("bounds", "keys", "sort", "build", "traverse", "recheck", "output", "climb", "slabs", "fixup")

# Every entry point declared in include/bvhg.h.
EXPORTS = (
    "bvhg_config_default", "bvhg_create", "bvhg_destroy", "bvhg_object_create", "bvhg_object_destroy",
    "bvhg_set_elements", "bvhg_build", "bvhg_broadphase", "bvhg_self_collision", "bvhg_get_morton",
    "bvhg_get_kdops", "bvhg_get_kdops_f32", "bvhg_get_centroids", "bvhg_validate_tree", "bvhg_last_candidates",
    "bvhg_get_stage_times", "bvhg_launch_count", "bvhg_set_spin_limit", "bvhg_test_stall_sort", "bvhg_debug_normal",
    "bvhg_synchronize", "bvhg_last_error", "bvhg_status_string", "bvhg_radix_sort_noalloc",
    "bvhg_batch_broadphase", "bvhg_batch_autotune", "bvhg_sort_and_sweep", "bvhg_test_dense_stack",
    "bvhg_cluster", "bvhg_patch_pairs", "bvhg_patch_kdops", "bvhg_test_batch_form",
)


class Config(ctypes.Structure):
    _fields_ = [
        ("k", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("sort_digit_bits", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("epsilon", ctypes.c_double),
        ("stream", ctypes.c_void_p),
        ("spin_limit", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
    ]


class BvhgError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"bvhg status {status}: {message}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m distbvh_b200._build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    P, U64, I32, U32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint32
    sig = {
        "bvhg_config_default": (None, [ctypes.POINTER(Config)]),
        "bvhg_create": (I32, [ctypes.POINTER(P), ctypes.POINTER(Config)]),
        "bvhg_destroy": (I32, [P]),
        "bvhg_object_create": (I32, [P, ctypes.POINTER(I32)]),
        "bvhg_object_destroy": (I32, [P, I32]),
        "bvhg_set_elements": (I32, [P, I32, P, U32, P, U64, I32]),
        "bvhg_build": (I32, [P, I32, I32]),
        "bvhg_broadphase": (I32, [P, I32, I32, P, U64, ctypes.POINTER(U64), I32]),
        "bvhg_self_collision": (I32, [P, I32, P, U64, ctypes.POINTER(U64), I32]),
        "bvhg_get_morton": (I32, [P, I32, P, P, P, P]),
        "bvhg_get_kdops": (I32, [P, I32, P]),
        "bvhg_get_kdops_f32": (I32, [P, I32, P]),
        "bvhg_get_centroids": (I32, [P, I32, P]),
        "bvhg_validate_tree": (I32, [P, I32, ctypes.POINTER(U32)]),
        "bvhg_last_candidates": (I32, [P, ctypes.POINTER(U64)]),
        "bvhg_get_stage_times": (I32, [P, P, P]),
        "bvhg_launch_count": (I32, [P, ctypes.POINTER(U64)]),
        "bvhg_set_spin_limit": (I32, [P, U32]),
        "bvhg_test_stall_sort": (I32, [P, I32]),
        "bvhg_test_dense_stack": (I32, [P, I32]),
        "bvhg_test_batch_form": (I32, [P, U32, U32]),
        "bvhg_cluster": (I32, [P, I32, U32, P, P, I32]),
        "bvhg_patch_kdops": (I32, [P, I32, P, I32]),
        "bvhg_patch_pairs": (I32, [P, I32, I32, P, U64, ctypes.POINTER(U64), P, U64, ctypes.POINTER(U64), I32]),
        "bvhg_debug_normal": (I32, [I32, I32, I32, P, P, P]),
        "bvhg_synchronize": (I32, [P]),
        "bvhg_last_error": (ctypes.c_char_p, [P]),
        "bvhg_status_string": (ctypes.c_char_p, [I32]),
        "bvhg_radix_sort_noalloc": (I32, [P, P, P, U64, P]),
        "bvhg_batch_broadphase": (I32, [P, U32, P, P, I32, P, U64, P, P, I32]),
        "bvhg_batch_autotune": (I32, [P, U32, P, P, I32, ctypes.POINTER(U32), ctypes.POINTER(U32),
                                      ctypes.POINTER(ctypes.c_double)]),
        "bvhg_sort_and_sweep": (I32, [P, I32, I32, I32, P, U64, ctypes.POINTER(U64), ctypes.POINTER(I32), I32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be C-contiguous"
        return a.ctypes.data
    # torch tensors (device or host) and raw integers
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


def debug_normal(k, axis, comp):
    v = ctypes.c_double()
    lo = ctypes.c_float()
    hi = ctypes.c_float()
    st = lib.bvhg_debug_normal(k, axis, comp, ctypes.byref(v), ctypes.byref(lo), ctypes.byref(hi))
    if st != OK:
        raise BvhgError(st, "bad normal index")
    return v.value, lo.value, hi.value


class Context:
    """One bvhg_ctx: a CUDA device, a stream and the objects living on it."""

    def __init__(self, k=18, precision=PLAIN_FP64, digit_bits=8, epsilon=0.0, device=0, stream=None,
                 spin_limit=0, stage_timing=False):
        cfg = Config()
        lib.bvhg_config_default(ctypes.byref(cfg))
        cfg.k = k
        cfg.precision = precision
        cfg.sort_digit_bits = digit_bits
        cfg.device = device
        cfg.epsilon = epsilon
        cfg.stream = stream
        cfg.spin_limit = spin_limit
        cfg.flags = FLAG_STAGE_TIMING if stage_timing else 0
        self.cfg = cfg
        self.k = k
        self.precision = precision
        h = ctypes.c_void_p()
        st = lib.bvhg_create(ctypes.byref(h), ctypes.byref(cfg))
        if st != OK:
            raise BvhgError(st, "bvhg_create failed")
        self._h = h
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            lib.bvhg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != OK:
            raise BvhgError(st, lib.bvhg_last_error(self._h).decode())

    def object(self):
        o = ctypes.c_int32()
        self._check(lib.bvhg_object_create(self._h, ctypes.byref(o)))
        return o.value

    def set_elements(self, obj, xyz, verts_per_elem=None, gid=None, mem=None):
        """xyz: (n, V, 3) float64, a numpy array (host) or a CUDA torch tensor (device, borrowed)."""
        if mem is None:
            mem = MEM_DEVICE if (hasattr(xyz, "is_cuda") and xyz.is_cuda) else MEM_HOST
        if isinstance(xyz, np.ndarray):
            xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        n = xyz.shape[0]
        V = verts_per_elem if verts_per_elem is not None else xyz.shape[1]
        if gid is not None and isinstance(gid, np.ndarray):
            gid = np.ascontiguousarray(gid, dtype=np.uint64)
        self._keep[obj] = (xyz, gid)  # host copies are stream-ordered; keep the buffers alive
        self._check(lib.bvhg_set_elements(self._h, obj, _ptr(xyz), V, _ptr(gid), n, mem))

    def build(self, obj, mode=REBUILD):
        self._check(lib.bvhg_build(self._h, obj, mode))

    def broadphase(self, a, b, capacity=None):
        """Returns an (m, 2) uint64 array of (gid in a, gid in b)."""
        cnt = ctypes.c_uint64()
        if capacity is None:
            st = lib.bvhg_broadphase(self._h, a, b, None, 0, ctypes.byref(cnt), MEM_HOST)
            capacity = cnt.value
        out = np.empty((max(capacity, 1), 2), dtype=np.uint64)
        st = lib.bvhg_broadphase(self._h, a, b, out.ctypes.data, capacity, ctypes.byref(cnt), MEM_HOST)
        if st == ERR_OVERFLOW:
            raise BvhgError(st, f"overflow: {cnt.value} pairs")
        self._check(st)
        return out[: cnt.value]

    def sort_and_sweep(self, a, b, axis=-1):
        """Sort-and-sweep pairs (gid in a, gid in b) as an (m, 2) uint64 array, and the axis swept. The sweep runs
        once into a buffer sized by the last call's count (at least 65,536 pairs); only a larger result runs it
        again, into a buffer of the exact size."""
        cnt = ctypes.c_uint64()
        used = ctypes.c_int32()
        cap = max(65536, getattr(self, "_sweep_cap", 0))
        out = np.empty((cap, 2), dtype=np.uint64)
        st = lib.bvhg_sort_and_sweep(self._h, a, b, axis, out.ctypes.data, cap, ctypes.byref(cnt), ctypes.byref(used),
                                     MEM_HOST)
        if st == ERR_OVERFLOW:
            cap = cnt.value
            out = np.empty((cap, 2), dtype=np.uint64)
            st = lib.bvhg_sort_and_sweep(self._h, a, b, axis, out.ctypes.data, cap, ctypes.byref(cnt),
                                         ctypes.byref(used), MEM_HOST)
        self._check(st)
        self._sweep_cap = max(cap, cnt.value)
        return out[: cnt.value], used.value

    def sort_and_sweep_raw(self, a, b, axis, out_ptr, capacity, mem):
        cnt = ctypes.c_uint64()
        used = ctypes.c_int32()
        st = lib.bvhg_sort_and_sweep(self._h, a, b, axis, out_ptr, capacity, ctypes.byref(cnt), ctypes.byref(used), mem)
        return st, cnt.value, used.value

    def broadphase_raw(self, a, b, out_ptr, capacity, mem):
        cnt = ctypes.c_uint64()
        st = lib.bvhg_broadphase(self._h, a, b, out_ptr, capacity, ctypes.byref(cnt), mem)
        return st, cnt.value

    def self_collision(self, obj, capacity=None):
        cnt = ctypes.c_uint64()
        if capacity is None:
            lib.bvhg_self_collision(self._h, obj, None, 0, ctypes.byref(cnt), MEM_HOST)
            capacity = cnt.value
        out = np.empty((max(capacity, 1), 2), dtype=np.uint64)
        st = lib.bvhg_self_collision(self._h, obj, out.ctypes.data, capacity, ctypes.byref(cnt), MEM_HOST)
        if st == ERR_OVERFLOW:
            raise BvhgError(st, f"overflow: {cnt.value} pairs")
        self._check(st)
        return out[: cnt.value]

    def batch_broadphase(self, scenes, mode=0, capacity=None):
        """scenes: list of (obj_a, obj_b) (equal ids: self-collision). Returns a list of (m_s, 2) uint64 arrays."""
        a = np.ascontiguousarray([x[0] for x in scenes], dtype=np.int32)
        b = np.ascontiguousarray([x[1] for x in scenes], dtype=np.int32)
        n = len(scenes)
        counts = np.zeros(n, dtype=np.uint64)
        offsets = np.zeros(n, dtype=np.uint64)
        if capacity is None:
            st = lib.bvhg_batch_broadphase(self._h, n, a.ctypes.data, b.ctypes.data, mode, None, 0,
                                           counts.ctypes.data, offsets.ctypes.data, MEM_HOST)
            if st not in (0, ERR_OVERFLOW):
                self._check(st)
            capacity = int(counts.sum())
        out = np.empty((max(capacity, 1), 2), dtype=np.uint64)
        self._check(lib.bvhg_batch_broadphase(self._h, n, a.ctypes.data, b.ctypes.data, mode, out.ctypes.data,
                                              capacity, counts.ctypes.data, offsets.ctypes.data, MEM_HOST))
        return [out[int(o):int(o) + int(c)] for o, c in zip(offsets, counts)]

    def batch_broadphase_raw(self, a_ptr, b_ptr, n, mode, out_ptr, capacity, counts_ptr, mem):
        return lib.bvhg_batch_broadphase(self._h, n, a_ptr, b_ptr, mode, out_ptr, capacity, counts_ptr, None, mem)

    def batch_autotune(self, scenes, mode=0):
        """Picks the batching form's configuration: returns (groups (0 = per-object launches), lanes, ms)."""
        a = np.ascontiguousarray([x[0] for x in scenes], dtype=np.int32)
        b = np.ascontiguousarray([x[1] for x in scenes], dtype=np.int32)
        groups = ctypes.c_uint32()
        lanes = ctypes.c_uint32()
        ms = ctypes.c_double()
        self._check(lib.bvhg_batch_autotune(self._h, len(scenes), a.ctypes.data, b.ctypes.data, mode,
                                            ctypes.byref(groups), ctypes.byref(lanes), ctypes.byref(ms)))
        return groups.value, lanes.value, ms.value

    def cluster(self, obj, patches, n):
        """Patches of a built object: (bounds (patches + 1,) uint64, order (n,) uint32)."""
        bounds = np.empty(patches + 1, dtype=np.uint64)
        order = np.empty(max(n, 1), dtype=np.uint32)
        self._check(lib.bvhg_cluster(self._h, obj, patches, bounds.ctypes.data, order.ctypes.data, MEM_HOST))
        return bounds, order[:n]

    def patch_kdops(self, obj, patches):
        """Patch boxes of a clustered object: (patches, K/2, 2) float64 (min, max) per slab."""
        out = np.empty((patches, self.k // 2, 2), dtype=np.float64)
        self._check(lib.bvhg_patch_kdops(self._h, obj, out.ctypes.data, MEM_HOST))
        return out

    def patch_pairs(self, a, b):
        """Element pairs grouped by patch pair: (groups (g, 4) uint32 rows (patch a, patch b, first, count),
        pairs (m, 2) uint32 of (position in patch a, position in patch b))."""
        ng, npairs = ctypes.c_uint64(), ctypes.c_uint64()
        st = lib.bvhg_patch_pairs(self._h, a, b, None, 0, ctypes.byref(ng), None, 0, ctypes.byref(npairs), MEM_HOST)
        if st not in (OK, ERR_OVERFLOW):
            self._check(st)
        groups = np.empty((max(ng.value, 1), 4), dtype=np.uint32)
        pairs = np.empty((max(npairs.value, 1), 2), dtype=np.uint32)
        self._check(lib.bvhg_patch_pairs(self._h, a, b, groups.ctypes.data, ng.value, ctypes.byref(ng),
                                         pairs.ctypes.data, npairs.value, ctypes.byref(npairs), MEM_HOST))
        return groups[:ng.value], pairs[:npairs.value]

    def morton(self, obj, n):
        keys = np.empty(n, dtype=np.uint64)
        perm = np.empty(n, dtype=np.uint32)
        mn = np.empty(3)
        inv = np.empty(3)
        self._check(lib.bvhg_get_morton(self._h, obj, keys.ctypes.data, perm.ctypes.data, mn.ctypes.data,
                                        inv.ctypes.data))
        return keys, perm, mn, inv

    def kdops(self, obj, n):
        d = self.k // 2
        if self.precision == FILTER_FP32:
            out = np.empty((n, d, 2), dtype=np.float32)
            self._check(lib.bvhg_get_kdops_f32(self._h, obj, out.ctypes.data))
        else:
            out = np.empty((n, d, 2), dtype=np.float64)
            self._check(lib.bvhg_get_kdops(self._h, obj, out.ctypes.data))
        return out

    def centroids(self, obj, n):
        out = np.empty((n, 3), dtype=np.float64)
        self._check(lib.bvhg_get_centroids(self._h, obj, out.ctypes.data))
        return out

    def validate_tree(self, obj):
        depth = ctypes.c_uint32()
        self._check(lib.bvhg_validate_tree(self._h, obj, ctypes.byref(depth)))
        return depth.value

    def last_candidates(self):
        c = ctypes.c_uint64()
        self._check(lib.bvhg_last_candidates(self._h, ctypes.byref(c)))
        return c.value

    def stage_times(self):
        ms = np.zeros(len(STAGES))
        launches = np.zeros(len(STAGES), dtype=np.uint64)
        self._check(lib.bvhg_get_stage_times(self._h, ms.ctypes.data, launches.ctypes.data))
        return dict(zip(STAGES, ms.tolist())), dict(zip(STAGES, launches.tolist()))

    def launch_count(self):
        c = ctypes.c_uint64()
        self._check(lib.bvhg_launch_count(self._h, ctypes.byref(c)))
        return c.value

    def set_spin_limit(self, limit):
        self._check(lib.bvhg_set_spin_limit(self._h, limit))

    def test_stall_sort(self, enable):
        self._check(lib.bvhg_test_stall_sort(self._h, 1 if enable else 0))

    def test_batch_form(self, groups, lanes):
        self._check(lib.bvhg_test_batch_form(self._h, groups, lanes))

    def test_dense_stack(self, limit):
        self._check(lib.bvhg_test_dense_stack(self._h, limit))

    def synchronize(self):
        self._check(lib.bvhg_synchronize(self._h))
