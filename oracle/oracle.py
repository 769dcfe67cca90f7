"""ctypes wrapper of the CPU oracle (oracle/liboracle.so, built from oracle/bvh_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use it. The product library (distbvh_b200) never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False):
    src = os.path.join(HERE, "bvh_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "liboracle.so"], check=True)
    return LIB


def _load():
    build()
    lib = ctypes.CDLL(LIB)
    P, U64, I64, I32, U32, D = (ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32,
                                ctypes.c_double)
    sig = {
        "orc_normals": (I32, [I32, P]),
        "orc_project": (D, [P, P]),
        "orc_kdops": (I32, [P, U32, U64, I32, D, P]),
        "orc_centroids": (None, [P, U32, U64, P]),
        "orc_morton_bounds": (None, [P, U64, I32, P, P]),
        "orc_quantize64": (None, [P, P, P, P]),
        "orc_quantize32": (None, [P, P, P, P]),
        "orc_morton64": (U64, [U64, U64, U64]),
        "orc_morton32": (U32, [U32, U32, U32]),
        "orc_morton_keys": (None, [P, U64, P, P, P]),
        "orc_exclusive_scan_i64": (None, [P, U64]),
        "orc_radix_sort_1bit_u64": (None, [P, P, U64]),
        "orc_radix_sort_1bit_u32": (None, [P, P, U64]),
        "orc_stable_sort_perm_u64": (None, [P, U64, P]),
        "orc_overlap": (I32, [P, P, I32]),
        "orc_pairs_brute": (I64, [P, U64, P, U64, I32, P, U64]),
        "orc_self_pairs_brute": (I64, [P, U64, I32, P, U64]),
        "orc_pairs_tree": (I64, [P, P, U64, P, P, U64, I32, P, U64]),
        "orc_self_pairs_tree": (I64, [P, P, U64, I32, P, U64]),
        "orc_tree_node_count": (I64, [P, P, U64, I32]),
        "orc_max_variant_axis": (I32, [P, U64, P, U64]),
        "orc_sort_and_sweep": (I64, [P, U64, P, U64, I32, I32, P, U64]),
        "orc_pipeline": (I64, [P, U64, P, U64, U32, I32, D, I32, P, P, U64]),
        "orc_max_threads": (I32, []),
        "orc_morton_cluster": (None, [P, U64, P, P, U32, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def normals(k):
    out = np.zeros((13, 3))
    c = lib.orc_normals(k, out.ctypes.data)
    return out[:c]


def kdops(xyz, k, eps=0.0):
    """(n, V, 3) float64 -> (n, K/2, 2) FP64 slabs as kdop_base::from_vertices."""
    xyz = _c(xyz, np.float64)
    n, V = xyz.shape[0], xyz.shape[1]
    out = np.empty((n, k // 2, 2))
    if lib.orc_kdops(xyz.ctypes.data, V, n, k, eps, out.ctypes.data) < 0:
        raise ValueError("unsupported k")
    return out


def centroids(xyz):
    xyz = _c(xyz, np.float64)
    out = np.empty((xyz.shape[0], 3))
    lib.orc_centroids(xyz.ctypes.data, xyz.shape[1], xyz.shape[0], out.ctypes.data)
    return out


def morton_bounds(slabs, k):
    slabs = _c(slabs, np.float64)
    mn = np.empty(3)
    inv = np.empty(3)
    lib.orc_morton_bounds(slabs.ctypes.data, slabs.shape[0], k, mn.ctypes.data, inv.ctypes.data)
    return mn, inv


def quantize64(p, mn, inv):
    q = np.empty(3, dtype=np.uint64)
    lib.orc_quantize64(_c(p, np.float64).ctypes.data, _c(mn, np.float64).ctypes.data,
                       _c(inv, np.float64).ctypes.data, q.ctypes.data)
    return q


def quantize32(p, mn, inv):
    q = np.empty(3, dtype=np.uint32)
    lib.orc_quantize32(_c(p, np.float64).ctypes.data, _c(mn, np.float64).ctypes.data,
                       _c(inv, np.float64).ctypes.data, q.ctypes.data)
    return q


def morton64(x, y, z):
    return lib.orc_morton64(x, y, z)


def morton32(x, y, z):
    return lib.orc_morton32(x, y, z)


def morton_keys(cent, mn, inv):
    cent = _c(cent, np.float64)
    keys = np.empty(cent.shape[0], dtype=np.uint64)
    lib.orc_morton_keys(cent.ctypes.data, cent.shape[0], _c(mn, np.float64).ctypes.data,
                        _c(inv, np.float64).ctypes.data, keys.ctypes.data)
    return keys


def exclusive_scan(v):
    v = _c(v, np.int64).copy()
    lib.orc_exclusive_scan_i64(v.ctypes.data, v.shape[0])
    return v


def radix_sort_1bit(keys, idx=None):
    """The reference's one-bit-per-pass radix sorter; returns (sorted keys, permuted indices)."""
    keys = np.array(keys, copy=True)
    n = keys.shape[0]
    idx = np.arange(n, dtype=np.uint64) if idx is None else _c(idx, np.uint64).copy()
    if keys.dtype == np.uint64:
        lib.orc_radix_sort_1bit_u64(keys.ctypes.data, idx.ctypes.data, n)
    elif keys.dtype == np.uint32:
        lib.orc_radix_sort_1bit_u32(keys.ctypes.data, idx.ctypes.data, n)
    else:
        raise TypeError("keys must be uint32 or uint64")
    return keys, idx


def stable_perm(keys):
    keys = _c(keys, np.uint64)
    perm = np.empty(keys.shape[0], dtype=np.uint32)
    lib.orc_stable_sort_perm_u64(keys.ctypes.data, keys.shape[0], perm.ctypes.data)
    return perm


def overlap(a, b, k):
    return bool(lib.orc_overlap(_c(a, np.float64).ctypes.data, _c(b, np.float64).ctypes.data, k))


def _pairs_call(fn, args, cap_hint):
    cap = max(cap_hint, 1)
    while True:
        out = np.empty((cap, 2), dtype=np.uint32)
        cnt = fn(*args, out.ctypes.data, cap)
        if cnt <= cap:
            return out[:cnt]
        cap = cnt


def max_variant_axis(ca, cb):
    """The sweep axis of sort-and-sweep: the cardinal axis of largest centroid variance over A and B."""
    ca = _c(ca, np.float64)
    cb = _c(cb, np.float64)
    return int(lib.orc_max_variant_axis(ca.ctypes.data, ca.shape[0], cb.ctypes.data, cb.shape[0]))


def sort_and_sweep(sa, sb, k, axis):
    """Pairs (index into A, index into B) of the reference's sort-and-sweep over two element slab sets."""
    sa = _c(sa, np.float64)
    sb = _c(sb, np.float64)
    return _pairs_call(lib.orc_sort_and_sweep, (sa.ctypes.data, sa.shape[0], sb.ctypes.data, sb.shape[0], k, axis),
                       4 * (sa.shape[0] + sb.shape[0]))


def pairs_brute(sa, sb, k):
    sa = _c(sa, np.float64)
    sb = _c(sb, np.float64)
    return _pairs_call(lib.orc_pairs_brute, (sa.ctypes.data, sa.shape[0], sb.ctypes.data, sb.shape[0], k),
                       4 * (sa.shape[0] + sb.shape[0]))


def self_pairs_brute(s, k):
    s = _c(s, np.float64)
    return _pairs_call(lib.orc_self_pairs_brute, (s.ctypes.data, s.shape[0], k), 4 * s.shape[0])


def pairs_tree(sa, ca, sb, cb, k):
    sa, ca, sb, cb = (_c(x, np.float64) for x in (sa, ca, sb, cb))
    return _pairs_call(lib.orc_pairs_tree, (sa.ctypes.data, ca.ctypes.data, sa.shape[0], sb.ctypes.data,
                                            cb.ctypes.data, sb.shape[0], k), 4 * (sa.shape[0] + sb.shape[0]))


def self_pairs_tree(s, c, k):
    s, c = _c(s, np.float64), _c(c, np.float64)
    return _pairs_call(lib.orc_self_pairs_tree, (s.ctypes.data, c.ctypes.data, s.shape[0], k), 4 * s.shape[0])


def tree_node_count(s, c, k):
    s, c = _c(s, np.float64), _c(c, np.float64)
    return lib.orc_tree_node_count(s.ctypes.data, c.ctypes.data, s.shape[0], k)


def pair_set(xyz_a, xyz_b, k, eps=0.0, method="tree", gid_a=None, gid_b=None):
    """The exact pair set S(A, B) as a sorted (m, 2) uint64 array of (gid_a, gid_b)."""
    sa, sb = kdops(xyz_a, k, eps), kdops(xyz_b, k, eps)
    if method == "brute":
        p = pairs_brute(sa, sb, k)
    else:
        p = pairs_tree(sa, centroids(xyz_a), sb, centroids(xyz_b), k)
    return canonical(p, gid_a, gid_b)


def self_pair_set(xyz, k, eps=0.0, method="tree", gid=None):
    s = kdops(xyz, k, eps)
    p = self_pairs_brute(s, k) if method == "brute" else self_pairs_tree(s, centroids(xyz), k)
    return canonical(p, gid, gid)


PIPELINE_STAGES = ("slabs", "bounds", "keys", "sort", "tree", "traverse", "total")


def pipeline(xyz_a, xyz_b, k, eps=0.0, threads=0, keep_pairs=False):
    """The whole path on the CPU (all threads by default). Returns (|S|, {stage: seconds}), and with keep_pairs
    the pair set as a third item (canonical: sorted (m, 2) uint64 of (index in A, index in B))."""
    xa, xb = _c(xyz_a, np.float64), _c(xyz_b, np.float64)
    assert xa.shape[1] == xb.shape[1]
    st = np.zeros(7)
    if not keep_pairs:
        cnt = lib.orc_pipeline(xa.ctypes.data, xa.shape[0], xb.ctypes.data, xb.shape[0], xa.shape[1], k, eps,
                               threads, st.ctypes.data, None, 0)
        return cnt, dict(zip(PIPELINE_STAGES, st.tolist()))
    cap = 4 * (xa.shape[0] + xb.shape[0]) + 1
    while True:
        out = np.empty((cap, 2), dtype=np.uint32)
        cnt = lib.orc_pipeline(xa.ctypes.data, xa.shape[0], xb.ctypes.data, xb.shape[0], xa.shape[1], k, eps,
                               threads, st.ctypes.data, out.ctypes.data, cap)
        if cnt <= cap:
            break
        cap = cnt
    return cnt, dict(zip(PIPELINE_STAGES, st.tolist())), canonical(out[:cnt])


def morton_cluster(xyz, k, patches, eps=0.0):
    """The reference's Morton clustering of elements into `patches` patches: (element order (n,) uint32, patch
    bounds (patches + 1,) uint64), from the 32-bit hashes of the centroids over the k-DOP Morton bounds."""
    c = centroids(xyz)
    mn, inv = morton_bounds(kdops(xyz, k, eps), k)
    n = c.shape[0]
    order = np.empty(max(n, 1), dtype=np.uint32)
    bounds = np.empty(patches + 1, dtype=np.uint64)
    lib.orc_morton_cluster(c.ctypes.data, n, mn.ctypes.data, inv.ctypes.data, patches, order.ctypes.data,
                           bounds.ctypes.data)
    return order[:n], bounds


def max_threads():
    return lib.orc_max_threads()


def canonical(p, gid_a=None, gid_b=None):
    p = np.asarray(p).astype(np.uint64).reshape(-1, 2)
    if gid_a is not None:
        p[:, 0] = np.asarray(gid_a, dtype=np.uint64)[p[:, 0].astype(np.int64)]
    if gid_b is not None:
        p[:, 1] = np.asarray(gid_b, dtype=np.uint64)[p[:, 1].astype(np.int64)]
    if p.shape[0] == 0:
        return p
    order = np.lexsort((p[:, 1], p[:, 0]))
    return p[order]
