"""ctypes bindings of the reference cross-check libraries in oracle/_ref (built by oracle/ref_build.sh from the
reference's own headers). Test infrastructure: the oracle tests and the golden-vector generator use them to pin
the oracle's restatement to the reference's code; nothing of the product imports this module."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P, _U, _I, _D = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_double


def lib_path(tree_k):
    return os.path.join(HERE, "_ref", f"libbvhref{tree_k}.so")


def available():
    return all(os.path.exists(lib_path(k)) for k in (6, 26))


class Ref:
    """One build of the reference: element trees of dop_26 (tree_k=26) or dop_6 (tree_k=6)."""

    def __init__(self, tree_k=26):
        L = ctypes.CDLL(lib_path(tree_k))
        L.ref_tree_k.restype = _I
        L.ref_kdops.argtypes = [_P, _U, _I, _I, _D, _P]
        L.ref_kdops.restype = _I
        L.ref_centroids.argtypes = [_P, _U, _I, _P]
        L.ref_morton.argtypes = [_P, _U, _I, _D, _P, _P, _P]
        L.ref_morton64.argtypes = [_U, _U, _U]
        L.ref_morton64.restype = _U
        for f in (L.ref_tree_pairs, L.ref_brute_pairs18):
            f.argtypes = [_P, _U, _P, _U, _I, _D, _P, _U]
            f.restype = _U
        L.ref_self_pairs.argtypes = [_P, _U, _I, _D, _P, _U]
        L.ref_self_pairs.restype = _U
        L.ref_radix_sort_u64.argtypes = [_P, _U, _P, _P]
        L.ref_cluster.argtypes = [_P, _U, _I, _U, _P, _P]
        L.ref_sort_and_sweep.argtypes = [_P, _U, _P, _U, _I, _D, _I, _P, _P, _U]
        L.ref_sort_and_sweep.restype = _U
        self.lib = L
        self.tree_k = L.ref_tree_k()
        assert self.tree_k == tree_k

    def kdops(self, xyz, k, eps=0.0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        out = np.zeros((xyz.shape[0], k // 2, 2))
        assert self.lib.ref_kdops(xyz.ctypes.data, xyz.shape[0], xyz.shape[1], k, eps, out.ctypes.data) == 0
        return out

    def centroids(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        out = np.zeros((xyz.shape[0], 3))
        self.lib.ref_centroids(xyz.ctypes.data, xyz.shape[0], xyz.shape[1], out.ctypes.data)
        return out

    def morton(self, xyz, eps=0.0):
        """Morton bounds (min, inv) over this build's tree k-DOPs and the elements' 64-bit Morton codes."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        mn, inv = np.zeros(3), np.zeros(3)
        keys = np.zeros(xyz.shape[0], dtype=np.uint64)
        self.lib.ref_morton(xyz.ctypes.data, xyz.shape[0], xyz.shape[1], eps, mn.ctypes.data, inv.ctypes.data,
                            keys.ctypes.data)
        return mn, inv, keys

    def morton64(self, x, y, z):
        return self.lib.ref_morton64(x, y, z)

    def _pairs(self, fn, *args, cap):
        out = np.zeros((max(cap, 1), 2), dtype=np.uint64)
        cnt = fn(*args, out.ctypes.data, cap)
        return int(cnt), out[:min(cnt, cap)].astype(np.int64)

    def tree_pairs(self, a, b, eps=0.0, cap=1 << 20):
        """potential_collision_set over two top-down element trees: (count, pairs as the reference emits them)."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return self._pairs(self.lib.ref_tree_pairs, a.ctypes.data, a.shape[0], b.ctypes.data, b.shape[0],
                           a.shape[1], eps, cap=cap)

    def self_pairs(self, a, eps=0.0, cap=1 << 20):
        a = np.ascontiguousarray(a, dtype=np.float64)
        return self._pairs(self.lib.ref_self_pairs, a.ctypes.data, a.shape[0], a.shape[1], eps, cap=cap)

    def brute_pairs18(self, a, b, eps=0.0, cap=1 << 20):
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return self._pairs(self.lib.ref_brute_pairs18, a.ctypes.data, a.shape[0], b.ctypes.data, b.shape[0],
                           a.shape[1], eps, cap=cap)

    def radix_sort_u64(self, keys):
        """The reference's stable 1-bit radix sort: (sorted keys, permutation)."""
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        out = np.zeros_like(keys)
        perm = np.zeros(keys.shape[0], dtype=np.uint64)
        self.lib.ref_radix_sort_u64(keys.ctypes.data, keys.shape[0], out.ctypes.data, perm.ctypes.data)
        return out, perm

    def sort_and_sweep(self, a, b, eps=0.0, axis=-1, cap=1 << 20):
        """sort_and_sweep_local with each set as one patch: (count, pairs in the functor's order, axis swept)."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        used = ctypes.c_int(-1)
        cnt, pairs = self._pairs(self.lib.ref_sort_and_sweep, a.ctypes.data, a.shape[0], b.ctypes.data, b.shape[0],
                                 a.shape[1], eps, axis, ctypes.byref(used), cap=cap)
        return cnt, pairs, used.value

    def cluster(self, xyz, clusters):
        """morton_cluster: (element order, clusters - 1 split positions)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        order = np.zeros(xyz.shape[0], dtype=np.uint64)
        splits = np.zeros(max(clusters - 1, 0), dtype=np.uint64)
        self.lib.ref_cluster(xyz.ctypes.data, xyz.shape[0], xyz.shape[1], clusters, order.ctypes.data,
                             splits.ctypes.data)
        return order, splits
