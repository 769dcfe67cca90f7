"""Pins the CPU oracle to the known answers in the reference's own unit tests (no GPU).

Each test names the reference test it restates. The oracle is the checker of every GPU parity test, so these are
the anchor of the whole parity chain.
"""
import sys

import numpy as np
import pytest

from oracle import oracle as orc
from tests.grids import element_grid, make_cube

EPS = sys.float_info.epsilon


# tests/hash_test.cpp:41-160 — morton hashing, 32 and 64 bit
@pytest.mark.parametrize("xyz,expected", [
    ((0x3ff, 0x3ff, 0x3ff), 0x3fffffff),
    ((0x3ff, 0, 0), 0x09249249),
    ((0, 0x3ff, 0), 0x12492492),
    ((0, 0, 0x3ff), 0x24924924),
])
def test_morton32_known_answers(xyz, expected):
    assert orc.morton32(*xyz) == expected


@pytest.mark.parametrize("xyz,expected", [
    ((0x1fffff, 0x1fffff, 0x1fffff), 0x7fffffffffffffff),
    ((0x1fffff, 0, 0), 0x1249249249249249),
    ((0, 0x1fffff, 0), 0x2492492492492492),
    ((0, 0, 0x1fffff), 0x4924924924924924),
])
def test_morton64_known_answers(xyz, expected):
    assert orc.morton64(*xyz) == expected


def test_morton64_is_the_bit_interleave():
    # hash_test.cpp:180-199 checks the multiply-mask expansion against BMI2 pdep; restated as a plain interleave.
    rng = np.random.default_rng(0)
    for _ in range(200):
        x, y, z = (int(v) for v in rng.integers(0, 0x200000, 3))
        ref = 0
        for b in range(21):
            ref |= ((x >> b) & 1) << (3 * b) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b + 2)
        assert orc.morton64(x, y, z) == ref


# tests/hash_test.cpp:162-178 — quantization bounds
def test_quantize32_bounds():
    mn = np.array([-1.0, 0.0, 3.0])
    mx = np.array([-0.5, 2.0, 4.0])
    inv = 1.0 / (mx - mn)
    assert list(orc.quantize32(mn, mn, inv)) == [0, 0, 0]
    assert list(orc.quantize32(mx - 0.00001, mn, inv)) == [0x3ff, 0x3ff, 0x3ff]


def test_quantize64_degenerate_axis_and_wrap():
    # A flat axis has width 0 -> inv = inf -> 0 * inf = NaN -> 0 after the mask; a normalised 1.0 wraps to 0.
    q = orc.quantize64(np.array([0.5, 0.25, 0.0]), np.zeros(3), np.array([1.0, 1.0, np.inf]))
    assert list(q) == [0x100000, 0x80000, 0]
    assert orc.morton64(*(int(v) for v in q)) == 0x1400000000000000
    assert list(orc.quantize64(np.ones(3), np.zeros(3), np.ones(3))) == [0, 0, 0]


# tests/snapshot_test.cpp:31-72 — Morton32 of an 8^3 grid under a fixed bounds override
def test_snapshot_morton32_grid():
    bmin = np.array([-100.0] * 3)
    bmax = np.array([100.0] * 3)
    half_cell = (bmax - bmin) / 2048.0
    incr = ((bmax + half_cell) - (bmin + half_cell)) / 8.0
    inv = np.array([0.005] * 3)
    pos = (bmin + half_cell).copy()
    q = [0, 0, 0]
    for z in range(8):
        for y in range(8):
            for x in range(8):
                got = orc.quantize32(pos, bmin, inv)
                assert orc.morton32(*(int(v) for v in got)) == orc.morton32(*q)
                pos[0] += incr[0]
                q[0] += 0x80
            pos[1] += incr[1]
            pos[0] = (bmin + half_cell)[0]
            q[1] += 0x80
            q[0] = 0
        pos[2] += incr[2]
        pos[1] = (bmin + half_cell)[1]
        q[2] += 0x80
        q[1] = 0


# tests/sort_test.cpp:9-30 — stable radix sort known answer
def test_radix_sort_known_answer():
    keys = np.array([3, 7, 2, 1, 4, 9, 1, 3], dtype=np.uint32)
    sk, idx = orc.radix_sort_1bit(keys)
    assert list(sk) == [1, 1, 2, 3, 3, 4, 7, 9]
    assert list(idx) == [3, 6, 2, 0, 7, 4, 1, 5]
    sk64, idx64 = orc.radix_sort_1bit(keys.astype(np.uint64))
    assert list(sk64) == [1, 1, 2, 3, 3, 4, 7, 9]
    assert list(idx64) == [3, 6, 2, 0, 7, 4, 1, 5]
    assert list(orc.stable_perm(keys.astype(np.uint64))) == [3, 6, 2, 0, 7, 4, 1, 5]


def test_one_bit_radix_equals_stable_sort():
    rng = np.random.default_rng(1)
    for n in (1, 2, 17, 1000, 4099):
        keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
        keys[rng.integers(0, n, n // 3)] = keys[0]  # duplicates
        sk, idx = orc.radix_sort_1bit(keys)
        perm = orc.stable_perm(keys)
        assert np.array_equal(idx.astype(np.uint32), perm)
        assert np.array_equal(sk, keys[perm])


# tests/UtilTest.cpp:42-55 — exclusive scan known answer
def test_exclusive_scan_known_answer():
    assert list(orc.exclusive_scan([3, 7, 2, 1, 4, 9, 1, 3])) == [0, 3, 10, 12, 13, 17, 26, 27]


# tests/KDopTest.cpp:241-314 — strict overlap edges with +-DBL_EPSILON nudges (K = 6 and 26 in the reference,
# 18 added: the same cubes give the same answers)
CUBE_CASES = [
    ((3.0, 0.0, 0.0), False),
    ((2.0 - EPS, 0.0, 0.0), True),
    ((0.0, 0.0, 0.0), True),
    ((-2.0 + EPS, 0.0, 0.0), True),
    ((-3.0, 0.0, 0.0), False),
    ((2.0 - EPS, 2.0 - EPS, 0.0), True),
    ((-2.0 + EPS, -2.0 + EPS, 0.0), True),
    ((2.0 - EPS, 2.0 - EPS, 2.0 - EPS), True),
    ((-2.0 + EPS, -2.0 + EPS, -2.0 + EPS), True),
]


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("center,expected", CUBE_CASES)
def test_kdop_cube_overlap(k, center, expected):
    kd1 = orc.kdops(make_cube((0.0, 0.0, 0.0)), k)[0]
    kd2 = orc.kdops(make_cube(center), k)[0]
    assert orc.overlap(kd1, kd2, k) == expected
    assert orc.overlap(kd2, kd1, k) == expected


@pytest.mark.parametrize("k", [6, 18, 26])
def test_touching_cubes_do_not_overlap(k):
    # strict '<': cubes sharing a face (distance exactly 2) are not a pair
    kd1 = orc.kdops(make_cube((0.0, 0.0, 0.0)), k)[0]
    kd2 = orc.kdops(make_cube((2.0, 0.0, 0.0)), k)[0]
    assert not orc.overlap(kd1, kd2, k)


def test_normals_tables():
    r, s = 0.7071067811865475, 0.5773502691896258
    assert np.array_equal(orc.normals(6), np.eye(3))
    n18 = orc.normals(18)
    assert n18.shape == (9, 3)
    assert np.array_equal(n18[3:], [[r, r, 0], [r, 0, r], [0, r, r], [r, -r, 0], [r, 0, -r], [0, r, -r]])
    n26 = orc.normals(26)
    assert n26.shape == (13, 3)
    assert np.array_equal(n26[3:7], [[s, s, s], [s, -s, s], [s, s, -s], [s, -s, -s]])
    assert np.array_equal(n26[7:], n18[3:])


def test_projection_is_not_fused():
    # ((v0*n0) + (v1*n1)) + (v2*n2) rounded step by step: differs from an FMA evaluation on this input.
    v = np.array([0.1, 0.2, 0.3])
    ax = np.array([0.7071067811865475, 0.0, 0.7071067811865475])
    t0, t1, t2 = v[0] * ax[0], v[1] * ax[1], v[2] * ax[2]
    kd = orc.kdops(v.reshape(1, 1, 3), 18)[0]
    assert kd[4, 0] == (t0 + t1) + t2


# tests/CollisionTest.cpp:43-81 — pair counts over the reference's hex grids (bphase_kdop = dop_26)
def test_fully_overlapping_groups_all_collide():
    a, _ = element_grid(4, 4, 4)
    b, _ = element_grid(1, 1, 1, a.shape[0])
    assert orc.pair_set(a, b, 26).shape[0] == 64
    assert orc.pair_set(a, b, 26, method="brute").shape[0] == 64


def test_non_overlapping_group_does_not_self_collide():
    a, _ = element_grid(2, 2, 1)
    assert orc.self_pair_set(a, 26).shape[0] == 0
    assert orc.self_pair_set(a, 26, method="brute").shape[0] == 0


def test_overlapping_group_self_collides():
    a, _ = element_grid(2, 2, 2)
    b, _ = element_grid(1, 1, 1, a.shape[0])
    x = np.concatenate([a, b])
    assert orc.self_pair_set(x, 26).shape[0] == 8
    assert orc.self_pair_set(x, 26, method="brute").shape[0] == 8


# tests/TreeTest.cpp:49-90 — one element per leaf: 2n - 1 nodes (127 for 64 elements)
def test_tree_node_count():
    a, _ = element_grid(4, 4, 4)
    assert orc.tree_node_count(orc.kdops(a, 26), orc.centroids(a), 26) == 127


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("V", [3, 4, 8])
def test_tree_traversal_equals_brute_force(k, V):
    from distbvh_b200 import meshes
    a = meshes.random_soup(400, V, seed=11, size=0.08)
    b = meshes.random_soup(300, V, seed=12, size=0.08, stream=1)
    for eps in (0.0, 0.01):
        assert np.array_equal(orc.pair_set(a, b, k, eps), orc.pair_set(a, b, k, eps, method="brute"))
        assert np.array_equal(orc.self_pair_set(a, k, eps), orc.self_pair_set(a, k, eps, method="brute"))


def test_centroid_is_mean_accumulated_from_zero():
    xyz = np.array([[[0.1, 0.2, 0.3], [0.4, 0.5, 0.6], [0.7, 0.8, 0.9]]])
    c = orc.centroids(xyz)[0]
    assert c[0] == ((0.0 + 0.1) + 0.4 + 0.7) / 3.0
    assert c[2] == ((0.0 + 0.3) + 0.6 + 0.9) / 3.0


def test_morton_bounds_serial_semantics():
    a, _ = element_grid(3, 2, 1)
    s = orc.kdops(a, 18)
    mn, inv = orc.morton_bounds(s, 18)
    assert list(mn) == [0.0, 0.0, 0.0]
    assert np.array_equal(inv, 1.0 / (np.array([1.0, 1.0, 1.0]) - 0.0))


# Golden vectors computed by the reference's own headers (tests/golden/make_golden.py through oracle/_ref):
# kdop_base::from_vertices (src/bvh/kdop.hpp:238-264), TestCommon's centroid, compute_bounds + morton
# (src/bvh/contact_entity.hpp:104-148), potential_collision_set / self_collision_set over top-down trees of dop_26
# and dop_6 (src/bvh/collision_query.hpp:331-379), 18-DOP overlap by brute force (src/bvh/kdop.hpp:538-549).
GOLDEN = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "ref_vectors.npz"))
CASES = [str(c) for c in GOLDEN["cases"]]


def u64(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_vectors(case):
    g = lambda key: GOLDEN[f"{case}/{key}"]  # noqa: E731
    a, b, eps = g("a"), g("b"), float(g("eps"))
    for side, x in (("a", a), ("b", b)):
        for k in (6, 18, 26):
            assert np.array_equal(u64(orc.kdops(x, k, eps)), u64(g(f"{side}/kdops{k}"))), (side, k)
        c = orc.centroids(x)
        assert np.array_equal(u64(c), u64(g(f"{side}/centroids")))
        mn, inv = orc.morton_bounds(orc.kdops(x, 26, eps), 26)
        assert np.array_equal(u64(mn), u64(g(f"{side}/min3"))) and np.array_equal(u64(inv), u64(g(f"{side}/inv3")))
        assert np.array_equal(orc.morton_keys(c, mn, inv), g(f"{side}/keys"))
    for k in (26, 6):
        # two trees: the reference's count is right, its emitted ids are not (collision_query.hpp:310-312)
        assert orc.pair_set(a, b, k, eps).shape[0] == int(g(f"tree_count{k}"))
        # one tree: its ids are right (either order within a pair), the whole set must match
        assert np.array_equal(orc.self_pair_set(a, k, eps), orc.canonical(np.sort(g(f"self{k}"), axis=1)))
    assert np.array_equal(orc.pair_set(a, b, 18, eps), orc.canonical(g("pairs18")))


def test_stable_sort_matches_the_reference_radix_sorter():
    """radix_sorter (src/bvh/util/sort.hpp:75-144) run by the reference's own code on 3000 keys with duplicates."""
    keys = GOLDEN["radix/keys"]
    perm = orc.stable_perm(keys)
    assert np.array_equal(perm.astype(np.uint64), GOLDEN["radix/perm"])
    assert np.array_equal(keys[perm], GOLDEN["radix/sorted"])


def test_sort_and_sweep_matches_the_reference_vectors():
    """The oracle's sort-and-sweep and axis choice against sort_and_sweep_local / max_variant_axis outputs of the
    reference's own code (dop_26 and dop_6 builds) stored in the fixture."""
    g = GOLDEN
    checked = 0
    for name in g["cases"]:
        name = str(name)
        if not name.startswith("soup"):
            continue
        for k in (26, 6):
            axis = int(g[f"{name}/sweep{k}/axis"])
            assert orc.max_variant_axis(g[f"{name}/a/centroids"], g[f"{name}/b/centroids"]) == axis
            mine = orc.sort_and_sweep(g[f"{name}/a/kdops{k}"], g[f"{name}/b/kdops{k}"], k, axis).astype(np.int64)
            assert np.array_equal(np.unique(mine, axis=0), g[f"{name}/sweep{k}/pairs"].astype(np.int64)), (name, k)
            checked += 1
    assert checked == 12


@pytest.mark.parametrize("od", [1, 8, 64])
def test_oracle_morton_cluster_matches_the_reference_vectors(od):
    """morton_cluster restated (32-bit hashes, stable sorts by hash and by split depth) against the element order and
    splits that the reference's own code wrote."""
    xyz = GOLDEN["cluster/xyz"]
    order, bounds = orc.morton_cluster(xyz, 26, od)
    assert np.array_equal(order.astype(np.int64), GOLDEN[f"cluster/od{od}/order"].astype(np.int64))
    want = np.concatenate([[0], GOLDEN[f"cluster/od{od}/splits"].astype(np.int64), [xyz.shape[0]]])
    assert np.array_equal(bounds.astype(np.int64), want)


def test_oracle_morton_cluster_edge_cases():
    # no elements: every split is 0; fewer elements than patches: unchosen splits hold n - 1
    order, bounds = orc.morton_cluster(np.zeros((0, 3, 3)), 18, 4)
    assert order.shape == (0,) and np.array_equal(bounds, np.zeros(5, dtype=np.uint64))
    xyz = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[5, 5, 5], [6, 5, 5], [5, 6, 5]]], dtype=np.float64)
    order, bounds = orc.morton_cluster(xyz, 18, 4)
    assert np.array_equal(order, [0, 1]) and np.array_equal(bounds, [0, 0, 1, 1, 2])
