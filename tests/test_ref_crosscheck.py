"""The oracle against the reference's own code on fresh seeded inputs (no GPU).

oracle/_ref holds two builds of the reference's headers (oracle/ref_build.sh): element trees of dop_26 and of
dop_6. Skipped where they were not built (the reference sources are needed to build them); the committed golden
vectors in tests/golden cover the same functions everywhere.
"""
import numpy as np
import pytest

from distbvh_b200 import meshes
from oracle import oracle as orc
from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def u64(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.fixture(scope="module")
def refs():
    return {26: ref.Ref(26), 6: ref.Ref(6)}


@pytest.mark.parametrize("V", [3, 4, 8])
@pytest.mark.parametrize("eps", [0.0, 0.003])
def test_slabs_keys_and_pairs(refs, V, eps):
    a = meshes.random_soup(1500, V, seed=11 + V, size=0.05)
    b = meshes.random_soup(1200, V, seed=21 + V, size=0.05, stream=1)
    r = refs[26]
    for k in (6, 18, 26):
        assert np.array_equal(u64(r.kdops(a, k, eps)), u64(orc.kdops(a, k, eps))), k
    assert np.array_equal(u64(r.centroids(a)), u64(orc.centroids(a)))
    for tk, rr in refs.items():
        mn, inv, keys = rr.morton(a, eps)
        omn, oinv = orc.morton_bounds(orc.kdops(a, tk, eps), tk)
        assert np.array_equal(u64(mn), u64(omn)) and np.array_equal(u64(inv), u64(oinv))
        assert np.array_equal(keys, orc.morton_keys(orc.centroids(a), omn, oinv))
        cnt, _ = rr.tree_pairs(a, b, eps)
        assert cnt == orc.pair_set(a, b, tk, eps).shape[0]
        _, sp = rr.self_pairs(a, eps)
        assert np.array_equal(orc.canonical(np.sort(sp, axis=1)), orc.self_pair_set(a, tk, eps))
    _, p18 = r.brute_pairs18(a, b, eps)
    assert np.array_equal(orc.canonical(p18), orc.pair_set(a, b, 18, eps))


def test_degenerate_axis_keys(refs):
    """A flat plate: the z width is 0, inv = +inf, 0 * inf = NaN quantises to 0 in both."""
    from tests.grids import element_grid
    a = element_grid(20, 10, 1)[0][:, :3, :].copy()
    a[:, :, 2] = 0.0
    mn, inv, keys = refs[26].morton(a)
    omn, oinv = orc.morton_bounds(orc.kdops(a, 26), 26)
    assert np.isinf(inv[2]) and np.array_equal(u64(inv), u64(oinv))
    assert np.array_equal(keys, orc.morton_keys(orc.centroids(a), omn, oinv))


def test_morton64_known_answers(refs):
    r = refs[26]
    assert r.morton64(0x1fffff, 0, 0) == 0x1249249249249249
    assert r.morton64(0, 0x1fffff, 0) == 0x2492492492492492
    assert r.morton64(0, 0, 0x1fffff) == 0x4924924924924924
    rng = np.random.default_rng(3)
    for x, y, z in rng.integers(0, 1 << 21, (200, 3)):
        assert r.morton64(int(x), int(y), int(z)) == int(orc.morton64(int(x), int(y), int(z)))


def test_radix_sorter_and_cluster(refs):
    rng = np.random.default_rng(17)
    keys = rng.integers(0, 1 << 63, 5000, dtype=np.uint64)
    keys[::5] = keys[11]
    s, p = refs[26].radix_sort_u64(keys)
    assert np.array_equal(p.astype(np.int64), orc.stable_perm(keys).astype(np.int64))
    assert np.array_equal(s, np.sort(keys, kind="stable"))


@pytest.mark.parametrize("V", [3, 4, 8])
@pytest.mark.parametrize("eps", [0.0, 0.003])
def test_sort_and_sweep_against_the_reference(refs, V, eps):
    """The oracle's sort-and-sweep and axis choice against the reference's sort_and_sweep_local and
    max_variant_axis (dop_26 and dop_6 builds): the same axis, the same emitted pairs on every axis."""
    a = meshes.random_soup(900, V, seed=1300 + V, size=0.05)
    b = meshes.random_soup(700, V, seed=1400 + V, size=0.05, stream=1)
    for k, r in refs.items():
        sa, sb = orc.kdops(a, k, eps), orc.kdops(b, k, eps)
        cnt, pairs, axis = r.sort_and_sweep(a, b, eps, -1)
        assert axis == orc.max_variant_axis(orc.centroids(a), orc.centroids(b))
        assert cnt > 0
        mine = orc.sort_and_sweep(sa, sb, k, axis).astype(np.int64)
        assert np.array_equal(np.unique(pairs, axis=0), np.unique(mine, axis=0)), (k, axis)
        for ax in (0, 1, 2):
            cnt2, pairs2, used = r.sort_and_sweep(a, b, eps, ax)
            assert used == ax
            mine2 = orc.sort_and_sweep(sa, sb, k, ax).astype(np.int64)
            assert np.array_equal(np.unique(pairs2, axis=0), np.unique(mine2, axis=0)), (k, ax)
