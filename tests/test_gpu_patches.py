"""Patches on the device (bvhg_cluster) and element pairs grouped by patch pair (bvhg_patch_pairs).

bvhg_cluster is the reference's morton_cluster (src/bvh/split/cluster.hpp:89-179) computed on the GPU from the
build's sorted Morton keys: its element order and patch boundaries must equal the golden vectors written by the
reference's own code and, on larger inputs, the oracle's restatement (which hashes with quantize32 + morton32
itself). Inputs cover soups at many patch counts, runs of equal 32-bit hashes beyond the device's in-place limit
(32) and its shared-memory limit (2048), all elements equal, and objects with fewer elements than patches.
bvhg_patch_pairs must give exactly the pair set of bvhg_broadphase, every pair in the group of its two patches.
"""
import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc
from tests.grids import clustered_soup, distinct_cells

pytestmark = pytest.mark.gpu

GOLDEN = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "ref_vectors.npz"))


def gpu_cluster(xyz, k, patches, precision=bvhg.PLAIN_FP64):
    with bvhg.Context(k=k, precision=precision) as ctx:
        o = ctx.object()
        ctx.set_elements(o, xyz)
        ctx.build(o)
        bounds, order = ctx.cluster(o, patches, xyz.shape[0])
        return order, bounds


@pytest.mark.parametrize("od", [1, 8, 64])
def test_cluster_matches_the_reference_vectors(od):
    xyz = GOLDEN["cluster/xyz"]
    order, bounds = gpu_cluster(xyz, 26, od)
    assert np.array_equal(order.astype(np.int64), GOLDEN[f"cluster/od{od}/order"].astype(np.int64))
    want = np.concatenate([[0], GOLDEN[f"cluster/od{od}/splits"].astype(np.int64), [xyz.shape[0]]])
    assert np.array_equal(bounds.astype(np.int64), want)


def check_against_oracle(xyz, k, patches, precision=bvhg.PLAIN_FP64):
    order, bounds = gpu_cluster(xyz, k, patches, precision)
    oorder, obounds = orc.morton_cluster(xyz, k, patches)
    assert np.array_equal(order, oorder), "patch order differs"
    assert np.array_equal(bounds, obounds), "patch bounds differ"


@pytest.mark.parametrize("patches", [1, 2, 7, 64, 1024, 70000])
def test_cluster_matches_the_oracle_on_a_soup(patches):
    check_against_oracle(meshes.random_soup(300000, 3, seed=51, size=0.003), 18, patches)


@pytest.mark.parametrize("k,V", [(6, 4), (26, 8)])
def test_cluster_other_kdops_and_vertex_counts(k, V):
    check_against_oracle(meshes.random_soup(20000, V, seed=52, size=0.02), k, 16)
    check_against_oracle(meshes.random_soup(20000, V, seed=52, size=0.02), k, 16, bvhg.FILTER_FP32)


def test_cluster_on_the_sphere_plate():
    s, p = meshes.sphere_plate(level=5, nx=256, ny=128)
    check_against_oracle(s, 18, 32)
    check_against_oracle(p, 18, 32)  # flat plate: the z axis takes the NaN -> 0 path


@pytest.mark.parametrize("counts", [(40, 3, 33), (2500, 2048, 2049, 5), (100000, 34)])
def test_cluster_with_long_runs_of_equal_hashes(counts):
    xyz = clustered_soup(counts, seed=sum(counts))
    for patches in (2, 16, 512):
        check_against_oracle(xyz, 18, patches)


def test_cluster_with_many_long_runs():
    rng = np.random.default_rng(53)
    counts = rng.integers(33, 200, size=500)
    xyz = clustered_soup(counts, seed=54, cells=distinct_cells(counts.shape[0], 55))
    check_against_oracle(xyz, 18, 128)


def test_cluster_all_elements_equal():
    tri = meshes.random_soup(1, 3, seed=56, size=0.1)
    xyz = np.ascontiguousarray(np.repeat(tri, 6000, axis=0))
    for patches in (1, 4, 6000, 7000):
        check_against_oracle(xyz, 18, patches)


@pytest.mark.parametrize("n", [1, 2, 3, 9])
def test_cluster_fewer_elements_than_patches(n):
    xyz = meshes.random_soup(n, 3, seed=57 + n, size=0.2)
    check_against_oracle(xyz, 18, 16)


def expand_groups(groups, pairs, order_a, bounds_a, order_b, bounds_b):
    out = []
    for pa, pb, first, count in groups.astype(np.int64):
        chunk = pairs[first:first + count].astype(np.int64)
        ea = order_a[bounds_a[pa].astype(np.int64) + chunk[:, 0]]
        eb = order_b[bounds_b[pb].astype(np.int64) + chunk[:, 1]]
        assert np.all(chunk[:, 0] < bounds_a[pa + 1] - bounds_a[pa])
        assert np.all(chunk[:, 1] < bounds_b[pb + 1] - bounds_b[pb])
        out.append(np.stack([ea, eb], axis=1))
    return orc.canonical(np.concatenate(out) if out else np.zeros((0, 2)))


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
@pytest.mark.parametrize("pa,pb", [(1, 1), (8, 4), (64, 128)])
def test_patch_pairs_group_the_exact_pair_set(precision, pa, pb):
    a = meshes.random_soup(40000, 3, seed=61, size=0.01)
    b = meshes.random_soup(30000, 3, seed=62, size=0.01, stream=1)
    want = orc.pair_set(a, b, 18)
    with bvhg.Context(k=18, precision=precision) as ctx:
        oa, ob = ctx.object(), ctx.object()
        ctx.set_elements(oa, a)
        ctx.set_elements(ob, b)
        ctx.build(oa)
        ctx.build(ob)
        ba, orda = ctx.cluster(oa, pa, a.shape[0])
        bb, ordb = ctx.cluster(ob, pb, b.shape[0])
        for _ in range(2):  # the second call runs after the contact-density decision of the first
            groups, pairs = ctx.patch_pairs(oa, ob)
            assert groups.shape[0] > 0 and pairs.shape[0] == want.shape[0]
            keys = groups[:, 0].astype(np.int64) * pb + groups[:, 1]
            assert np.all(np.diff(keys) > 0) and np.all(groups[:, 3] > 0)
            assert np.array_equal(np.cumsum(np.concatenate([[0], groups[:-1, 3].astype(np.int64)])),
                                  groups[:, 2].astype(np.int64))
            assert np.array_equal(expand_groups(groups, pairs, orda, ba, ordb, bb), want)


def test_patch_pairs_errors_and_empty_objects():
    a = meshes.random_soup(500, 3, seed=63, size=0.05)
    with bvhg.Context(k=18) as ctx:
        oa, ob, oe = ctx.object(), ctx.object(), ctx.object()
        ctx.set_elements(oa, a)
        ctx.set_elements(ob, a)
        ctx.set_elements(oe, np.zeros((0, 3, 3)))
        for o in (oa, ob, oe):
            ctx.build(o)
        with pytest.raises(bvhg.BvhgError) as e:
            ctx.patch_pairs(oa, ob)  # not clustered yet
        assert e.value.status == bvhg.ERR_STATE
        ctx.cluster(oa, 4, 500)
        ctx.cluster(ob, 4, 500)
        bounds, _ = ctx.cluster(oe, 4, 0)
        assert np.array_equal(bounds, np.zeros(5, dtype=np.uint64))
        with pytest.raises(bvhg.BvhgError):
            ctx.patch_pairs(oa, oa)
        groups, pairs = ctx.patch_pairs(oa, oe)
        assert groups.shape[0] == 0 and pairs.shape[0] == 0
        g, p = ctx.patch_pairs(oa, ob)
        assert p.shape[0] == orc.pair_set(a, a, 18).shape[0]
        ctx.set_elements(oa, a)  # new elements: the patches are gone
        ctx.build(oa)
        with pytest.raises(bvhg.BvhgError):
            ctx.patch_pairs(oa, ob)
