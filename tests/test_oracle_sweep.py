"""The oracle's restatement of the reference's sort-and-sweep (src/bvh/narrowphase/kokkos.hpp:125-248) against
the brute-force pair set: the sweep emits exactly S(A, B) on every axis, including a degenerate one."""
import numpy as np
import pytest

from distbvh_b200 import meshes
from oracle import oracle as orc


@pytest.mark.parametrize("V,k,eps", [(3, 18, 0.0), (4, 26, 0.004), (8, 6, 0.0), (3, 6, 0.002)])
def test_sweep_equals_brute_force_on_every_axis(V, k, eps):
    a = meshes.random_soup(1500, V, seed=400 + V, size=0.04)
    b = meshes.random_soup(1200, V, seed=500 + V, size=0.04, stream=1)
    sa, sb = orc.kdops(a, k, eps), orc.kdops(b, k, eps)
    want = orc.canonical(orc.pairs_brute(sa, sb, k).astype(np.uint64))
    assert want.shape[0] > 0
    for axis in (0, 1, 2):
        assert np.array_equal(orc.canonical(orc.sort_and_sweep(sa, sb, k, axis).astype(np.uint64)), want), axis


def test_sweep_on_flat_plates_and_a_degenerate_axis():
    pa = meshes.plate(40, 20, 0.0, 1.0, 0.0, 1.0, 0.0)
    pb = meshes.plate(30, 30, 0.0, 1.0, 0.0, 1.0, 0.0)
    for eps in (0.0, 0.003):
        sa, sb = orc.kdops(pa, 18, eps), orc.kdops(pb, 18, eps)
        want = orc.canonical(orc.pairs_brute(sa, sb, 18).astype(np.uint64))
        for axis in (0, 1, 2):  # z is degenerate when eps = 0 (global max = global min)
            assert np.array_equal(orc.canonical(orc.sort_and_sweep(sa, sb, 18, axis).astype(np.uint64)), want)


def test_max_variant_axis_picks_the_long_direction():
    rng = np.random.default_rng(7)
    for axis in range(3):
        scale = np.array([0.1, 0.1, 0.1])
        scale[axis] = 5.0
        ca = rng.random((500, 3)) * scale
        cb = rng.random((400, 3)) * scale
        assert orc.max_variant_axis(ca, cb) == axis


# Known answers of the reference's own tests (tests/KokkosTest.cpp:37-140): the axis of a 12-element grid along x,
# y or z against one element, and 12 pairs from sort_and_sweep_local in both roles.
def _grids():
    from tests.grids import element_grid
    return element_grid


@pytest.mark.parametrize("dims,axis", [((12, 1, 1), 0), ((1, 12, 1), 1), ((1, 1, 12), 2)])
def test_reference_max_variant_axis_cases(dims, axis):
    element_grid = _grids()
    a, _ = element_grid(*dims)
    b, _ = element_grid(1, 1, 1)
    assert orc.max_variant_axis(orc.centroids(a), orc.centroids(b)) == axis


@pytest.mark.parametrize("k", [6, 18, 26])
def test_reference_sort_and_sweep_cases(k):
    element_grid = _grids()
    a, _ = element_grid(12, 1, 1)
    b, _ = element_grid(1, 1, 1)
    sa, sb = orc.kdops(a, k), orc.kdops(b, k)
    p = orc.sort_and_sweep(sa, sb, k, 0)
    assert p.shape[0] == 12 and set(p[:, 1].tolist()) == {0} and sorted(p[:, 0].tolist()) == list(range(12))
    q = orc.sort_and_sweep(sb, sa, k, 0)  # "x-axis flipped"
    assert q.shape[0] == 12 and set(q[:, 0].tolist()) == {0}
