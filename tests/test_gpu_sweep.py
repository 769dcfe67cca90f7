"""GPU sort-and-sweep (bvhg_sort_and_sweep) against the oracle's restatement of the reference's
sort_and_sweep_local and against the exact pair set, through the C ABI. The pair set must be S(A, B) bit for bit
(integer pairs) on every axis; the axis chosen for axis = -1 must be the oracle's max_variant_axis on clear-cut
inputs."""
import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def build_pair(ctx, a, b, ga=None, gb=None):
    oa, ob = ctx.object(), ctx.object()
    ctx.set_elements(oa, a, gid=ga)
    ctx.set_elements(ob, b, gid=gb)
    ctx.build(oa)
    ctx.build(ob)
    return oa, ob


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("V", [3, 4, 8])
@pytest.mark.parametrize("eps", [0.0, 0.004])
def test_sweep_matches_oracle_and_pair_set(k, V, eps):
    a = meshes.random_soup(3000, V, seed=600 + V, size=0.03)
    b = meshes.random_soup(2500, V, seed=700 + V, size=0.03, stream=1)
    sa, sb = orc.kdops(a, k, eps), orc.kdops(b, k, eps)
    want = orc.pair_set(a, b, k, eps)
    assert want.shape[0] > 0
    with bvhg.Context(k=k, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, a, b)
        for axis in (-1, 0, 1, 2):
            got, used = ctx.sort_and_sweep(oa, ob, axis)
            assert used == (axis if axis >= 0 else orc.max_variant_axis(orc.centroids(a), orc.centroids(b)))
            assert np.array_equal(orc.canonical(got), want), axis
            ref = orc.canonical(orc.sort_and_sweep(sa, sb, k, used).astype(np.uint64))
            assert np.array_equal(orc.canonical(got), ref), axis
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want)


def test_axis_choice_follows_the_largest_centroid_variance():
    for axis in range(3):
        base = meshes.random_soup(2000, 3, seed=800 + axis, size=0.01)
        stretch = np.ones(3)
        stretch[axis] = 6.0
        a = base * stretch
        b = meshes.random_soup(1500, 3, seed=900 + axis, size=0.01, stream=1) * stretch
        with bvhg.Context(k=18) as ctx:
            oa, ob = build_pair(ctx, a, b)
            got, used = ctx.sort_and_sweep(oa, ob, -1)
            assert used == axis == orc.max_variant_axis(orc.centroids(a), orc.centroids(b))
            assert np.array_equal(orc.canonical(got), orc.pair_set(a, b, 18))


@pytest.mark.parametrize("eps", [0.0, 0.003])
def test_flat_plates_and_a_degenerate_axis(eps):
    pa = meshes.plate(60, 30, 0.0, 1.0, 0.0, 1.0, 0.0)
    pb = meshes.plate(50, 40, 0.0, 1.0, 0.0, 1.0, 0.0)
    want = orc.pair_set(pa, pb, 18, eps)
    with bvhg.Context(k=18, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, pa, pb)
        for axis in (-1, 0, 1, 2):  # with eps = 0 the z range is a single value
            got, _ = ctx.sort_and_sweep(oa, ob, axis)
            assert np.array_equal(orc.canonical(got), want), axis


def test_many_tiles_mixed_vertex_counts_gids_and_repeated_calls():
    a = meshes.random_soup(40000, 3, seed=1001, size=0.006)
    b = meshes.random_soup(30000, 4, seed=1002, size=0.006, stream=1)
    ga = np.arange(a.shape[0], dtype=np.uint64) * 3 + 7
    gb = np.arange(b.shape[0], dtype=np.uint64) * 5 + 11
    want = orc.pair_set(a, b, 18, gid_a=ga, gid_b=gb)
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b, ga, gb)
        for _ in range(2):
            got, _ = ctx.sort_and_sweep(oa, ob, -1)
            assert np.array_equal(orc.canonical(got), want)
        got, _ = ctx.sort_and_sweep(ob, oa, 1)  # swapped roles: (gid in b, gid in a)
        assert np.array_equal(orc.canonical(got[:, ::-1].copy()), want)


def test_precision_form_gives_the_same_set():
    a = meshes.random_soup(3000, 3, seed=1101, size=0.03)
    b = meshes.random_soup(2500, 3, seed=1102, size=0.03, stream=1)
    want = orc.pair_set(a, b, 18)
    with bvhg.Context(k=18, precision=bvhg.FILTER_FP32) as ctx:
        oa, ob = build_pair(ctx, a, b)
        got, _ = ctx.sort_and_sweep(oa, ob, -1)
        assert np.array_equal(orc.canonical(got), want)


def test_python_call_grows_its_buffer_once():
    """More pairs than the binding's first buffer (65,536): the sweep runs again into a buffer of the reported size;
    the next call starts with that size and runs once."""
    m = 40
    xyz = meshes.tet_lattice(m)
    even = meshes.checkerboard(m)
    a, b = np.ascontiguousarray(xyz[even]), np.ascontiguousarray(xyz[~even])
    want = orc.pair_set(a, b, 18)
    assert want.shape[0] > 65536
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b)
        for _ in range(2):
            got, _ = ctx.sort_and_sweep(oa, ob, -1)
            assert np.array_equal(orc.canonical(got), want)


def test_device_output_overflow_and_errors():
    torch = pytest.importorskip("torch")
    a = meshes.random_soup(3000, 3, seed=1201, size=0.03)
    b = meshes.random_soup(2500, 3, seed=1202, size=0.03, stream=1)
    want = orc.pair_set(a, b, 18)
    n = want.shape[0]
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b)
        out = torch.empty((n, 2), dtype=torch.int64, device="cuda")
        st, cnt, _ = ctx.sort_and_sweep_raw(oa, ob, -1, out.data_ptr(), n, bvhg.MEM_DEVICE)
        assert st == 0 and cnt == n
        assert np.array_equal(orc.canonical(out.cpu().numpy().view(np.uint64)), want)
        small = np.empty((4, 2), dtype=np.uint64)
        st, cnt, _ = ctx.sort_and_sweep_raw(oa, ob, -1, small.ctypes.data, 4, bvhg.MEM_HOST)
        assert st == bvhg._abi.ERR_OVERFLOW and cnt == n
        assert ctx.sort_and_sweep_raw(oa, oa, -1, None, 0, bvhg.MEM_HOST)[0] == bvhg._abi.ERR_ARG
        assert ctx.sort_and_sweep_raw(oa, ob, 3, None, 0, bvhg.MEM_HOST)[0] == bvhg._abi.ERR_ARG
        oc = ctx.object()
        assert ctx.sort_and_sweep_raw(oa, oc, -1, None, 0, bvhg.MEM_HOST)[0] == bvhg._abi.ERR_STATE
        empty = np.empty((0, 3, 3))
        ctx.set_elements(oc, empty)
        ctx.build(oc)
        got, _ = ctx.sort_and_sweep(oa, oc, -1)
        assert got.shape[0] == 0
        # the context is still usable after the error returns
        got, _ = ctx.sort_and_sweep(oa, ob, 0)
        assert np.array_equal(orc.canonical(got), want)
        # a refit keeps the last rebuild's bounds and centroids: the sweep needs a rebuild first
        ctx.build(ob, bvhg.REFIT)
        assert ctx.sort_and_sweep_raw(oa, ob, -1, None, 0, bvhg.MEM_HOST)[0] == bvhg._abi.ERR_STATE
        ctx.build(ob)
        got, _ = ctx.sort_and_sweep(oa, ob, -1)
        assert np.array_equal(orc.canonical(got), want)


@pytest.mark.parametrize("k", [6, 18, 26])
def test_reference_known_answers(k):
    """tests/KokkosTest.cpp:37-140: max_variant_axis picks the grid's long axis; sort_and_sweep_local of a
    12-element grid against one element finds 12 pairs in both roles."""
    from tests.grids import element_grid
    b, gb = element_grid(1, 1, 1, 0)
    with bvhg.Context(k=k) as ctx:
        for dims, axis in (((12, 1, 1), 0), ((1, 12, 1), 1), ((1, 1, 12), 2)):
            a, ga = element_grid(*dims, 0)
            oa, ob = build_pair(ctx, a, b, ga, gb)
            got, used = ctx.sort_and_sweep(oa, ob, -1)
            assert used == axis
            assert got.shape[0] == 12 and set(got[:, 1].tolist()) == {0} and sorted(got[:, 0].tolist()) == list(range(12))
            got, _ = ctx.sort_and_sweep(ob, oa, 0)
            assert got.shape[0] == 12 and set(got[:, 0].tolist()) == {0}


def test_gpu_sweep_matches_the_reference_vectors():
    """bvhg_sort_and_sweep against the pairs and axis of the reference's own sort_and_sweep_local and
    max_variant_axis (dop_26 and dop_6), stored in tests/golden/ref_vectors.npz."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_vectors.npz"))
    checked = 0
    for name in g["cases"]:
        name = str(name)
        if not name.startswith("soup"):
            continue
        a, b, eps = g[f"{name}/a"], g[f"{name}/b"], float(g[f"{name}/eps"])
        for k in (26, 6):
            with bvhg.Context(k=k, epsilon=eps) as ctx:
                oa, ob = build_pair(ctx, a, b)
                got, used = ctx.sort_and_sweep(oa, ob, -1)
                assert used == int(g[f"{name}/sweep{k}/axis"])
                assert np.array_equal(orc.canonical(got), orc.canonical(g[f"{name}/sweep{k}/pairs"])), (name, k)
                checked += 1
    assert checked == 12
