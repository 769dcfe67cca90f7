"""GPU parity: every stage of the CUDA path against the CPU oracle, through the C ABI.

Bit-exact for everything integer or FP64 (slabs, centroids, Morton bounds and keys, permutation, pair sets).
The FP32 precision form must give the identical pair set after its FP64 recheck, and its FP32 slabs must
enclose the FP64 slabs. Sizes keep the oracle to seconds; the benchmark-sized scenes are checked against the
oracle in test_gpu_full_size.py.
"""
import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc
from tests.grids import clustered_soup, distinct_cells, element_grid

pytestmark = pytest.mark.gpu


def u64(a):
    return np.ascontiguousarray(a).view(np.uint64)


def build_pair(ctx, a, b, ga=None, gb=None):
    oa, ob = ctx.object(), ctx.object()
    ctx.set_elements(oa, a, gid=ga)
    ctx.set_elements(ob, b, gid=gb)
    ctx.build(oa)
    ctx.build(ob)
    return oa, ob


def check_stages(ctx, obj, xyz, k, eps):
    n = xyz.shape[0]
    s = orc.kdops(xyz, k, eps)
    c = orc.centroids(xyz)
    assert np.array_equal(u64(ctx.kdops(obj, n)), u64(s)), "FP64 slabs differ from kdop_base::from_vertices"
    assert np.array_equal(u64(ctx.centroids(obj, n)), u64(c)), "centroids differ"
    mn, inv = orc.morton_bounds(s, k)
    okeys = orc.morton_keys(c, mn, inv)
    operm = orc.stable_perm(okeys)
    keys, perm, gmn, ginv = ctx.morton(obj, n)
    assert np.array_equal(gmn, mn) and np.array_equal(u64(ginv), u64(inv)), "Morton bounds differ"
    assert np.array_equal(perm, operm), "permutation differs from the stable sort"
    assert np.array_equal(keys, okeys[operm]), "sorted Morton keys differ"
    ctx.validate_tree(obj)


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("V", [3, 4, 8])
@pytest.mark.parametrize("eps", [0.0, 0.004])
def test_stages_and_pairs(k, V, eps):
    a = meshes.random_soup(3000, V, seed=100 + V, size=0.03)
    b = meshes.random_soup(2500, V, seed=200 + V, size=0.03, stream=1)
    with bvhg.Context(k=k, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, a, b)
        check_stages(ctx, oa, a, k, eps)
        check_stages(ctx, ob, b, k, eps)
        got = orc.canonical(ctx.broadphase(oa, ob))
        want = orc.pair_set(a, b, k, eps)
        assert want.shape[0] > 0
        assert np.array_equal(got, want)
        # swapped roles give the transposed set
        got_ba = orc.canonical(ctx.broadphase(ob, oa))
        assert np.array_equal(got_ba, orc.canonical(want[:, ::-1]))


@pytest.mark.parametrize("bits", [1, 2, 4])
def test_digit_width_gives_the_same_permutation(bits):
    a = meshes.random_soup(20000, 3, seed=5, size=0.01)
    b = meshes.random_soup(15000, 3, seed=6, size=0.01, stream=1)
    with bvhg.Context(k=18, digit_bits=8) as c8, bvhg.Context(k=18, digit_bits=bits) as cb:
        a8, b8 = build_pair(c8, a, b)
        ab, bb = build_pair(cb, a, b)
        k8, p8, _, _ = c8.morton(a8, a.shape[0])
        kb, pb, _, _ = cb.morton(ab, a.shape[0])
        assert np.array_equal(p8, pb) and np.array_equal(k8, kb)
        assert np.array_equal(orc.canonical(c8.broadphase(a8, b8)), orc.canonical(cb.broadphase(ab, bb)))


def test_many_tiles_sort():
    a = meshes.random_soup(300000, 3, seed=9, size=0.002)
    with bvhg.Context(k=18) as ctx:
        oa = ctx.object()
        ctx.set_elements(oa, a)
        ctx.build(oa)
        check_stages(ctx, oa, a, 18, 0.0)


@pytest.mark.parametrize("counts", [(2, 5, 31, 32), (33, 3), (500, 40, 7), (2048, 2049, 1), (100000, 34)])
def test_runs_of_equal_high_key_halves(counts):
    """The build sorts by the high key half, then orders each run of equal high halves by the low half on the
    device: runs of up to 32 by every element's own rank, longer ones by the run sort (a shared-memory network up to
    2048 elements, LSD passes beyond). The permutation read back is the device's own, and it must be the stable order
    of the oracle's keys; the pair sets must be exact."""
    a = clustered_soup(counts, seed=sum(counts))
    b = clustered_soup(counts[::-1], seed=7 + sum(counts))
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b)
        check_stages(ctx, oa, a, 18, 0.0)
        check_stages(ctx, ob, b, 18, 0.0)
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), orc.pair_set(a, b, 18))
        assert np.array_equal(orc.canonical(ctx.self_collision(oa)), orc.self_pair_set(a, 18))


@pytest.mark.parametrize("bits", [1, 8])
def test_many_long_runs(bits):
    """Hundreds of runs beyond the fix-up's limit, more than there are blocks of the run sort, at two digit
    widths of the high-half passes."""
    rng = np.random.default_rng(77)
    counts = rng.integers(33, 300, size=400)
    a = clustered_soup(counts, seed=78, cells=distinct_cells(counts.shape[0], 79))
    with bvhg.Context(k=18, digit_bits=bits) as ctx:
        o = ctx.object()
        ctx.set_elements(o, a)
        ctx.build(o)
        check_stages(ctx, o, a, 18, 0.0)


def test_all_keys_equal():
    """Every element identical: one run covering the whole object (the LSD path), key ties kept in index order."""
    tri = meshes.random_soup(1, 3, seed=4, size=0.1)
    a = np.ascontiguousarray(np.repeat(tri, 5000, axis=0))
    with bvhg.Context(k=18) as ctx:
        o = ctx.object()
        ctx.set_elements(o, a)
        ctx.build(o)
        check_stages(ctx, o, a, 18, 0.0)
        keys, perm, _, _ = ctx.morton(o, a.shape[0])
        assert np.all(keys == keys[0]) and np.array_equal(perm, np.arange(a.shape[0], dtype=np.uint32))


def test_two_plates_config():
    a, b = meshes.two_plates()
    eps = meshes.TWO_PLATES_EPSILON
    with bvhg.Context(k=18, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, a, b)
        check_stages(ctx, oa, a, 18, eps)  # plate A is flat: the z axis takes the NaN -> 0 path
        check_stages(ctx, ob, b, 18, eps)
        got = orc.canonical(ctx.broadphase(oa, ob))
    want = orc.pair_set(a, b, 18, eps)
    assert want.shape[0] > 10000
    assert np.array_equal(got, want)


def test_sphere_plate_small():
    s, p = meshes.sphere_plate(level=5, nx=256, ny=128)
    with bvhg.Context(k=18) as ctx:
        os_, op = build_pair(ctx, s, p)
        check_stages(ctx, os_, s, 18, 0.0)
        check_stages(ctx, op, p, 18, 0.0)
        got = orc.canonical(ctx.broadphase(os_, op))
    want = orc.pair_set(s, p, 18)
    assert want.shape[0] > 0
    assert np.array_equal(got, want)


@pytest.mark.parametrize("k", [6, 18, 26])
def test_self_collision(k):
    a = meshes.random_soup(4000, 4, seed=31, size=0.03)
    with bvhg.Context(k=k) as ctx:
        oa = ctx.object()
        ctx.set_elements(oa, a)
        ctx.build(oa)
        got = orc.canonical(ctx.self_collision(oa))
    assert np.all(got[:, 0] < got[:, 1])
    assert np.array_equal(got, orc.self_pair_set(a, k))


def test_reference_grids():
    # tests/CollisionTest.cpp:43-81 on the GPU: 64 pairs; 0 self pairs for touching cubes; 8 self pairs
    a, ga = element_grid(4, 4, 4)
    b, gb = element_grid(1, 1, 1, a.shape[0])
    with bvhg.Context(k=26) as ctx:
        oa, ob = build_pair(ctx, a, b, ga, gb)
        got = orc.canonical(ctx.broadphase(oa, ob))
        assert got.shape[0] == 64
        assert np.array_equal(got, orc.pair_set(a, b, 26, gid_a=ga, gid_b=gb))
        t = ctx.object()
        x, _ = element_grid(2, 2, 1)
        ctx.set_elements(t, x)
        ctx.build(t)
        assert ctx.self_collision(t).shape[0] == 0
        u = ctx.object()
        x2 = np.concatenate([element_grid(2, 2, 2)[0], element_grid(1, 1, 1)[0]])
        ctx.set_elements(u, x2)
        ctx.build(u)
        assert ctx.self_collision(u).shape[0] == 8


def test_duplicate_keys_and_dense_pairs():
    tet = meshes.random_soup(1, 4, seed=3, size=0.1)
    a = np.repeat(tet, 300, axis=0)
    b = np.repeat(tet, 200, axis=0)
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b)
        check_stages(ctx, oa, a, 18, 0.0)
        got = orc.canonical(ctx.broadphase(oa, ob))
        assert got.shape[0] == 300 * 200
        assert np.array_equal(got, orc.pair_set(a, b, 18, method="brute"))
        assert ctx.self_collision(oa).shape[0] == 300 * 299 // 2


@pytest.mark.parametrize("na,nb", [(0, 5), (5, 0), (1, 1), (1, 50), (2, 3), (50, 1)])
def test_tiny_objects(na, nb):
    a = meshes.random_soup(max(na, 1), 3, seed=41, size=0.4)[:na]
    b = meshes.random_soup(max(nb, 1), 3, seed=42, size=0.4, stream=1)[:nb]
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b)
        got = orc.canonical(ctx.broadphase(oa, ob))
        want = orc.pair_set(a, b, 18, method="brute") if na and nb else np.zeros((0, 2), np.uint64)
        assert np.array_equal(got, want)
        if na >= 2:
            assert np.array_equal(orc.canonical(ctx.self_collision(oa)), orc.self_pair_set(a, 18, method="brute"))


@pytest.mark.parametrize("k", [18, 26])
def test_fp32_filter_exact_after_recheck(k):
    a = meshes.random_soup(6000, 3, seed=51, size=0.02)
    b = meshes.random_soup(5000, 3, seed=52, size=0.02, stream=1)
    eps = 0.001
    with bvhg.Context(k=k, precision=bvhg.FILTER_FP32, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, a, b)
        f32 = ctx.kdops(oa, a.shape[0]).astype(np.float64)
        f64 = orc.kdops(a, k, eps)
        assert np.all(f32[..., 0] <= f64[..., 0]) and np.all(f32[..., 1] >= f64[..., 1]), "FP32 slabs not enclosing"
        got = orc.canonical(ctx.broadphase(oa, ob))
        cand = ctx.last_candidates()
        ctx.validate_tree(oa)
    want = orc.pair_set(a, b, k, eps)
    assert np.array_equal(got, want)
    assert cand >= want.shape[0]


def test_fp32_filter_touching_boundaries():
    # Exactly touching elements (FP64 slabs equal at the boundary) are not pairs; the FP32 filter keeps them as
    # candidates and the FP64 recheck removes them.
    a, _ = element_grid(6, 6, 6)
    b, _ = element_grid(6, 6, 6, origin_shift=1.0 / 6.0)
    with bvhg.Context(k=26, precision=bvhg.FILTER_FP32) as ctx:
        oa, ob = build_pair(ctx, a, b)
        got = orc.canonical(ctx.broadphase(oa, ob))
        cand = ctx.last_candidates()
    want = orc.pair_set(a, b, 26)
    assert np.array_equal(got, want)
    assert cand > want.shape[0]


def test_gid_mapping_and_device_input():
    torch = pytest.importorskip("torch")
    a = meshes.random_soup(2000, 3, seed=61, size=0.03)
    b = meshes.random_soup(2000, 3, seed=62, size=0.03, stream=1)
    rng = np.random.default_rng(0)
    ga = rng.choice(1 << 40, a.shape[0], replace=False).astype(np.uint64)
    gb = rng.choice(1 << 40, b.shape[0], replace=False).astype(np.uint64)
    want = orc.pair_set(a, b, 18, gid_a=ga, gid_b=gb)
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b, ga, gb)
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want)
        da = torch.from_numpy(a).cuda()
        db = torch.from_numpy(b).cuda()
        dga = torch.from_numpy(ga.view(np.int64)).cuda()
        dgb = torch.from_numpy(gb.view(np.int64)).cuda()
        torch.cuda.synchronize()
        ctx.set_elements(oa, da, gid=dga)
        ctx.set_elements(ob, db, gid=dgb)
        ctx.build(oa)
        ctx.build(ob)
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want)
        # device output buffer
        out = torch.empty((want.shape[0], 2), dtype=torch.int64, device="cuda")
        st, cnt = ctx.broadphase_raw(oa, ob, out.data_ptr(), want.shape[0], bvhg.MEM_DEVICE)
        assert st == 0 and cnt == want.shape[0]
        assert np.array_equal(orc.canonical(out.cpu().numpy().view(np.uint64)), want)


def test_overflow_reports_required_count():
    a = meshes.random_soup(3000, 3, seed=71, size=0.05)
    b = meshes.random_soup(3000, 3, seed=72, size=0.05, stream=1)
    want = orc.pair_set(a, b, 18)
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b)
        out = np.empty((10, 2), dtype=np.uint64)
        st, cnt = ctx.broadphase_raw(oa, ob, out.ctypes.data, 10, bvhg.MEM_HOST)
        assert st == 3 and cnt == want.shape[0]
        # the first `capacity` pairs written are genuine pairs
        wset = set(map(tuple, want.tolist()))
        assert all(tuple(p) in wset for p in out.tolist())
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob, capacity=cnt)), want)


def test_non_finite_input_is_rejected():
    a = meshes.random_soup(500, 3, seed=81)
    a[17, 1, 2] = np.nan
    b = meshes.random_soup(500, 3, seed=82, stream=1)
    with bvhg.Context(k=18) as ctx:
        oa, ob = build_pair(ctx, a, b)
        with pytest.raises(bvhg.BvhgError) as e:
            ctx.broadphase(oa, ob)
        assert e.value.status == 1


def test_bounded_lookback_times_out_and_context_recovers():
    a = meshes.random_soup(50000, 3, seed=91, size=0.01)
    b = meshes.random_soup(20000, 3, seed=92, size=0.01, stream=1)
    with bvhg.Context(k=18) as ctx:
        ctx.set_spin_limit(2000)
        ctx.test_stall_sort(True)
        oa, ob = build_pair(ctx, a, b)
        with pytest.raises(bvhg.BvhgError) as e:
            ctx.broadphase(oa, ob)
        assert e.value.status == 4
        ctx.test_stall_sort(False)
        ctx.set_spin_limit(0)
        ctx.build(oa)
        ctx.build(ob)
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), orc.pair_set(a, b, 18))


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
def test_refit_after_motion(precision):
    a = meshes.random_soup(4000, 3, seed=101, size=0.03)
    b = meshes.random_soup(4000, 3, seed=102, size=0.03, stream=1)
    with bvhg.Context(k=18, precision=precision) as ctx:
        oa, ob = build_pair(ctx, a, b)
        for step in range(3):
            b2 = b + np.array([0.01 * (step + 1), -0.005 * step, 0.003])
            ctx.set_elements(ob, b2)
            ctx.build(ob, bvhg.REFIT)
            ctx.validate_tree(ob)
            assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), orc.pair_set(a, b2, 18))


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
@pytest.mark.parametrize("k", [6, 18, 26])
def test_refit_after_deformation_over_many_blocks(k, precision):
    """A non-rigid motion over 25,000 buckets (196 refit blocks, the last one ragged): every node's slabs after the
    refit are the exact unions of what they cover, whether the node lies inside one block's buckets or crosses
    blocks, and the pair set is the oracle's for the moved vertices."""
    a = meshes.random_soup(150000, 3, seed=103, size=0.004)
    b = meshes.random_soup(199993, 3, seed=104, size=0.004, stream=1)
    with bvhg.Context(k=k, precision=precision) as ctx:
        oa, ob = build_pair(ctx, a, b)
        for step in range(2):
            w = 0.01 * (step + 1)
            b2 = b + w * np.sin(7.0 * b[..., ::-1] + step)
            ctx.set_elements(ob, b2)
            ctx.build(ob, bvhg.REFIT)
            ctx.validate_tree(ob)
            assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), orc.pair_set(a, b2, k))


def test_stage_timing_and_launch_count():
    a = meshes.random_soup(10000, 3, seed=111, size=0.02)
    with bvhg.Context(k=18, stage_timing=True) as ctx:
        oa = ctx.object()
        ctx.set_elements(oa, a)
        ctx.build(oa)
        ctx.self_collision(oa)
        ms, launches = ctx.stage_times()
        # four radix passes over the high key half, then the low-half fix-up and the sort of its long runs
        assert launches["sort"] == 4 and launches["fixup"] == 2 and launches["slabs"] == 1 and launches["build"] == 1 and launches["climb"] == 1
        assert launches["traverse"] >= 1
        assert all(v >= 0 for v in ms.values()) and ms["sort"] > 0
        assert ctx.launch_count() >= 12


GOLDEN = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "ref_vectors.npz"))


@pytest.mark.parametrize("case", [str(c) for c in GOLDEN["cases"]])
@pytest.mark.parametrize("k", [6, 18, 26])
def test_gpu_matches_reference_vectors(case, k):
    """The CUDA path against vectors computed by the reference's own code (tests/golden/make_golden.py)."""
    g = lambda key: GOLDEN[f"{case}/{key}"]  # noqa: E731
    a, b, eps = g("a"), g("b"), float(g("eps"))
    with bvhg.Context(k=k, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, a, b)
        for side, o, x in (("a", oa, a), ("b", ob, b)):
            n = x.shape[0]
            assert np.array_equal(u64(ctx.kdops(o, n)), u64(g(f"{side}/kdops{k}")))
            assert np.array_equal(u64(ctx.centroids(o, n)), u64(g(f"{side}/centroids")))
            keys, perm, mn, inv = ctx.morton(o, n)
            assert np.array_equal(u64(mn), u64(g(f"{side}/min3"))) and np.array_equal(u64(inv), u64(g(f"{side}/inv3")))
            want = g(f"{side}/keys")
            assert np.array_equal(perm, np.argsort(want, kind="stable")) and np.array_equal(keys, want[perm])
        got = orc.canonical(ctx.broadphase(oa, ob))
        self_got = orc.canonical(ctx.self_collision(oa))
        if k == 18:
            assert np.array_equal(got, orc.canonical(g("pairs18")))
        else:
            assert got.shape[0] == int(g(f"tree_count{k}"))
            assert np.array_equal(self_got, orc.canonical(np.sort(g(f"self{k}"), axis=1)))


def test_precision_form_on_the_tet_lattice():
    """The precision-form case at small size: a jittered 20^3 tet lattice, checkerboard objects, 26-DOP. FP64
    plain and FP32 filter + recheck both give the oracle's pair set; FP32 slabs enclose the FP64 slabs."""
    m = 20
    xyz = meshes.tet_lattice(m)
    even = meshes.checkerboard(m)
    a, b = np.ascontiguousarray(xyz[even]), np.ascontiguousarray(xyz[~even])
    want = orc.pair_set(a, b, 26)
    assert want.shape[0] > a.shape[0]  # dense contact: every tet overlaps several neighbours
    with bvhg.Context(k=26) as c64, bvhg.Context(k=26, precision=bvhg.FILTER_FP32) as c32:
        a64, b64 = build_pair(c64, a, b)
        a32, b32 = build_pair(c32, a, b)
        assert np.array_equal(orc.canonical(c64.broadphase(a64, b64)), want)
        assert np.array_equal(orc.canonical(c32.broadphase(a32, b32)), want)
        assert c32.last_candidates() >= want.shape[0]
        s64 = c64.kdops(a64, a.shape[0])
        s32 = c32.kdops(a32, a.shape[0]).astype(np.float64)
        assert (s32[:, :, 0] <= s64[:, :, 0]).all() and (s64[:, :, 1] <= s32[:, :, 1]).all()


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
@pytest.mark.parametrize("k", [6, 18, 26])
def test_stored_and_computed_element_slabs_agree(precision, k):
    """Traversals compute the element slabs they test from the vertices (sparse contact) or read the ones the build
    stored (dense contact, decided from the previous broadphase's candidate count; the walk then queues its leaf
    buckets and tests them in batches): both give the exact set."""
    m = 14
    xyz = meshes.tet_lattice(m)
    even = meshes.checkerboard(m)
    a, b = np.ascontiguousarray(xyz[even]), np.ascontiguousarray(xyz[~even])
    want = orc.pair_set(a, b, k)
    want_self = orc.self_pair_set(a, k)
    with bvhg.Context(k=k, precision=precision) as ctx:
        for step in range(3):  # first build: computed; later builds: stored (the contact is dense)
            oa, ob = (build_pair(ctx, a, b) if step == 0 else (oa, ob))
            if step:
                ctx.build(oa)
                ctx.build(ob)
            assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want), step
            assert np.array_equal(orc.canonical(ctx.self_collision(oa)), want_self), step
            ctx.validate_tree(oa)


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
def test_objects_with_different_vertex_counts(precision):
    """A triangle object against a tetrahedron object and a hexahedron object (the traversal's generic vertex
    path), sparse and dense, both orders."""
    tri = meshes.random_soup(3000, 3, seed=301, size=0.03)
    tet = meshes.random_soup(2500, 4, seed=302, size=0.03, stream=1)
    hexa = meshes.random_soup(800, 8, seed=303, size=0.06, stream=2)
    with bvhg.Context(k=18, precision=precision) as ctx:
        objs = {}
        for name, x in (("tri", tri), ("tet", tet), ("hex", hexa)):
            objs[name] = ctx.object()
            ctx.set_elements(objs[name], x)
            ctx.build(objs[name])
        for rep in range(2):  # the second pass runs after the density decision of the first
            for a, b in (("tri", "tet"), ("tet", "tri"), ("tri", "hex"), ("hex", "tet")):
                xa, xb = {"tri": tri, "tet": tet, "hex": hexa}[a], {"tri": tri, "tet": tet, "hex": hexa}[b]
                got = orc.canonical(ctx.broadphase(objs[a], objs[b]))
                assert np.array_equal(got, orc.pair_set(xa, xb, 18)), (rep, a, b)
            for name in objs:
                ctx.build(objs[name])


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("V", [3, 4, 8])
@pytest.mark.parametrize("eps", [0.0, -0.0, 0.25])
def test_signed_zeros_and_exact_cancellations(k, V, eps):
    """Coordinates from {+-0, +-0.25, +-1}: many projections cancel exactly or add signed zeros, which is where
    the kernels' shortcuts for the normal components 0 and +-1 must still give the bits of
    ((v0 * n0) + (v1 * n1)) + (v2 * n2) - eps / + eps. Slabs, centroids, bounds, keys and pairs, bit for bit."""
    rng = np.random.default_rng(1000 + 10 * k + V)
    values = np.array([-0.0, 0.0, 0.25, -0.25, 1.0, -1.0])
    a = values[rng.integers(0, len(values), size=(1500, V, 3))]
    b = values[rng.integers(0, len(values), size=(1200, V, 3))]
    assert np.signbit(a).any() and (a == 0).any()
    with bvhg.Context(k=k, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, a, b)
        check_stages(ctx, oa, a, k, eps)
        check_stages(ctx, ob, b, k, eps)
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), orc.pair_set(a, b, k, eps))


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("V", [3, 4, 8])
@pytest.mark.parametrize("eps", [0.0, 0.25])
def test_signed_zeros_filter_form_recheck(k, V, eps):
    """The same coordinates through the precision form: the FP32 candidates are rechecked in FP64 by projections
    that skip products by 0 and 1 and share the products by the normal magnitudes. Many slabs touch exactly
    (strict overlap fails by equality) or meet at signed zeros, so the recheck's outcome must be the FP64 one on
    every candidate: the pair set equals the oracle's, in both roles and for self-collision."""
    rng = np.random.default_rng(2000 + 10 * k + V)
    values = np.array([-0.0, 0.0, 0.25, -0.25, 1.0, -1.0])
    a = values[rng.integers(0, len(values), size=(1500, V, 3))]
    b = values[rng.integers(0, len(values), size=(1200, V, 3))]
    with bvhg.Context(k=k, epsilon=eps, precision=bvhg.FILTER_FP32) as ctx:
        oa, ob = build_pair(ctx, a, b)
        want = orc.pair_set(a, b, k, eps)
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want)
        assert np.array_equal(orc.canonical(ctx.broadphase(ob, oa)), orc.pair_set(b, a, k, eps))
        assert np.array_equal(orc.canonical(ctx.self_collision(oa)), orc.self_pair_set(a, k, eps))


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("V", [3, 4, 8])
def test_slab_paths_agree_bitwise(precision, k, V):
    """Elements of 3, 4 and 8 vertices take the kernels' unrolled slab code (FP32: every enclosure of an element
    from shared per-vertex roundings and products); any other vertex count takes the generic code, one vertex and
    one slab at a time. The same elements with their first vertex repeated (V + 1 vertices, the same slabs) must
    give the same bits through both, for random coordinates over many magnitudes and for cancelling ones."""
    rng = np.random.default_rng(3000 + 10 * k + V)
    soup = meshes.random_soup(4000, V, seed=40 + V, size=0.01)
    scaled = soup * (10.0 ** rng.integers(-20, 20, size=(4000, 1, 1)))
    values = np.array([-0.0, 0.0, 0.25, -0.25, 1.0, -1.0, 1e-40, -3e38])
    special = values[rng.integers(0, len(values), size=(2000, V, 3))]
    for xyz in (soup, scaled, special):
        padded = np.ascontiguousarray(np.concatenate([xyz, xyz[:, :1, :]], axis=1))
        for eps in (0.0, 0.003):
            with bvhg.Context(k=k, epsilon=eps, precision=precision) as ctx:
                o1, o2 = ctx.object(), ctx.object()
                ctx.set_elements(o1, xyz)
                ctx.set_elements(o2, padded)
                s1, s2 = ctx.kdops(o1, xyz.shape[0]), ctx.kdops(o2, xyz.shape[0])
                assert np.array_equal(s1.view(np.uint8), s2.view(np.uint8)), (eps, np.argwhere(s1 != s2)[:4])


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
def test_dense_walk_stack_bound_falls_back(precision):
    """The dense-contact walk pops several nodes per step, so its stack can grow past the tree depth; when it
    reaches its bound the library searches again with the single-node walk. A test hook lowers the bound until
    it is reached: the pair sets (inter-object, self, and in a batch) stay exact."""
    m = 14
    xyz = meshes.tet_lattice(m)
    even = meshes.checkerboard(m)
    a, b = np.ascontiguousarray(xyz[even]), np.ascontiguousarray(xyz[~even])
    want = orc.pair_set(a, b, 18)
    with bvhg.Context(k=18, precision=precision) as ctx:
        ctx.test_dense_stack(3)
        oa, ob = build_pair(ctx, a, b)
        assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want)  # dense from now on
        for _ in range(2):
            ctx.build(oa)
            ctx.build(ob)
            assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want)
            assert np.array_equal(orc.canonical(ctx.self_collision(oa)), orc.self_pair_set(a, 18))
    with bvhg.Context(k=18, precision=precision) as ctx:
        ctx.test_dense_stack(3)
        oa, ob = build_pair(ctx, a, b)
        for _ in range(3):
            got = ctx.batch_broadphase([(oa, ob)])
            assert np.array_equal(orc.canonical(got[0]), want)


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("eps", [0.0, 1e-3])
def test_fp32_dense_contact_of_touching_elements(k, eps):
    """Hexahedra of a grid touch their neighbours exactly, and the grid is split checkerboard-wise into two objects
    in dense contact: with epsilon 0 the touching faces are FP32 candidates (the outward-rounded slabs overlap) but
    not pairs, and the FP64 recheck must drop every one of them, in the computed-slab walk and in the dense walk over
    stored slabs; coordinates are scaled by an irrational factor so the 18- and 26-DOP projections round."""
    xyz, _ = element_grid(12, 12, 12)
    xyz = np.ascontiguousarray(xyz * np.sqrt(2.0) + 0.1)
    idx = np.arange(xyz.shape[0])
    i, j, l = idx % 12, (idx // 12) % 12, idx // 144
    even = (i + j + l) % 2 == 0
    a, b = np.ascontiguousarray(xyz[even]), np.ascontiguousarray(xyz[~even])
    want = orc.pair_set(a, b, k, eps)
    with bvhg.Context(k=k, precision=bvhg.FILTER_FP32, epsilon=eps) as ctx:
        oa, ob = build_pair(ctx, a, b)
        for _ in range(3):  # the first pass decides dense contact; later builds store the slabs
            assert np.array_equal(orc.canonical(ctx.broadphase(oa, ob)), want)
            ctx.build(oa)
            ctx.build(ob)
