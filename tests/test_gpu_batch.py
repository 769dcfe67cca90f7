"""Batching form: many independent scenes as one CUDA graph (bvhg_batch_broadphase), against the oracle.

Scenes of uneven sizes (including an empty object and a self-collision scene) must each give the exact pair set
of the single-scene path, in every form of the batch graph (fused: one launch per pipeline stage for one group of
objects or several; per-object launches on concurrent streams); replays of the captured graph after coordinates
change in place must too (REBUILD and REFIT); the autotuner must pick one of its configurations and leave the
context usable.
"""
import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def make_scenes(seed, nscenes, k):
    rng = np.random.default_rng(seed)
    bodies = []
    for s in range(nscenes):
        n_a, n_b = (int(x) for x in np.exp(rng.uniform(np.log(50), np.log(4000), 2)))
        size = 0.6 * (n_a + n_b) ** (-1.0 / 3.0)
        a = meshes.random_soup(n_a, 3, seed=seed * 1000 + 2 * s, size=size)
        b = meshes.random_soup(n_b, 3, seed=seed * 1000 + 2 * s + 1, size=size, stream=1)
        bodies.append((a, b))
    return bodies


FORMS = [(1, 1), (5, 3), (16, 16), (0, 4)]  # (groups, lanes): fused with 1, 5 or 16 groups; per-object launches


@pytest.mark.parametrize("precision", [bvhg.PLAIN_FP64, bvhg.FILTER_FP32])
@pytest.mark.parametrize("form", FORMS)
def test_batch_matches_single_scenes(precision, form):
    bodies = make_scenes(5, 12, 18)
    with bvhg.Context(k=18, precision=precision) as ctx:
        ctx.test_batch_form(*form)
        objs = []
        for a, b in bodies:
            oa, ob = ctx.object(), ctx.object()
            ctx.set_elements(oa, a)
            ctx.set_elements(ob, b)
            objs.append((oa, ob))
        empty = ctx.object()
        ctx.set_elements(empty, np.zeros((0, 3, 3)))
        scenes = objs + [(objs[0][0], objs[0][0]), (empty, objs[1][1])]
        for rep in range(2):  # capture, then replay
            got = ctx.batch_broadphase(scenes)
            for s, (a, b) in enumerate(bodies):
                assert np.array_equal(orc.canonical(got[s]), orc.pair_set(a, b, 18)), (rep, s)
            assert np.array_equal(orc.canonical(got[len(bodies)]), orc.self_pair_set(bodies[0][0], 18))
            assert got[len(bodies) + 1].shape[0] == 0
        # the objects are built: single-scene calls agree
        assert np.array_equal(orc.canonical(ctx.broadphase(*objs[3])), orc.pair_set(*bodies[3], 18))


@pytest.mark.parametrize("form", FORMS)
def test_batch_replay_after_motion_rebuild_and_refit(form):
    bodies = make_scenes(9, 8, 18)
    dev = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in bodies]
    with bvhg.Context(k=18) as ctx:
        ctx.test_batch_form(*form)
        objs = []
        for da, db in dev:
            oa, ob = ctx.object(), ctx.object()
            ctx.set_elements(oa, da)
            ctx.set_elements(ob, db)
            objs.append((oa, ob))
        ctx.batch_broadphase(objs, mode=bvhg.REBUILD)
        for step, mode in enumerate((bvhg.REFIT, bvhg.REBUILD, bvhg.REFIT)):
            shift = torch.tensor([0.003 * (step + 1), -0.002, 0.001], dtype=torch.float64, device="cuda")
            for (da, db) in dev:
                db += shift  # in place: the borrowed device pointers stay the same, the graph replays
            torch.cuda.synchronize()
            got = ctx.batch_broadphase(objs, mode=mode)
            for s, (da, db) in enumerate(dev):
                want = orc.pair_set(da.cpu().numpy(), db.cpu().numpy(), 18)
                assert np.array_equal(orc.canonical(got[s]), want), (step, s)


def test_batch_autotune_picks_a_configuration():
    bodies = make_scenes(13, 24, 18)
    with bvhg.Context(k=18) as ctx:
        objs = []
        for a, b in bodies:
            oa, ob = ctx.object(), ctx.object()
            ctx.set_elements(oa, a)
            ctx.set_elements(ob, b)
            objs.append((oa, ob))
        groups, lanes, ms = ctx.batch_autotune(objs)
        assert (groups, lanes) in ((1, 1), (4, 4), (16, 16), (64, 16), (256, 16), (0, 16), (0, 64)) and ms > 0
        got = ctx.batch_broadphase(objs)
        for s, (a, b) in enumerate(bodies):
            assert np.array_equal(orc.canonical(got[s]), orc.pair_set(a, b, 18))


def test_batch_refuses_device_memory_for_host_arrays():
    """Scene arrays, counts and offsets are host memory: a device pointer among them is an argument error (the call
    must not write through it), and the context stays usable."""
    a = meshes.random_soup(2000, 3, seed=71, size=0.04)
    b = meshes.random_soup(1500, 3, seed=72, size=0.04, stream=1)
    with bvhg.Context(k=18) as ctx:
        oa, ob = ctx.object(), ctx.object()
        ctx.set_elements(oa, a)
        ctx.set_elements(ob, b)
        ia = np.array([oa], dtype=np.int32)
        ib = np.array([ob], dtype=np.int32)
        out = torch.empty((1 << 16, 2), dtype=torch.int64, device="cuda")
        d_counts = torch.zeros(1, dtype=torch.int64, device="cuda")
        st = ctx.batch_broadphase_raw(ia.ctypes.data, ib.ctypes.data, 1, bvhg.REBUILD, out.data_ptr(), out.shape[0],
                                      d_counts.data_ptr(), bvhg.MEM_DEVICE)
        assert st == bvhg._abi.ERR_ARG
        d_ia = torch.from_numpy(ia).cuda()
        counts = np.zeros(1, dtype=np.uint64)
        st = ctx.batch_broadphase_raw(d_ia.data_ptr(), ib.ctypes.data, 1, bvhg.REBUILD, out.data_ptr(), out.shape[0],
                                      counts.ctypes.data, bvhg.MEM_DEVICE)
        assert st == bvhg._abi.ERR_ARG
        got = ctx.batch_broadphase([(oa, ob)])
        assert np.array_equal(orc.canonical(got[0]), orc.pair_set(a, b, 18))
