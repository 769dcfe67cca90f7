"""The multi-rank broadphase (distbvh_b200.dist) as two gloo ranks on CPU.

Every rank holds part of the elements of objects A and B. The driver's host logic runs as in production (patch
boxes all-gathered, B patches requested and shipped as ghosts by all-to-all, exact pairs per rank); the element
work of each rank comes from the oracle here (patches by its morton_cluster restatement, boxes as unions of its
slabs, pairs by its exact pair set), since this machine has no GPU. The union of the ranks' pairs must be the
oracle's global pair set, every pair found once. A GPU test runs the same driver with the CUDA backend.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from distbvh_b200 import meshes  # noqa: E402


class OracleBackend:
    def __init__(self, k):
        from oracle import oracle as orc
        self.orc = orc
        self.k = k

    def patches(self, name, xyz, patches):
        orc = self.orc
        order, bounds = orc.morton_cluster(xyz, self.k, patches)
        d = self.k // 2
        boxes = np.empty((patches, d, 2))
        boxes[:, :, 0] = np.inf
        boxes[:, :, 1] = -np.inf
        if xyz.shape[0]:
            s = orc.kdops(xyz, self.k)
            for p in range(patches):
                idx = order[int(bounds[p]):int(bounds[p + 1])].astype(np.int64)
                if idx.size:
                    boxes[p, :, 0] = s[idx, :, 0].min(axis=0)
                    boxes[p, :, 1] = s[idx, :, 1].max(axis=0)
        return order, bounds, boxes

    def pairs(self, xyz_a, gid_a, xyz_b, gid_b):
        if xyz_a.shape[0] == 0 or xyz_b.shape[0] == 0:
            return np.zeros((0, 2), dtype=np.uint64)
        return self.orc.pair_set(xyz_a, xyz_b, self.k, gid_a=gid_a, gid_b=gid_b)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def scene():
    a = meshes.random_soup(3000, 3, seed=81, size=0.03)
    b = meshes.random_soup(2500, 3, seed=82, size=0.03, stream=1)
    return a, b, np.arange(a.shape[0], dtype=np.uint64) + 7, np.arange(b.shape[0], dtype=np.uint64) + 100000


def split(n, rank, world, how):
    idx = np.arange(n)
    if how == "interleaved":
        return idx[idx % world == rank]
    if how == "halves":
        return np.array_split(idx, world)[rank]
    return idx if rank == 0 else idx[:0]  # "one-sided": the last rank holds nothing


def worker(rank, world, port, how, patches, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    from distbvh_b200.dist import DistributedBroadphase
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        a, b, ga, gb = scene()
        ia, ib = split(a.shape[0], rank, world, how), split(b.shape[0], rank, world, "halves")
        db = DistributedBroadphase(OracleBackend(18), patches=patches)
        got = db.broadphase(a[ia], ga[ia], b[ib], gb[ib])
        q.put((rank, got.tolist(), db.stats))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("how", ["interleaved", "halves", "one-sided"])
@pytest.mark.parametrize("patches", [1, 8])
def test_two_ranks_find_the_global_pair_set_once(how, patches):
    from oracle import oracle as orc
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(worker, args=(2, free_port(), how, patches, q), nprocs=2, start_method="spawn")
    res = sorted(q.get() for _ in range(2))
    got = np.array([p for _, pairs, _ in res for p in pairs], dtype=np.uint64).reshape(-1, 2)
    a, b, ga, gb = scene()
    want = orc.pair_set(a, b, 18, gid_a=ga, gid_b=gb)
    assert want.shape[0] > 0
    assert got.shape[0] == want.shape[0], "a pair was found twice or missed"
    assert np.array_equal(orc.canonical(got), want)
    # every rank fetched at most all B patches of every rank
    assert all(st["patches_needed"] <= 2 * patches for _, _, st in res)


@pytest.mark.gpu
def test_cuda_backend_single_rank():
    """The driver on one rank with the CUDA backend (patches and boxes from the device, pairs through the C ABI)."""
    from oracle import oracle as orc
    from distbvh_b200.dist import CudaBackend, DistributedBroadphase
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(free_port()))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        a, b, ga, gb = scene()
        be = CudaBackend(k=18)
        db = DistributedBroadphase(be, patches=8)
        got = db.broadphase(a, ga, b, gb)
        assert np.array_equal(orc.canonical(got), orc.pair_set(a, b, 18, gid_a=ga, gid_b=gb))
        # the device's patch boxes are the unions of the oracle's element slabs
        _, _, boxes = be.patches("B", b, 8)
        _, _, want_boxes = OracleBackend(18).patches("B", b, 8)
        assert np.array_equal(boxes, want_boxes)
        be.close()
    finally:
        dist.destroy_process_group()
