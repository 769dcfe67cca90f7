"""Multi-rank broadphase: objects whose elements are spread over ranks (one process per GPU, torch.distributed).

This is the distributed layer of the reference's collision_object (src/bvh/collision_object.cpp:148-397) without
its vt runtime. There every rank cuts its local elements into od_factor patches; the patches' k-DOPs are reduced to
one rank, which builds the patch tree and broadcasts it (src/bvh/collision_object/top_down.cpp:103-127); patch
pairs whose k-DOPs overlap are then narrowphased on one rank, with the remote patch's elements fetched as a ghost
(src/bvh/collision_object/impl.cpp:230-265). Here one broadphase between objects A and B is:

  1. on every rank, the local elements of A and of B are built and cut into patches on the device
     (bvhg_build, bvhg_cluster) and the patch boxes computed there (bvhg_patch_kdops);
  2. one all-gather gives every rank every B patch box (the reduce + broadcast of the patch tree, as one
     collective);
  3. every rank asks each rank for the B patches whose boxes overlap one of its own A patch boxes (strict overlap
     on every slab: an element pair can only overlap if their patches' boxes do), and receives their elements'
     vertices and global ids in one all-to-all (the ghost exchange);
  4. every rank runs the exact element broadphase of its A elements against the B elements it holds (its own
     needed patches and the ghosts) on its GPU.

Every pair (a, b) of S(A, B) is found exactly once, by the rank that owns a; the union over ranks is the global
pair set. Self-collision across ranks is not handled (the reference's narrowphase skips it too).

The element work goes through a backend: CudaBackend runs it on this rank's GPU through the C ABI. The collectives
run on the process group's device: CUDA tensors for NCCL, host tensors for gloo.
"""
import numpy as np


def _strict_overlap(boxes_a, boxes_b):
    """(na, nb) bool: box i of a overlaps box j of b strictly on every slab (boxes: (n, D, 2))."""
    if boxes_a.shape[0] == 0 or boxes_b.shape[0] == 0:
        return np.zeros((boxes_a.shape[0], boxes_b.shape[0]), dtype=bool)
    amin = boxes_a[:, None, :, 0]
    amax = boxes_a[:, None, :, 1]
    bmin = boxes_b[None, :, :, 0]
    bmax = boxes_b[None, :, :, 1]
    return np.all((amin < bmax) & (bmin < amax), axis=2)


class CudaBackend:
    """The element work of one rank on its GPU: patches (bvhg_cluster, bvhg_patch_kdops) and exact pairs
    (bvhg_broadphase with global ids)."""

    def __init__(self, k=18, precision=0, epsilon=0.0, device=0):
        from . import _abi
        self._abi = _abi
        self.ctx = _abi.Context(k=k, precision=precision, epsilon=epsilon, device=device)
        self.k = k
        self._objs = {}

    def _obj(self, name):
        if name not in self._objs:
            self._objs[name] = self.ctx.object()
        return self._objs[name]

    def patches(self, name, xyz, patches):
        """Builds the local elements of object `name` and cuts them into patches: (order (n,), bounds (P + 1,),
        boxes (P, D, 2))."""
        o = self._obj(name)
        self.ctx.set_elements(o, np.ascontiguousarray(xyz, dtype=np.float64))
        self.ctx.build(o)
        bounds, order = self.ctx.cluster(o, patches, xyz.shape[0])
        return order, bounds, self.ctx.patch_kdops(o, patches)

    def pairs(self, xyz_a, gid_a, xyz_b, gid_b):
        """Exact pairs (gid_a, gid_b) between two element sets, as an (m, 2) uint64 array."""
        if xyz_a.shape[0] == 0 or xyz_b.shape[0] == 0:
            return np.zeros((0, 2), dtype=np.uint64)
        oa, ob = self._obj("__pairs_a"), self._obj("__pairs_b")
        self.ctx.set_elements(oa, np.ascontiguousarray(xyz_a, dtype=np.float64),
                              gid=np.ascontiguousarray(gid_a, dtype=np.uint64))
        self.ctx.set_elements(ob, np.ascontiguousarray(xyz_b, dtype=np.float64),
                              gid=np.ascontiguousarray(gid_b, dtype=np.uint64))
        self.ctx.build(oa)
        self.ctx.build(ob)
        return self.ctx.broadphase(oa, ob)

    def close(self):
        self.ctx.close()


class DistributedBroadphase:
    """One broadphase between two objects whose elements are spread over the ranks of a process group.

    backend: the element work of this rank (CudaBackend, or any object with the same `patches` and `pairs`
    methods). patches: od_factor, the patches per object and rank. device: where the collectives' tensors live
    ("cuda:i" for NCCL, "cpu" for gloo)."""

    def __init__(self, backend, patches=8, group=None, device="cpu"):
        import torch
        import torch.distributed as dist
        self.torch = torch
        self.dist = dist
        self.backend = backend
        self.patches = patches
        self.group = group
        self.device = torch.device(device)
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.stats = {}

    def _all_gather(self, arr):
        t = self.torch.from_numpy(np.ascontiguousarray(arr)).to(self.device)
        outs = [self.torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(outs, t, group=self.group)
        return [o.cpu().numpy() for o in outs]

    def _all_to_all(self, parts, dtype, width):
        """parts[r]: an (m_r, width) array for rank r; returns the arrays the other ranks sent here, in rank order."""
        torch = self.torch
        send_sizes = [int(p.shape[0]) * width for p in parts]
        ss = torch.tensor(send_sizes, dtype=torch.int64, device=self.device)
        rs = torch.empty(self.world, dtype=torch.int64, device=self.device)
        self.dist.all_to_all_single(rs, ss, group=self.group)
        recv_sizes = rs.cpu().tolist()
        flat = np.concatenate([np.ascontiguousarray(p, dtype=dtype).reshape(-1) for p in parts]) if parts else \
            np.zeros(0, dtype=dtype)
        send = torch.from_numpy(np.ascontiguousarray(flat)).to(self.device)
        recv = torch.empty(int(sum(recv_sizes)), dtype=send.dtype, device=self.device)
        self.dist.all_to_all_single(recv, send, output_split_sizes=recv_sizes, input_split_sizes=send_sizes,
                                    group=self.group)
        out = recv.cpu().numpy()
        res, off = [], 0
        for n in recv_sizes:
            res.append(out[off:off + n].reshape(-1, width))
            off += n
        return res

    def broadphase(self, xyz_a, gid_a, xyz_b, gid_b):
        """This rank's share of S(A, B): the exact pairs (gid_a, gid_b) of its A elements with every B element of
        any rank, as an (m, 2) uint64 array. Collective: every rank of the group calls it."""
        P = self.patches
        xyz_a = np.ascontiguousarray(xyz_a, dtype=np.float64)
        xyz_b = np.ascontiguousarray(xyz_b, dtype=np.float64)
        V = xyz_b.shape[1]
        _, _, boxes_a = self.backend.patches("A", xyz_a, P)
        order_b, bounds_b, boxes_b = self.backend.patches("B", xyz_b, P)
        # 2. every rank's B patch boxes
        all_boxes = self._all_gather(boxes_b)
        # 3. the B patches this rank needs from each rank; requests out, requested patches' elements back
        need = [np.nonzero(_strict_overlap(boxes_a, bx).any(axis=0))[0].astype(np.int64) for bx in all_boxes]
        asked = self._all_to_all([n.reshape(-1, 1) for n in need], np.int64, 1)
        send_xyz, send_gid = [], []
        gid_b = np.ascontiguousarray(gid_b, dtype=np.uint64)
        for req in asked:
            idx = np.concatenate([order_b[int(bounds_b[p]):int(bounds_b[p + 1])] for p in req.reshape(-1)]) \
                if req.size else np.zeros(0, dtype=np.uint32)
            idx = idx.astype(np.int64)
            send_xyz.append(xyz_b[idx].reshape(-1, V * 3))
            send_gid.append(gid_b[idx].view(np.int64).reshape(-1, 1))
        got_xyz = self._all_to_all(send_xyz, np.float64, V * 3)
        got_gid = self._all_to_all(send_gid, np.int64, 1)
        ghost_xyz = np.concatenate(got_xyz).reshape(-1, V, 3) if got_xyz else np.zeros((0, V, 3))
        ghost_gid = np.concatenate(got_gid).reshape(-1).view(np.uint64) if got_gid else np.zeros(0, np.uint64)
        self.stats = {"patches_needed": int(sum(n.size for n in need)), "ghost_elements": int(ghost_xyz.shape[0])}
        # 4. exact pairs of the local A elements against the B elements gathered here
        return self.backend.pairs(xyz_a, gid_a, ghost_xyz, ghost_gid)
