"""GPU pair sets at the benchmark's sizes against the oracle.

The oracle's OpenMP pipeline (from_vertices, compute_bounds, morton, the one-bit stable radix sort, the top-down
tree and the tree-vs-tree query, all restated on the CPU) runs on the same seeded scenes the benchmark times, and
its pair list must equal the CUDA path's exactly, in the FP64 plain form and in the FP32 filter form after its
FP64 recheck:
  - the sphere-plate scene: icosphere L9 (5,242,880 triangles) pressed 0.01 into a 2048 x 1024-quad plate
    (4,194,304 triangles), 18-DOP, and the same scene at a quarter of the size;
  - the precision case's tet lattice at 128^3 (2,097,152 tets, checkerboard objects) for 26-DOP and 18-DOP.
At these sizes the Morton permutation is also checked against the oracle's stable sort of the oracle's keys.
"""
import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def gpu_pairs(a, b, k, precision):
    """Pair sets of two builds: the first traversal computes the element slabs it tests; when it finds the contact
    dense, the second build stores every element's slabs and the second traversal reads them."""
    with bvhg.Context(k=k, precision=precision) as ctx:
        oa, ob = ctx.object(), ctx.object()
        ctx.set_elements(oa, a)
        ctx.set_elements(ob, b)
        ctx.build(oa)
        ctx.build(ob)
        first = orc.canonical(ctx.broadphase(oa, ob))
        ctx.build(oa)
        ctx.build(ob)
        second = orc.canonical(ctx.broadphase(oa, ob))
        _, perm, mn, inv = ctx.morton(oa, a.shape[0])
    return (first, second), perm, mn, inv


def check_scene(a, b, k):
    cnt, _, want = orc.pipeline(a, b, k, keep_pairs=True)
    assert cnt > 0
    okeys = orc.morton_keys(orc.centroids(a), *orc.morton_bounds(orc.kdops(a, k), k))
    operm = orc.stable_perm(okeys)
    for precision in (bvhg.PLAIN_FP64, bvhg.FILTER_FP32):
        sets, perm, _, _ = gpu_pairs(a, b, k, precision)
        for which, got in zip(("first", "second"), sets):
            assert got.shape == want.shape, f"precision {precision}, {which} build: {got.shape[0]} pairs, " \
                                            f"oracle {want.shape[0]}"
            assert np.array_equal(got, want), f"precision {precision}, {which} build: pair set differs"
        assert np.array_equal(perm, operm), f"precision {precision}: Morton permutation differs"


@pytest.mark.parametrize("level,nx,ny", [(8, 1024, 512), (9, 2048, 1024)])
def test_sphere_plate_scene_against_the_oracle(level, nx, ny):
    s, p = meshes.sphere_plate(level, nx, ny)
    check_scene(s, p, 18)


@pytest.mark.parametrize("k", [26, 18])
def test_tet_lattice_against_the_oracle(k):
    m = 128
    xyz = meshes.tet_lattice(m)
    even = meshes.checkerboard(m)
    a, b = np.ascontiguousarray(xyz[even]), np.ascontiguousarray(xyz[~even])
    check_scene(a, b, k)
