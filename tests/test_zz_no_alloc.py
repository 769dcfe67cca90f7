"""The allocation-free radix sort (bvhg_radix_sort_noalloc) against the library's own sort.

bvhg_radix_sort_noalloc exists for callers that cannot allocate device memory (their pool allocator owns the
device, their step loop has a fixed memory budget, or they issue work during stream capture): it takes its scratch
from a fixed static device array instead. This checks, through the C ABI, that two calls in a row give exactly the
sorted keys and permutation that the regular build (bvhg_build, read back with bvhg_get_morton) gives for the same
elements, and that sizes beyond the array's capacity are refused. The file is named to run last.
"""
import ctypes

import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20


def reference_sort(ctx, xyz):
    """Morton keys of the elements (original order) and the library's sorted keys / permutation for them."""
    o = ctx.object()
    ctx.set_elements(o, xyz)
    ctx.build(o)
    keys_sorted, perm, _, _ = ctx.morton(o, xyz.shape[0])
    # unsorted keys: the oracle's keys, which the parity suite shows equal the library's bit for bit
    c = orc.centroids(xyz)
    mn, inv = orc.morton_bounds(orc.kdops(xyz, 18), 18)
    keys = orc.morton_keys(c, mn, inv)
    assert np.array_equal(keys[perm], keys_sorted)
    return keys, keys_sorted, perm


def noalloc_sort(torch, keys):
    n = keys.shape[0]
    d_in = torch.from_numpy(keys.view(np.int64)).cuda()
    d_out = torch.empty(n, dtype=torch.int64, device="cuda")
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = bvhg.lib.bvhg_radix_sort_noalloc(d_in.data_ptr(), d_out.data_ptr(), d_perm.data_ptr(), n, None)
    assert st == 0, f"status {st}"
    return d_out.cpu().numpy().view(np.uint64), d_perm.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_the_library_sort_twice():
    torch = pytest.importorskip("torch")
    a = meshes.random_soup(300000, 3, seed=201, size=0.002)
    b = meshes.random_soup(70001, 3, seed=202, size=0.004, stream=1)
    with bvhg.Context(k=18) as ctx:
        ka, sa, pa = reference_sort(ctx, a)
        kb, sb, pb = reference_sort(ctx, b)
    # first call: the larger object; second call: a smaller one reusing the same scratch
    out, perm = noalloc_sort(torch, ka)
    assert np.array_equal(out, sa) and np.array_equal(perm, pa)
    out, perm = noalloc_sort(torch, kb)
    assert np.array_equal(out, sb) and np.array_equal(perm, pb)


def test_noalloc_sort_refuses_more_than_its_capacity():
    torch = pytest.importorskip("torch")
    d = torch.zeros(2, dtype=torch.int64, device="cuda")
    p = torch.zeros(2, dtype=torch.int32, device="cuda")
    st = bvhg.lib.bvhg_radix_sort_noalloc(d.data_ptr(), d.data_ptr() + 8, p.data_ptr(), MAX_KEYS + 1, None)
    assert st == 1
    assert bvhg.lib.bvhg_radix_sort_noalloc(None, None, None, 0, None) == 0
