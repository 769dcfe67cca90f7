"""The allocation-free radix sort (bvhg_radix_sort_noalloc) against the oracle's stable sort.

bvhg_radix_sort_noalloc exists for callers that cannot allocate device memory: their pool allocator owns the
device (a cudaMalloc beside it fails or fragments the pool), their step loop runs under a fixed device-memory
budget, or a library boundary forbids the callee from owning device memory. It takes its scratch from a fixed
static device array instead. Through the C ABI, this checks:
  - two calls in a row give exactly the oracle's stable order (sorted keys and permutation), and agree with the
    library's regular sort (bvhg_build, read back with bvhg_get_morton) on the same Morton keys;
  - the full capacity (1,048,576 keys) with keys that use all 64 bits;
  - keys that start 8 bytes past a 16-byte boundary (the radix pass then reads tiles with plain loads);
  - a call after a warm-up call leaves the device's free memory unchanged;
  - sizes beyond the array's capacity are refused.
The file is named to run last.
"""
import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20


def morton_keys_of(xyz):
    c = orc.centroids(xyz)
    mn, inv = orc.morton_bounds(orc.kdops(xyz, 18), 18)
    return orc.morton_keys(c, mn, inv)


def library_sort(ctx, xyz):
    """The regular build's sorted keys and permutation for these elements."""
    o = ctx.object()
    ctx.set_elements(o, xyz)
    ctx.build(o)
    keys_sorted, perm, _, _ = ctx.morton(o, xyz.shape[0])
    return keys_sorted, perm


def noalloc_sort(torch, keys, offset_words=0):
    """Sorts `keys` with the allocation-free entry point; the input starts offset_words 8-byte words into its
    device buffer."""
    n = keys.shape[0]
    buf = torch.zeros(n + offset_words, dtype=torch.int64, device="cuda")
    buf[offset_words:] = torch.from_numpy(keys.view(np.int64)).cuda()
    d_out = torch.empty(n, dtype=torch.int64, device="cuda")
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = bvhg.lib.bvhg_radix_sort_noalloc(buf.data_ptr() + 8 * offset_words, d_out.data_ptr(), d_perm.data_ptr(),
                                          n, None)
    assert st == 0, f"status {st}"
    return d_out.cpu().numpy().view(np.uint64), d_perm.cpu().numpy().view(np.uint32)


def check(keys, out, perm):
    want = orc.stable_perm(keys)
    assert np.array_equal(perm, want), "permutation differs from the stable order"
    assert np.array_equal(out, keys[want]), "sorted keys differ"


def test_noalloc_sort_matches_the_oracle_twice():
    torch = pytest.importorskip("torch")
    a = meshes.random_soup(300000, 3, seed=201, size=0.002)
    b = meshes.random_soup(70001, 3, seed=202, size=0.004, stream=1)
    ka, kb = morton_keys_of(a), morton_keys_of(b)
    # first call: the larger object; second call: a smaller one reusing the same scratch
    out_a, perm_a = noalloc_sort(torch, ka)
    check(ka, out_a, perm_a)
    out_b, perm_b = noalloc_sort(torch, kb)
    check(kb, out_b, perm_b)
    with bvhg.Context(k=18) as ctx:
        for xyz, out, perm in ((a, out_a, perm_a), (b, out_b, perm_b)):
            lk, lp = library_sort(ctx, xyz)
            assert np.array_equal(lk, out) and np.array_equal(lp, perm)


def test_noalloc_sort_full_capacity_full_width_keys():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(203)
    keys = rng.integers(0, np.iinfo(np.uint64).max, size=MAX_KEYS, dtype=np.uint64, endpoint=True)
    keys[:1000] = keys[5000]  # ties, kept in input order
    keys[1000] = np.uint64(0xFFFFFFFFFFFFFFFF)
    keys[1001] = np.uint64(0)
    out, perm = noalloc_sort(torch, keys)
    check(keys, out, perm)
    assert np.array_equal(perm, np.argsort(keys, kind="stable").astype(np.uint32))


def test_noalloc_sort_unaligned_input():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(204)
    keys = rng.integers(0, 1 << 40, size=100003, dtype=np.uint64)
    out, perm = noalloc_sort(torch, keys, offset_words=1)
    check(keys, out, perm)


def test_noalloc_sort_allocates_nothing():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(205)
    keys = rng.integers(0, 1 << 62, size=500000, dtype=np.uint64)
    n = keys.shape[0]
    d_in = torch.from_numpy(keys.view(np.int64)).cuda()
    d_out = torch.empty(n, dtype=torch.int64, device="cuda")
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    # the warm-up call loads the module and resolves the scratch array's address
    assert bvhg.lib.bvhg_radix_sort_noalloc(d_in.data_ptr(), d_out.data_ptr(), d_perm.data_ptr(), n, None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert bvhg.lib.bvhg_radix_sort_noalloc(d_in.data_ptr(), d_out.data_ptr(), d_perm.data_ptr(), n, None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    check(keys, d_out.cpu().numpy().view(np.uint64), d_perm.cpu().numpy().view(np.uint32))


def test_noalloc_sort_refuses_more_than_its_capacity():
    torch = pytest.importorskip("torch")
    d = torch.zeros(2, dtype=torch.int64, device="cuda")
    p = torch.zeros(2, dtype=torch.int32, device="cuda")
    st = bvhg.lib.bvhg_radix_sort_noalloc(d.data_ptr(), d.data_ptr() + 8, p.data_ptr(), MAX_KEYS + 1, None)
    assert st == 1
    assert bvhg.lib.bvhg_radix_sort_noalloc(None, None, None, 0, None) == 0
