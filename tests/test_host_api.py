"""The C++ host mirror of collision_world / collision_object (distbvh_b200/host/bvhg/collision_world.hpp).

tests/host_api/collision_world_test.cpp drives it like the reference's collision_object test: two objects,
a narrowphase functor recording (patch, element) pairs, results read back with for_each_result. The CPU test
compiles it (warnings are errors); the GPU test runs it for several patch counts and k-DOPs and compares the
recorded element pairs with the oracle's exact pair set.
"""
import os
import subprocess

import numpy as np
import pytest

from distbvh_b200 import meshes
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host_api", "collision_world_test.cpp")
LIBDIR = os.path.join(ROOT, "distbvh_b200")


def compile_driver(out):
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(LIBDIR, "host"), SRC,
           "-L" + LIBDIR, "-lbvhg", "-Wl,-rpath," + LIBDIR, "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def write_elements(path, xyz):
    with open(path, "wb") as f:
        f.write(np.uint64(xyz.shape[0]).tobytes())
        f.write(np.ascontiguousarray(xyz, dtype=np.float64).tobytes())


def test_host_api_compiles(tmp_path):
    compile_driver(str(tmp_path / "cw"))
    assert os.path.exists(tmp_path / "cw")


@pytest.mark.gpu
@pytest.mark.parametrize("od,k", [(1, 26), (4, 18), (8, 6)])
def test_host_api_pairs_match_the_oracle(tmp_path, od, k):
    exe = str(tmp_path / "cw")
    compile_driver(exe)
    a = meshes.random_soup(6000, 3, seed=71, size=0.02)
    b = meshes.random_soup(5000, 3, seed=72, size=0.02, stream=1)
    write_elements(tmp_path / "a.bin", a)
    write_elements(tmp_path / "b.bin", b)
    out = subprocess.run([exe, str(tmp_path / "a.bin"), str(tmp_path / "b.bin"), str(od), str(k)], check=True,
                         capture_output=True, text=True).stdout.split("\n")
    head = out[0].split()
    count, calls = int(head[1]), int(head[3])
    body = [line for line in out[1:] if line.strip()]
    got = np.array([[int(x) for x in line.split()] for line in body if line[0].isdigit()],
                   dtype=np.int64).reshape(-1, 2)
    want = orc.pair_set(a, b, k).astype(np.int64)
    want[:, 1] += 1000000
    assert count == want.shape[0] > 0
    assert 1 <= calls <= od * od
    assert np.array_equal(got, want[np.lexsort((want[:, 1], want[:, 0]))])
    # local_patches: the oracle's Morton clustering, the union of its element slabs per patch, and the mean of its
    # element centroids summed in patch order; for_each_tree: one leaf per non-empty patch
    patches = [line.split()[1:] for line in body if line.startswith("patch")]
    order, bounds = orc.morton_cluster(a, k, od)
    slabs, cent = orc.kdops(a, k), orc.centroids(a)
    assert len(patches) == od
    for p, rec in enumerate(patches):
        gid, size = int(rec[0]), int(rec[1])
        vals = [float.fromhex(x) for x in rec[2:]]
        idx = order[int(bounds[p]):int(bounds[p + 1])].astype(np.int64)
        assert gid == p and size == idx.size
        if size == 0:
            continue
        box = np.empty((k // 2, 2))
        box[:, 0] = slabs[idx, :, 0].min(axis=0)
        box[:, 1] = slabs[idx, :, 1].max(axis=0)
        assert vals[:k] == box.reshape(-1).tolist()
        c = [0.0, 0.0, 0.0]
        for e in idx:
            for ax in range(3):
                c[ax] += float(cent[e, ax])
        assert vals[k:] == [x / size for x in c]
    tree = [line.split()[1:] for line in body if line.startswith("tree")]
    nonempty = int(np.count_nonzero(np.diff(bounds.astype(np.int64))))
    assert tree and int(tree[0][0]) == nonempty and int(tree[0][2]) == nonempty
    assert int(tree[0][1]) == 2 * nonempty - 1


@pytest.mark.gpu
@pytest.mark.parametrize("od", [1, 8, 64])
def test_host_api_empty_object(tmp_path, od):
    """An object without elements: od empty patches with the reference's default k-DOP and an empty tree."""
    exe = str(tmp_path / "cw")
    compile_driver(exe)
    out = subprocess.run([exe, "empty", str(od)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.split() == ["empty", "0"]
