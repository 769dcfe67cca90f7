"""Writes tests/golden/ref_vectors.npz: inputs and the reference's own outputs for them, computed by the
reference's headers through oracle/_ref (build it first with oracle/ref_build.sh; the reference sources are
needed only here, not by the tests that read the fixture).

Also the reference's Morton clustering of a 700-triangle soup into 1, 8 and 64 patches and its 1-bit radix sort of
3000 keys with duplicates.

Cases: seeded element soups of triangles, tetrahedra and hexahedra (two objects each) and two small plates in
the shape of the reference's two-plate contact case, each with inflation 0 and 0.003 (plates: 0.005). Stored per
case and object: vertices; k-DOP slabs for K = 6, 18, 26 (kdop_base::from_vertices; 18 through dop_18's
normals); centroids; Morton bounds and 64-bit codes (compute_bounds + morton); pair counts of
potential_collision_set over top-down trees of dop_26 and of dop_6; self_collision_set pairs of object a for
both; the 18-DOP pair set by brute force with the reference's overlap; the pairs and axis of sort_and_sweep_local
with max_variant_axis (narrowphase/kokkos.hpp) over dop_26 and dop_6 k-DOPs (soups only).

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from distbvh_b200 import meshes  # noqa: E402
from oracle import ref  # noqa: E402


def plates(nx, ny, seed):
    """Plate A at z = 0 on [0,1]^2 and plate B at z = 0.004 with per-vertex jitter of +-0.002 (seeded)."""
    rng = np.random.default_rng(seed)
    xs, ys = np.linspace(0, 1, nx + 1), np.linspace(0, 1, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")

    def tris(z):
        P = np.stack([X, Y, z], axis=-1)
        a, b, c, d = P[:-1, :-1], P[1:, :-1], P[1:, 1:], P[:-1, 1:]
        t1 = np.stack([a, b, c], axis=2).reshape(-1, 3, 3)
        t2 = np.stack([a, c, d], axis=2).reshape(-1, 3, 3)
        return np.ascontiguousarray(np.concatenate([t1, t2]))

    za = np.zeros_like(X)
    zb = 0.004 + rng.uniform(-0.002, 0.002, X.shape)
    return tris(za), tris(zb)


def cases():
    for V, na, nb, size in ((3, 150, 120, 0.08), (4, 110, 90, 0.09), (8, 70, 60, 0.12)):
        a = meshes.random_soup(na, V, seed=900 + V, size=size)
        b = meshes.random_soup(nb, V, seed=950 + V, size=size, stream=1)
        for eps in (0.0, 0.003):
            yield f"soup_v{V}_eps{eps}", a, b, eps
    a, b = plates(12, 6, seed=77)
    yield "plates_eps0.005", a, b, 0.005


def main():
    r26, r6 = ref.Ref(26), ref.Ref(6)
    out = {}
    names = []
    for name, a, b, eps in cases():
        names.append(name)
        out[f"{name}/a"], out[f"{name}/b"], out[f"{name}/eps"] = a, b, np.float64(eps)
        for side, x in (("a", a), ("b", b)):
            for k in (6, 18, 26):
                out[f"{name}/{side}/kdops{k}"] = r26.kdops(x, k, eps)
            out[f"{name}/{side}/centroids"] = r26.centroids(x)
            mn, inv, keys = r26.morton(x, eps)
            out[f"{name}/{side}/min3"], out[f"{name}/{side}/inv3"], out[f"{name}/{side}/keys"] = mn, inv, keys
        for tk, r in ((26, r26), (6, r6)):
            out[f"{name}/tree_count{tk}"] = np.int64(r.tree_pairs(a, b, eps)[0])
            out[f"{name}/self{tk}"] = r.self_pairs(a, eps)[1]
        out[f"{name}/pairs18"] = r26.brute_pairs18(a, b, eps)[1]
        if name.startswith("soup"):
            for tk, r in ((26, r26), (6, r6)):
                _, pairs, axis = r.sort_and_sweep(a, b, eps, -1)
                out[f"{name}/sweep{tk}/pairs"] = np.unique(pairs, axis=0)
                out[f"{name}/sweep{tk}/axis"] = np.int64(axis)
    out["cases"] = np.array(names)
    # Morton clustering into patches (morton_cluster) for the collision_world mirror, and the 1-bit radix sort
    cl = meshes.random_soup(700, 3, seed=4242, size=0.03)
    out["cluster/xyz"] = cl
    for od in (1, 8, 64):
        order, splits = r26.cluster(cl, od)
        out[f"cluster/od{od}/order"], out[f"cluster/od{od}/splits"] = order, splits
    rng = np.random.default_rng(99)
    keys = rng.integers(0, 1 << 63, 3000, dtype=np.uint64)
    keys[::7] = keys[3]  # duplicates
    out["radix/keys"] = keys
    out["radix/sorted"], out["radix/perm"] = r26.radix_sort_u64(keys)
    path = os.path.join(ROOT, "tests", "golden", "ref_vectors.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(names), "cases")


if __name__ == "__main__":
    main()
