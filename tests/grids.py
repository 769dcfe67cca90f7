"""Element fixtures restated from the reference's tests/TestCommon.hpp (same vertex order and arithmetic)."""
import numpy as np


def element_grid(nx, ny, nz, base_index=0, origin_shift=0.0):
    """buildElementGrid (tests/TestCommon.hpp:148-181): unit-cube grid of 8-vertex hexes, x fastest.
    Returns (xyz (n, 8, 3), gid (n,))."""
    dx, dy, dz = 1.0 / nx, 1.0 / ny, 1.0 / nz
    els = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                x = origin_shift + i * dx
                y = origin_shift + j * dy
                z = origin_shift + k * dz
                els.append([(x, y, z), (x + dx, y, z), (x + dx, y + dy, z), (x, y + dy, z),
                            (x, y, z + dz), (x + dx, y, z + dz), (x + dx, y + dy, z + dz), (x, y + dy, z + dz)])
    xyz = np.array(els, dtype=np.float64).reshape(-1, 8, 3)
    gid = np.arange(base_index, base_index + xyz.shape[0], dtype=np.uint64)
    return xyz, gid


def make_cube(center):
    """makeCube (tests/KDopTest.cpp:54-65): the 8 corners of a 2-wide cube around center."""
    c = np.asarray(center, dtype=np.float64)
    offs = [(1., 1., 1.), (-1., 1., 1.), (1., -1., 1.), (1., 1., -1.), (-1., -1., 1.), (-1., 1., -1.),
            (1., -1., -1.), (-1., -1., -1.)]
    return np.array([c + np.array(o) for o in offs]).reshape(1, 8, 3)


def clustered_soup(counts, seed, cells=None):
    """Tiny triangles in clusters of the given sizes, each inside one cell of the top 31 Morton bits (10 bits of
    x, 10 of y, 11 of z: the clusters sit at cell centres of a 1024 x 1024 x 2048 grid over the unit cube, 2e-4
    wide), plus two corner elements that fix the Morton bounds to the unit cube. Members of a cluster share the
    high key half and differ in the low. cells: the (ix, iy, iz) cell of each cluster (distinct), else a fixed
    diagonal of cells."""
    rng = np.random.default_rng(seed)
    parts = [np.array([[[0, 0, 0], [1e-3, 0, 0], [0, 1e-3, 0]]]),
             np.array([[[1, 1, 1], [1 - 1e-3, 1, 1], [1, 1 - 1e-3, 1]]])]
    for j, c in enumerate(counts):
        cell = np.array([307, 511 - 40 * j, 2 * (129 + 17 * j)]) if cells is None else np.asarray(cells[j])
        centre = (cell + 0.5) / np.array([1024.0, 1024.0, 2048.0])
        pts = centre + rng.uniform(-1e-4, 1e-4, (c, 1, 3)) + rng.uniform(-2e-6, 2e-6, (c, 3, 3))
        parts.append(pts)
    xyz = np.concatenate(parts).astype(np.float64)
    return np.ascontiguousarray(xyz[rng.permutation(xyz.shape[0])])


def distinct_cells(count, seed):
    rng = np.random.default_rng(seed)
    flat = rng.choice(1000 * 1000 * 2000, size=count, replace=False)
    return np.stack([flat % 1000 + 12, (flat // 1000) % 1000 + 12, flat // 1000000 + 24], axis=1)
