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
