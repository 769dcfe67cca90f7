"""Seeded synthetic element sets for the broadphase workloads (numpy, float64, element-major (n, V, 3)).

All randomness comes from a counter-based SplitMix64 stream, so any machine regenerates identical bytes for the
GPU path and the CPU oracle. The reference's own integration deck (NimbleSM sphere_plate_contact) is not
available; these generators stand in for it with the shapes and sizes of the benchmark configurations:

  two_plates        two 100x50-quad triangulated plates (10,000 triangles each), B offset in z and jittered
  sphere_plate      an icosphere (level 9: 5,242,880 triangles, radius 0.5) pressed 0.01 into a 2048x1024-quad
                    plate (4,194,304 triangles)
  tet_lattice       one jittered, log-normally scaled tetrahedron per cell of an m^3 lattice
  random_soup       small random triangles / tetrahedra / hexahedra in a box (parity tests)
"""
import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(seed, stream, n):
    """n doubles in [0, 1): the 53 high bits of SplitMix64(key + i), key derived from (seed, stream)."""
    key = _splitmix64(np.uint64(seed) ^ _splitmix64(np.uint64(stream)))
    with np.errstate(over="ignore"):
        ctr = key + np.arange(n, dtype=np.uint64)
    return (_splitmix64(ctr) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed, stream, n):
    """Standard normal deviates (Box-Muller over two uniform streams)."""
    u1 = uniform(seed, 2 * stream + 1, n)
    u2 = uniform(seed, 2 * stream + 2, n)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def plate(nx, ny, x0=0.0, x1=1.0, y0=0.0, y1=1.0, z=0.0, jitter=0.0, seed=0, stream=0):
    """Triangulated plate of nx*ny quads (2 triangles each), per-vertex z jitter U(-jitter, +jitter)."""
    i = np.arange(nx + 1, dtype=np.float64)
    j = np.arange(ny + 1, dtype=np.float64)
    X = x0 + (x1 - x0) * i / nx
    Y = y0 + (y1 - y0) * j / ny
    Z = np.full((ny + 1, nx + 1), z, dtype=np.float64)
    if jitter:
        Z = Z + (2.0 * uniform(seed, stream, (nx + 1) * (ny + 1)) - 1.0).reshape(ny + 1, nx + 1) * jitter
    V = np.empty((ny + 1, nx + 1, 3))
    V[..., 0] = X[None, :]
    V[..., 1] = Y[:, None]
    V[..., 2] = Z
    v00 = V[:-1, :-1].reshape(-1, 3)
    v10 = V[:-1, 1:].reshape(-1, 3)
    v11 = V[1:, 1:].reshape(-1, 3)
    v01 = V[1:, :-1].reshape(-1, 3)
    tris = np.empty((nx * ny, 2, 3, 3))
    tris[:, 0, 0], tris[:, 0, 1], tris[:, 0, 2] = v00, v10, v11
    tris[:, 1, 0], tris[:, 1, 1], tris[:, 1, 2] = v00, v11, v01
    return tris.reshape(-1, 3, 3)


def _icosahedron():
    p = (1.0 + np.sqrt(5.0)) / 2.0
    v = []
    for a in (-1.0, 1.0):
        for b in (-p, p):
            v += [(a, b, 0.0), (0.0, a, b), (b, 0.0, a)]
    v = np.array(v)
    d = np.linalg.norm(v[:, None, :] - v[None, :, :], axis=-1)
    edge = np.isclose(d, 2.0)
    faces = [(a, b, c) for a in range(12) for b in range(a + 1, 12) for c in range(b + 1, 12)
             if edge[a, b] and edge[b, c] and edge[a, c]]
    assert len(faces) == 20
    v = v / np.linalg.norm(v, axis=1, keepdims=True)
    return v[np.array(faces)]


def icosphere(level, radius=1.0, center=(0.0, 0.0, 0.0)):
    """Triangle soup of a level-`level` icosphere: 20 * 4**level triangles."""
    t = _icosahedron()
    for _ in range(level):
        a, b, c = t[:, 0], t[:, 1], t[:, 2]
        ab = a + b
        bc = b + c
        ca = c + a
        ab /= np.sqrt((ab * ab).sum(axis=1, keepdims=True))
        bc /= np.sqrt((bc * bc).sum(axis=1, keepdims=True))
        ca /= np.sqrt((ca * ca).sum(axis=1, keepdims=True))
        nt = np.empty((t.shape[0], 4, 3, 3))
        nt[:, 0, 0], nt[:, 0, 1], nt[:, 0, 2] = a, ab, ca
        nt[:, 1, 0], nt[:, 1, 1], nt[:, 1, 2] = ab, b, bc
        nt[:, 2, 0], nt[:, 2, 1], nt[:, 2, 2] = ca, bc, c
        nt[:, 3, 0], nt[:, 3, 1], nt[:, 3, 2] = ab, bc, ca
        t = nt.reshape(-1, 3, 3)
    return t * radius + np.asarray(center, dtype=np.float64)


def torus(nu, nv, major=0.5, minor=0.15):
    """Triangulated torus about the z axis: nu x nv quads (2 triangles each), centred at the origin."""
    u = np.linspace(0.0, 2.0 * np.pi, nu + 1)[:-1]
    v = np.linspace(0.0, 2.0 * np.pi, nv + 1)[:-1]
    U, Vv = np.meshgrid(u, v, indexing="ij")
    P = np.stack([(major + minor * np.cos(Vv)) * np.cos(U), (major + minor * np.cos(Vv)) * np.sin(U),
                  minor * np.sin(Vv)], axis=-1)
    P1 = np.roll(P, -1, axis=0)
    P2 = np.roll(P, -1, axis=1)
    P3 = np.roll(P1, -1, axis=1)
    t1 = np.stack([P, P1, P3], axis=2).reshape(-1, 3, 3)
    t2 = np.stack([P, P3, P2], axis=2).reshape(-1, 3, 3)
    return np.ascontiguousarray(np.concatenate([t1, t2]))


# --- the benchmark configurations ---------------------------------------------------------------------------

TWO_PLATES_EPSILON = 0.005  # plate A is flat at z = 0 and B sits at z >= 0.002: without inflation S is empty


def two_plates(seed=1):
    """Two 100x50-quad plates: A at z = 0 on [0,1]^2, B at z = 0.004 with per-vertex U(+-0.002) jitter."""
    a = plate(100, 50, z=0.0)
    b = plate(100, 50, z=0.004, jitter=0.002, seed=seed, stream=1)
    return a, b


SPHERE_PLATE_RADIUS = 0.5
SPHERE_PLATE_PENETRATION = 0.01


def sphere_plate(level=9, nx=2048, ny=1024):
    """Icosphere (radius 0.5) centred at z = 0.5 - 0.01 over a plate at z = 0 on [-1,1]x[-0.5,0.5]."""
    sphere = icosphere(level, SPHERE_PLATE_RADIUS, (0.0, 0.0, SPHERE_PLATE_RADIUS - SPHERE_PLATE_PENETRATION))
    pl = plate(nx, ny, -1.0, 1.0, -0.5, 0.5, 0.0)
    return sphere, pl


def tet_lattice(m, seed=3, jitter=0.3, sigma=0.4):
    """One tetrahedron per cell of an m^3 lattice (cell size 1/m): corners (0,0,0), (1,0,0), (0,1,0), (0,0,1) of
    the cell, each vertex jittered U(+-jitter cells), then scaled about its centroid by LogNormal(0, sigma)."""
    h = 1.0 / m
    idx = np.arange(m ** 3, dtype=np.int64)
    i = idx % m
    j = (idx // m) % m
    k = idx // (m * m)
    base = np.stack([i, j, k], axis=1).astype(np.float64) * h
    corners = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64) * h
    t = base[:, None, :] + corners[None, :, :]
    t = t + (2.0 * uniform(seed, 1, t.size).reshape(t.shape) - 1.0) * (jitter * h)
    c = t.mean(axis=1, keepdims=True)
    s = np.exp(sigma * normal(seed, 2, m ** 3))[:, None, None]
    return c + (t - c) * s


def batch_scenes(nscenes=512, lo=1000, hi=200000, seed=11):
    """Two-body scenes for the batching form: per-scene element counts LogUniform[lo, hi] (split between the two
    bodies), element centroids uniform in the body's unit cube, triangle size 1.5 n^(-1/3), and a random rigid
    offset of each body (up to half a cube) so that scenes have uneven overlap. Returns [(a, b), ...].

    The counts are a stratified LogUniform sample (scene s draws its log-count from its own 1/nscenes quantile
    band, in shuffled order), so the batch's total is the distribution's mean times nscenes (19.2M triangles for
    512 scenes over [1k, 200k]) rather than whatever one independent draw gives."""
    rng = np.random.default_rng(seed)
    u = (np.arange(nscenes) + rng.uniform(0.0, 1.0, nscenes)) / nscenes
    rng.shuffle(u)
    counts = np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo))).astype(np.int64)
    out = []
    for s in range(nscenes):
        n = int(counts[s])
        na = max(1, n // 2)
        nb = max(1, n - na)
        size = 0.75 * n ** (-1.0 / 3.0)  # vertices within +-size of the centroid: edge about 1.5 n^(-1/3)
        a = random_soup(na, 3, seed=seed * 100003 + 2 * s, size=size)
        b = random_soup(nb, 3, seed=seed * 100003 + 2 * s + 1, size=size, stream=1)
        b = b + rng.uniform(-0.5, 0.5, 3)
        out.append((a, b))
    return out


def checkerboard(m):
    """Object membership of the tet_lattice cells: True for (i + j + k) even (object A), False for odd (B)."""
    idx = np.arange(m ** 3, dtype=np.int64)
    return ((idx % m + (idx // m) % m + idx // (m * m)) & 1) == 0


def random_soup(n, V=3, seed=0, box=1.0, size=0.05, stream=0):
    """n random elements of V vertices: centre U(0, box)^3, each vertex within +-size of the centre."""
    c = uniform(seed, 3 * stream + 1, 3 * n).reshape(n, 1, 3) * box
    off = (2.0 * uniform(seed, 3 * stream + 2, 3 * n * V).reshape(n, V, 3) - 1.0) * size
    return c + off
