"""The identity behind the precision form's FP64 recheck, checked on the CPU.

The recheck decides strict overlap from projections that skip products by 0 and 1, form each product of a
coordinate by 1/sqrt(2) or 1/sqrt(3) once for every normal that uses it, and apply the epsilon shift once per slab
after the min / max over the vertices (kdop_math.cuh, project_group and group_overlap64). Those projections must
equal the reference's ((v0 * n0) + (v1 * n1)) + (v2 * n2) (src/bvh/kdop.hpp:223-227) in value: only the sign of a
zero may differ, which no comparison sees. numpy evaluates both in IEEE double with every product and sum rounded
separately, on the oracle's normal tables.
"""
import numpy as np
import pytest

from oracle import oracle as orc

R2 = 0.7071067811865475
R3 = 0.5773502691896258


def reference_projections(v, k):
    n = orc.normals(k)
    return (v[:, None, 0] * n[None, :, 0] + v[:, None, 1] * n[None, :, 1]) + v[:, None, 2] * n[None, :, 2]


def grouped_projections(v, k):
    """The recheck's projections, in the oracle's normal order: axes, then (26-DOP) corners, then edges."""
    v0, v1, v2 = v[:, 0], v[:, 1], v[:, 2]
    out = [v0, v1, v2]
    m0, m1, m2 = v0 * R2, v1 * R2, v2 * R2
    edges = [m0 + m1, m0 + m2, m1 + m2, m0 - m1, m0 - m2, m1 - m2]
    c0, c1, c2 = v0 * R3, v1 * R3, v2 * R3
    s, d = c0 + c1, c0 - c1
    corners = [s + c2, d + c2, s - c2, d - c2]
    if k == 18:
        out += edges
    if k == 26:
        out += corners + edges
    return np.stack(out, axis=1)


def samples(seed):
    rng = np.random.default_rng(seed)
    special = np.array([0.0, -0.0, 0.25, -0.25, 1.0, -1.0, 1e-300, -1e-300, 5e-324, 1e300, -1e300, 0.1, 3.0])
    yield special[rng.integers(0, len(special), size=(50000, 3))]
    yield rng.uniform(-1.0, 1.0, size=(50000, 3))
    yield rng.uniform(-1.0, 1.0, size=(50000, 3)) * 10.0 ** rng.integers(-12, 12, size=(50000, 1))


@pytest.mark.parametrize("k", [6, 18, 26])
def test_grouped_projections_equal_the_reference_in_value(k):
    for v in samples(10 + k):
        ref, grp = reference_projections(v, k), grouped_projections(v, k)
        assert ref.shape == grp.shape
        assert np.array_equal(ref, grp)  # == treats -0 and +0 as equal


@pytest.mark.parametrize("k", [6, 18, 26])
@pytest.mark.parametrize("eps", [0.0, 0.003, 0.25])
def test_epsilon_once_per_slab_gives_the_same_slabs_in_value(k, eps):
    """min over vertices of (p - eps) equals (min over vertices of p) - eps under round-to-nearest (monotone), and
    the same for max and + eps: the slabs of 4-vertex elements built both ways compare equal."""
    rng = np.random.default_rng(100 + k)
    v = rng.uniform(-1.0, 1.0, size=(20000, 4, 3)) * 10.0 ** rng.integers(-6, 6, size=(20000, 1, 1))
    p = reference_projections(v.reshape(-1, 3), k).reshape(20000, 4, -1)
    lo_ref, hi_ref = (p - eps).min(axis=1), (p + eps).max(axis=1)
    lo_once, hi_once = p.min(axis=1) - eps, p.max(axis=1) + eps
    assert np.array_equal(lo_ref, lo_once) and np.array_equal(hi_ref, hi_once)
    assert np.array_equal(lo_ref, orc.kdops(v, k, eps)[:, :, 0])
