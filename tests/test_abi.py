"""The C ABI library loads and exports every symbol include/bvhg.h declares; host-side tables match the oracle.

No kernel runs here (no GPU on the build machine).
"""
import ctypes
import os
import re

import numpy as np
import pytest

import distbvh_b200 as bvhg
from distbvh_b200 import meshes
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "bvhg.h")).read()
    return sorted(set(re.findall(r"BVHG_API\s+[\w\s\*]+?\b(bvhg_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    lib = ctypes.CDLL(bvhg.LIB_PATH)
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(bvhg.EXPORTS) == names


def test_build_recipe_targets_sm100a_only():
    # every nvcc invocation of the recipe (compile and link) names one target, sm_100a, and no other
    from distbvh_b200 import _build
    flags = list(_build.NVCC_FLAGS)
    gencodes = [flags[i + 1] for i, f in enumerate(flags) if f == "-gencode"]
    assert gencodes == ["arch=compute_100a,code=sm_100a"]
    assert not any(f.startswith(("-arch", "--gpu-architecture", "--generate-code")) for f in flags)
    assert _build.LINK_GENCODE == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_package_import_does_not_load_the_library():
    # the mesh generators (used by the CPU reference arm) import without mapping libbvhg.so
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); from distbvh_b200 import meshes; "
            "print(any('libbvhg' in l for l in open('/proc/self/maps')))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout.strip()
    assert out == "False"


@pytest.mark.parametrize("k", [6, 18, 26])
def test_device_normal_table_matches_oracle(k):
    ref = orc.normals(k)
    for a in range(k // 2):
        for c in range(3):
            v, lo, hi = bvhg.debug_normal(k, a, c)
            assert v == ref[a, c]
            assert np.float64(lo) <= v <= np.float64(hi)
            # tight: adjacent floats (or equal when exact)
            assert hi == lo or np.nextafter(np.float32(lo), np.float32(np.inf)) == np.float32(hi)


def test_debug_normal_rejects_bad_index():
    with pytest.raises(bvhg.BvhgError):
        bvhg.debug_normal(18, 9, 0)
    with pytest.raises(bvhg.BvhgError):
        bvhg.debug_normal(12, 0, 0)


def test_status_strings():
    for code in range(7):
        assert bvhg.lib.bvhg_status_string(code)
    assert bvhg.lib.bvhg_status_string(99) == b"unknown status"


def test_create_rejects_bad_config():
    for kwargs in ({"k": 12}, {"digit_bits": 3}, {"precision": 5}, {"epsilon": -1.0}):
        with pytest.raises(bvhg.BvhgError):
            bvhg.Context(**kwargs)


def test_synthetic_streams_are_stable():
    # The generators must give identical bytes on every machine (GPU box and CPU container).
    u = meshes.uniform(7, 3, 4)
    assert np.array_equal(u, meshes.uniform(7, 3, 4))
    assert 0.0 <= u.min() and u.max() < 1.0
    assert abs(meshes.uniform(1, 0, 100000).mean() - 0.5) < 0.01
    a, b = meshes.two_plates()
    assert a.shape == (10000, 3, 3) and b.shape == (10000, 3, 3)
    assert a[:, :, 2].max() == 0.0 and b[:, :, 2].min() >= 0.002 and b[:, :, 2].max() <= 0.006
    s = meshes.icosphere(2)
    assert s.shape == (320, 3, 3)
    assert np.allclose(np.linalg.norm(s, axis=2), 1.0)
    t = meshes.tet_lattice(4)
    assert t.shape == (64, 4, 3)
