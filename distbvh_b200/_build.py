"""Build recipe for libbvhg.so (the sm_100a CUDA library behind include/bvhg.h).

The library is compiled in-tree with nvcc for sm_100a only; the shared object lands next to this file so it is
loaded from the package directory (never from a JIT cache or site-packages).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbvhg.so")
SOURCES = ["bvhg_api.cu", "k_element.cu", "k_sort.cu", "k_tree.cu", "k_traverse.cu", "k_sweep.cu", "k_cluster.cu", "k_noalloc.cu"]
HEADERS = ["bvhg_internal.cuh", "kdop_math.cuh", "bulk_copy.cuh", os.path.join("..", "..", "include", "bvhg.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    # FP64 slabs must round every product and sum separately (kdop.hpp:223-227 as written); the kernels use
    # __dmul_rn/__dadd_rn explicitly, and contraction is disabled as a second guard.
    "-fmad=false",
]
LINK_GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, h) for h in HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    """Compile every .cu to an object and link libbvhg.so (in parallel, one nvcc per source)."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    errors = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errors.append(f"{src}:\n{out.decode(errors='replace')}")
        elif verbose and out:
            print(out.decode(errors="replace"), file=sys.stderr)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *LINK_GENCODE, "-shared", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC", "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
