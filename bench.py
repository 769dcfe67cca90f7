#!/usr/bin/env python3
"""Benchmark: build + broadphase Mprims/s of the per-rank element broadphase on B200.

Workload (one step): an icosphere of 5,242,880 triangles (level 9, radius 0.5) pressed 0.01 into a plate of
4,194,304 triangles (2048 x 1024 quads), 18-DOP, epsilon 0, inter-object pairs: centroids and Morton bounds,
Morton keys, stable radix sort (8-bit digits over the high key half + low-half fix-up), element slabs, LBVH build
with node k-DOPs of both objects, traversal, exact pair set.
Synthetic seeded geometry (the reference's sphere/plate deck is not available); inputs 680 MB, larger than L2.

  value  device-resident vertices -> device-resident pair set, FP64 plain form, CUDA events on the library's
         stream, max over ranks; whole-job Mprims/s = (elements of both objects) * ranks / time.
  e2e    the same step through the C ABI with pinned HOST buffers: H2D of both vertex arrays and D2H of the
         pair list inside the timed region.

`--impl reference` times the reference's algorithms on the host cores instead (see run_reference()).
Under torchrun every rank runs its own copy of the scene (independent objects, no collective on the data path:
weak scaling); timing is max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# The batching form runs its scenes as parallel branches of one CUDA graph: let the device take up to 32 of them at a
# time (the default is 8 hardware work queues). Must be set before the process creates its CUDA context.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "build+broadphase Mprims/s, FP32-filter vs FP64 plain on B200, same exact pair set"
K = 18
EPS = 0.0


def workload_name(args):
    tris = 20 * 4 ** args.level
    return (f"sphere_plate: icosphere L{args.level} ({tris:,} tris, r=0.5, penetration 0.01) + plate "
            f"{args.nx}x{args.ny} quads ({2 * args.nx * args.ny:,} tris)")


def bench_config(args, world, elements, pairs):
    """The config object of both arms' lines (the same keys and values for the same workload)."""
    return {"workload": workload_name(args), "k": K, "epsilon": EPS, "elements": int(elements), "pairs": int(pairs),
            "form": "plain FP64", "l2": "inputs 680 MB > L2 (126 MB)",
            "parallelism": f"independent scene per rank x{world}"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="bvhg", choices=["bvhg", "reference"])
    p.add_argument("--level", type=int, default=9, help="icosphere level (9 = the benchmark configuration)")
    p.add_argument("--nx", type=int, default=2048)
    p.add_argument("--ny", type=int, default=1024)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--workload", default="sphere_plate",
                   choices=["sphere_plate", "tet_lattice", "batch", "timestep", "sweep"],
                   help="tet_lattice: the precision-form case (26-DOP, FP32 filter vs FP64 plain); batch: 512 "
                        "two-body scenes in one graph; timestep: 32 tumbling tori, refit vs rebuild; sweep: "
                        "sort-and-sweep between two patch-sized objects")
    p.add_argument("--lattice", type=int, default=256, help="tet_lattice cells per axis (256 = 16,777,216 tets)")
    p.add_argument("--kdop", type=int, default=26, choices=[6, 18, 26], help="tet_lattice k-DOP (26 = the precision case)")
    p.add_argument("--no-oracle", action="store_true", help="skip the full-size oracle pair-set check")
    p.add_argument("--batch-form", default=None, metavar="GROUPS,LANES",
                   help="batch: run this form (groups 0 = per-object launches) instead of the autotuner's choice")
    return p.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "bvhg":
        import torch.distributed as dist
        backend = "nccl" if args.impl == "bvhg" else "gloo"
        import datetime
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Algorithmic DRAM bytes per element of each stage for triangles (V = 3) with D = K/2 slabs of S bytes and leaf
# buckets of 8 elements:
#   bounds   read 72 (vertices) + write 24 (centroid, SoA)                                      = 96
#   keys     read 24 (centroid) + write 8 (key)                                                 = 32
#   sort     per pass read 12 + write 12 (key + index)                                          = 24 per pass
#   fixup    read 12 + write 12 (key + index; neighbours of a run are cache hits)               = 24
#   slabs    read 4 (index) + 72 (vertices, gathered) + write 2 D S / 8 (leaf-bucket boxes) + 2 D S / 32
#            (query-group boxes); element slabs are not stored (the traversal caches the ones it tests)
#                                                                                               = 76 + 2DS(1/8 + 1/32)
#   build    read 2 D S / 8 (bucket boxes) + 2 (boundary keys) + write (4 D S + 8 child + 8 range + 8 parent) / 8
#            (one internal node per bucket)                                                     = 2 + 2DS/8 + (4DS + 24)/8
#   traverse read 2 D S / 32 (query-group box) per query; survivors read their slabs and the tree
LEAF = 8


# Refit (k_refit, one thread per bucket climbing the stored parent links): read the bucket box 2 D S + parent 4;
# per internal node (one per bucket) write both children's sides 4 D S, read the sibling's side 2 D S, exchange and
# parent words 8; per element (buckets of 8):                                                  = (8DS + 12) / 8
def refit_bytes(D, S):
    return (8 * D * S + 12) / LEAF


def stage_bytes(D, S, passes):
    return {"bounds": 96, "keys": 32, "sort": 24 * passes, "fixup": 24,
            "slabs": 76 + 2 * D * S * (1 / LEAF + 1 / 32),
            "build": 2 + 2 * D * S / LEAF + (4 * D * S + 24) / LEAF,
            "traverse": 2 * D * S / 32}


def run_gpu(args, world, rank, local):
    import torch
    import distbvh_b200 as bvhg
    from distbvh_b200 import meshes

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sphere, plate = meshes.sphere_plate(args.level, args.nx, args.ny)
    na, nb = sphere.shape[0], plate.shape[0]
    prims = na + nb
    stream = torch.cuda.Stream(device=dev)
    d_a = torch.from_numpy(sphere).to(dev)
    d_b = torch.from_numpy(plate).to(dev)
    h_a = torch.from_numpy(sphere).pin_memory()
    h_b = torch.from_numpy(plate).pin_memory()
    torch.cuda.synchronize()

    def make_ctx(precision, timing=False):
        ctx = bvhg.Context(k=K, precision=precision, epsilon=EPS, device=local, stream=stream.cuda_stream,
                           stage_timing=timing)
        oa, ob = ctx.object(), ctx.object()
        return ctx, oa, ob

    cap = 1 << 22
    d_out = torch.empty((cap, 2), dtype=torch.int64, device=dev)
    h_out = torch.empty((cap, 2), dtype=torch.int64).pin_memory()

    def step_device(ctx, oa, ob):
        ctx.set_elements(oa, d_a, mem=bvhg.MEM_DEVICE)
        ctx.set_elements(ob, d_b, mem=bvhg.MEM_DEVICE)
        ctx.build(oa)
        ctx.build(ob)
        st, cnt = ctx.broadphase_raw(oa, ob, d_out.data_ptr(), cap, bvhg.MEM_DEVICE)
        if st != 0:
            raise RuntimeError(f"broadphase status {st}")
        return cnt

    def step_host(ctx, oa, ob):
        # the sphere's build runs on its own stream while the plate's vertices cross PCIe on the context stream
        ctx.set_elements(oa, h_a.numpy(), mem=bvhg.MEM_HOST)
        ctx.build(oa)
        ctx.set_elements(ob, h_b.numpy(), mem=bvhg.MEM_HOST)
        ctx.build(ob)
        st, cnt = ctx.broadphase_raw(oa, ob, h_out.data_ptr(), cap, bvhg.MEM_HOST)
        if st != 0:
            raise RuntimeError(f"broadphase status {st}")
        return cnt

    def timed(fn, ctx, oa, ob, steps, warmup, clocks=None):
        if clocks:
            clocks.__enter__()
            time.sleep(0.5)  # nvidia-smi takes a moment to emit its first sample
        for _ in range(warmup):
            fn(ctx, oa, ob)
        torch.cuda.synchronize(dev)
        barrier(world)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        launches0 = ctx.launch_count()
        e0.record(stream)
        cnt = 0
        for _ in range(steps):
            cnt = fn(ctx, oa, ob)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if clocks:
            clocks.__exit__(None, None, None)
        barrier(world)
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms, world, dev), cnt, (ctx.launch_count() - launches0) // steps

    # FP64 plain form, device-resident (the headline value)
    ctx64, a64, b64 = make_ctx(bvhg.PLAIN_FP64)
    clocks = ClockSampler(local)
    ms64, pairs64, launches = timed(step_device, ctx64, a64, b64, args.steps, args.warmup, clocks)
    # FP32 filter form, same workload
    ctx32, a32, b32 = make_ctx(bvhg.FILTER_FP32)
    ms32, pairs32, _ = timed(step_device, ctx32, a32, b32, args.steps, args.warmup)
    cand32 = ctx32.last_candidates()
    # identical exact pair sets (checked as sorted sets once, outside the timed regions)
    same = False
    p64 = None
    if rank == 0:
        step_device(ctx64, a64, b64)
        p64 = d_out[:pairs64].cpu().numpy().copy()
        step_device(ctx32, a32, b32)
        p32 = d_out[:pairs32].cpu().numpy().copy()
        same = pairs64 == pairs32 and np.array_equal(
            p64[np.lexsort((p64[:, 1], p64[:, 0]))], p32[np.lexsort((p32[:, 1], p32[:, 0]))])

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        ms_e2e, pe2e, _ = timed(step_host, ctx64, a64, b64, max(2, args.steps // 2), 2)
        e2e = {"value": prims * world / (ms_e2e * 1e-3) / 1e6, "unit": "Mprims/s", "ms_per_step": ms_e2e,
               "h2d_bytes_per_step": int(sphere.nbytes + plate.nbytes), "d2h_bytes_per_step": int(pe2e * 16 + 24)}

    # per-stage times (library CUDA events on the launching stream) for the roofline of the dominant kernel
    ctxt, at, bt = make_ctx(bvhg.PLAIN_FP64, timing=True)
    step_device(ctxt, at, bt)
    ctxt.stage_times()
    reps = max(3, args.steps // 2)
    for _ in range(reps):
        step_device(ctxt, at, bt)
    st_ms, st_launch = ctxt.stage_times()
    st_ms = {k: v / reps for k, v in st_ms.items()}
    st_launch = {k: v // reps for k, v in st_launch.items()}
    # refit (same topology, vertices re-read): element slabs, then the bottom-up refit of every internal node
    for _ in range(reps):
        ctxt.build(at, bvhg.REFIT)
        ctxt.build(bt, bvhg.REFIT)
    rf_ms, _ = ctxt.stage_times()
    rf_ms = {k: v / reps for k, v in rf_ms.items() if v > 0}
    passes = st_launch["sort"] // 2
    per_elem = stage_bytes(K // 2, 8, passes)
    stage_bw = {}
    for s, b in per_elem.items():
        if st_ms.get(s, 0) > 0:
            elems = prims if s != "traverse" else na
            stage_bw[s] = elems * b / (st_ms[s] * 1e-3) / 1e9
    dom = max(("bounds", "keys", "sort", "fixup", "slabs", "build"), key=lambda s: st_ms[s])
    peak, peak_kind = peaks()
    n_launch = max(1, st_launch[dom])
    per_launch_ms = st_ms[dom] / n_launch
    per_launch_bytes = prims * per_elem[dom] / n_launch
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        if dom in tj.get("bytes_per_element", {}):
            traffic = tj["bytes_per_element"][dom] * prims / n_launch
    roofline = {"bound": "hbm", "kernel": dom, "achieved": per_launch_bytes / (per_launch_ms * 1e-3) / 1e9,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "traffic": traffic, "algorithmic_bytes_per_launch": per_launch_bytes,
                "launch_ms": per_launch_ms}
    roofline["frac"] = roofline["achieved"] / peak

    result = {
        "metric": METRIC, "value": prims * world / (ms64 * 1e-3) / 1e6, "unit": "Mprims/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded icosphere + plate)",
        "config": bench_config(args, world, prims, pairs64),
        "sort_digit_bits": 8,
        "filter_fp32": {"ms_per_step": ms32, "value": prims * world / (ms32 * 1e-3) / 1e6, "pairs": int(pairs32),
                        "candidates": int(cand32), "same_pair_set": bool(same),
                        "speedup_vs_fp64": ms64 / ms32,
                        "false_positive_rate": (cand32 - pairs32) / cand32 if cand32 else 0.0},
        "stages_ms": st_ms, "stage_gbs": stage_bw,
        "refit": {"ms": sum(rf_ms.values()), "stages_ms": rf_ms,
                  "slabs_gbs": prims * per_elem["slabs"] / (rf_ms.get("slabs", float("inf")) * 1e-3) / 1e9,
                  "refit_gbs": prims * refit_bytes(K // 2, 8) / (rf_ms.get("build", float("inf")) * 1e-3) / 1e9},
        "roofline": roofline,
        "gpu_launches": int(launches),
        "e2e": e2e,
        "clocks": clocks.summary(),
    }
    ctx64.close()
    ctx32.close()
    ctxt.close()
    return result, sphere, plate, p64


def run_precision(args, world, rank, local):
    """Precision-form case: one tetrahedron per cell of a jittered lattice^3 (vertex jitter +-0.3 cell, scale
    LogNormal(0, 0.4)), split as a checkerboard into objects A ((i+j+k) even) and B (odd), 26-DOP, inter-object
    pairs. FP64 plain and FP32 filter + FP64 recheck, device-resident; the two pair sets compared on the device;
    the FP32 slab enclosure error against the FP64 slabs over all of object A."""
    import torch
    import distbvh_b200 as bvhg
    from distbvh_b200 import meshes

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    m = args.lattice
    xyz = meshes.tet_lattice(m)
    even = meshes.checkerboard(m)
    a_np, b_np = np.ascontiguousarray(xyz[even]), np.ascontiguousarray(xyz[~even])
    del xyz
    d_a, d_b = torch.from_numpy(a_np).to(dev), torch.from_numpy(b_np).to(dev)
    prims = a_np.shape[0] + b_np.shape[0]
    stream = torch.cuda.Stream(device=dev)
    k = args.kdop

    def run(precision):
        ctx = bvhg.Context(k=k, precision=precision, device=local, stream=stream.cuda_stream)
        oa, ob = ctx.object(), ctx.object()

        def step(cap, out):
            ctx.set_elements(oa, d_a, mem=bvhg.MEM_DEVICE)
            ctx.set_elements(ob, d_b, mem=bvhg.MEM_DEVICE)
            ctx.build(oa)
            ctx.build(ob)
            return ctx.broadphase_raw(oa, ob, out.data_ptr() if out is not None else None, cap, bvhg.MEM_DEVICE)

        st, cnt = step(0, None)  # count only
        out = torch.empty((max(cnt, 1), 2), dtype=torch.int64, device=dev)
        for _ in range(args.warmup):
            st, cnt = step(out.shape[0], out)
            assert st == 0, st
        torch.cuda.synchronize(dev)
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            st, cnt = step(out.shape[0], out)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
        cand = ctx.last_candidates() if precision == bvhg.FILTER_FP32 else cnt
        return ctx, oa, ms, cnt, cand, out[:cnt]

    def stage_ms(precision, reps=2):
        """Per-stage device times of one step (library CUDA events around each stage, stream-serialised)."""
        ctx = bvhg.Context(k=k, precision=precision, device=local, stream=stream.cuda_stream, stage_timing=True)
        oa, ob = ctx.object(), ctx.object()

        def step(cap, out):
            ctx.set_elements(oa, d_a, mem=bvhg.MEM_DEVICE)
            ctx.set_elements(ob, d_b, mem=bvhg.MEM_DEVICE)
            ctx.build(oa)
            ctx.build(ob)
            return ctx.broadphase_raw(oa, ob, out.data_ptr() if out is not None else None, cap, bvhg.MEM_DEVICE)

        _, cnt = step(0, None)
        out = torch.empty((max(cnt, 1), 2), dtype=torch.int64, device=dev)
        step(out.shape[0], out)
        ctx.stage_times()
        for _ in range(reps):
            step(out.shape[0], out)
        ms, _ = ctx.stage_times()
        ctx.close()
        del out
        return {s_: v / reps for s_, v in ms.items() if v > 0}

    ctx64, oa64, ms64, n64, _, p64 = run(bvhg.PLAIN_FP64)
    ctx32, oa32, ms32, n32, cand32, p32 = run(bvhg.FILTER_FP32)
    stages64 = stage_ms(bvhg.PLAIN_FP64)
    stages32 = stage_ms(bvhg.FILTER_FP32)
    key64 = torch.sort(p64[:, 0] * (1 << 32) + p64[:, 1])[0]
    key32 = torch.sort(p32[:, 0] * (1 << 32) + p32[:, 1])[0]
    same = n64 == n32 and bool(torch.equal(key64, key32))
    # FP32 enclosure error over object A: lo32 <= lo64 and hi64 <= hi32 on every slab
    na = a_np.shape[0]
    s64 = ctx64.kdops(oa64, na)
    s32 = ctx32.kdops(oa32, na).astype(np.float64)
    err_lo, err_hi = s64[:, :, 0] - s32[:, :, 0], s32[:, :, 1] - s64[:, :, 1]
    width = s64[:, :, 1] - s64[:, :, 0]
    err = np.concatenate([err_lo.ravel(), err_hi.ravel()])
    rel = np.concatenate([(err_lo / width).ravel(), (err_hi / width).ravel()])
    bound = {"elements": int(na), "slabs_per_element": k // 2, "violations": int((err < 0).sum()),
             "max_abs": float(err.max()), "mean_abs": float(err.mean()),
             "max_rel_width": float(rel.max()), "mean_rel_width": float(rel.mean())}
    del s64, s32, err_lo, err_hi, width, err, rel
    ctx64.close()
    ctx32.close()
    oracle = None
    if rank == 0 and not args.no_oracle:
        # the oracle's OpenMP pipeline on the same objects, its pair list against the FP64 one (rank 0 only)
        from oracle import oracle as orc
        t = time.perf_counter()
        ocnt, _, want = orc.pipeline(a_np, b_np, k, 0.0, keep_pairs=True)
        dt = time.perf_counter() - t
        got = p64.cpu().numpy().astype(np.uint64)
        got = got[np.lexsort((got[:, 1], got[:, 0]))]
        oracle = {"pairs_match_oracle": bool(np.array_equal(got, want)), "oracle_pairs": int(ocnt),
                  "cpu_baseline": {"value": prims / dt / 1e6, "unit": "Mprims/s", "cores": orc.max_threads(),
                                   "kind": "port", "sample": "the whole workload, one pass with the pair list kept",
                                   "seconds": dt}}
        del want, got
    return {
        "metric": METRIC, "value": prims * world / (ms32 * 1e-3) / 1e6, "unit": "Mprims/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded tet lattice)",
        "config": {"workload": f"tet_lattice: {m}^3 jittered cells, one tet each ({prims} tets), checkerboard "
                               f"objects A/B, {k}-DOP", "k": k, "epsilon": 0.0, "elements": prims,
                   "l2": "inputs larger than L2"},
        "oracle": oracle,
        "form": "FP32 filter + FP64 recheck (value); FP64 plain below",
        "fp64_plain": {"ms_per_step": ms64, "value": prims * world / (ms64 * 1e-3) / 1e6, "pairs": int(n64),
                       "stages_ms": stages64},
        "filter_fp32": {"ms_per_step": ms32, "pairs": int(n32), "candidates": int(cand32), "same_pair_set": same,
                        "stages_ms": stages32,
                        "speedup_vs_fp64": ms64 / ms32,
                        "false_positive_rate": (cand32 - n32) / cand32 if cand32 else 0.0},
        "fp32_bound_error": bound,
    }


def run_batch_form(args, world, rank, local):
    """Batching form: 512 two-body scenes (per-scene counts LogUniform[1k, 200k], about 20M triangles), FP64,
    18-DOP, every build and scene traversal as one replayed CUDA graph with the autotuned lane count; pairs stay on
    the device. Parity: every scene's batch pair set against the single-scene path on a sample of scenes."""
    import torch
    import distbvh_b200 as bvhg
    from distbvh_b200 import meshes

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scenes = meshes.batch_scenes(512)
    prims = sum(a.shape[0] + b.shape[0] for a, b in scenes)
    stream = torch.cuda.Stream(device=dev)
    ctx = bvhg.Context(k=K, device=local, stream=stream.cuda_stream)
    tensors, objs = [], []
    for a, b in scenes:
        da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        oa, ob = ctx.object(), ctx.object()
        ctx.set_elements(oa, da, mem=bvhg.MEM_DEVICE)
        ctx.set_elements(ob, db, mem=bvhg.MEM_DEVICE)
        tensors += [da, db]
        objs.append((oa, ob))
    if args.batch_form:
        groups, lanes = (int(v) for v in args.batch_form.split(","))
        ctx.test_batch_form(groups, lanes)
        tune_ms = None
    else:
        groups, lanes, tune_ms = ctx.batch_autotune(objs)
    ia = np.ascontiguousarray([o[0] for o in objs], dtype=np.int32)
    ib = np.ascontiguousarray([o[1] for o in objs], dtype=np.int32)
    counts = np.zeros(len(objs), dtype=np.uint64)
    st = ctx.batch_broadphase_raw(ia.ctypes.data, ib.ctypes.data, len(objs), bvhg.REBUILD, None, 0,
                                  counts.ctypes.data, bvhg.MEM_DEVICE)
    total = int(counts.sum())
    out = torch.empty((max(total, 1), 2), dtype=torch.int64, device=dev)

    def step():
        st = ctx.batch_broadphase_raw(ia.ctypes.data, ib.ctypes.data, len(objs), bvhg.REBUILD, out.data_ptr(),
                                      out.shape[0], counts.ctypes.data, bvhg.MEM_DEVICE)
        assert st == 0, st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
    # parity sample: the batch's pairs of a scene = the single-scene path's
    offs = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    got = out[:total].cpu().numpy()
    checked, same = 0, True
    for sidx in np.linspace(0, len(objs) - 1, 12).astype(int):
        single = np.asarray(ctx.broadphase(*objs[sidx]), dtype=np.int64)
        mine = got[offs[sidx]:offs[sidx] + int(counts[sidx])]
        same = same and np.array_equal(np.unique(single, axis=0), np.unique(mine, axis=0))
        checked += 1
    ctx.close()
    return {
        "metric": METRIC, "value": prims * world / (ms * 1e-3) / 1e6, "unit": "Mprims/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded two-body scenes)",
        "config": {"workload": f"batch: 512 two-body scenes, per-scene elements LogUniform[1k, 200k] ({prims} tris),"
                               " 18-DOP, one CUDA graph", "k": K, "elements": prims, "pairs": total,
                   "groups": groups, "lanes": lanes, "autotune_ms": tune_ms},
        "parity": {"scenes_checked_against_single_scene_path": checked, "same_pair_sets": bool(same)},
    }


def run_timestep(args, world, rank, local):
    """Time-stepped contact: 32 tori of 262,144 triangles tumbling with seeded linear and angular velocities over
    64 steps (dt: at most half a mean edge of vertex motion per step), all 496 body pairs batched, FP32 filter +
    FP64 recheck. Refit every step vs rebuild every step vs rebuild every 8 steps; the pair sets of the refit run
    are compared with the rebuild run's every step."""
    import torch
    import distbvh_b200 as bvhg
    from distbvh_b200 import meshes

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nb, steps = 32, 64
    base = torch.from_numpy(meshes.torus(512, 256)).to(dev)
    rng = np.random.default_rng(21)
    centers = np.array([[1.2 * (i % 4), 1.2 * ((i // 4) % 4), 0.9 * (i // 16)] for i in range(nb)], dtype=np.float64)
    v = rng.uniform(-1.0, 1.0, (nb, 3))
    w = rng.uniform(-1.0, 1.0, (nb, 3))
    edge = 0.00666
    dt = 0.5 * edge / float(np.max(np.linalg.norm(v, axis=1) + np.linalg.norm(w, axis=1) * 0.65))

    def rot(axis_angle):
        th = np.linalg.norm(axis_angle)
        if th == 0:
            return np.eye(3)
        k = axis_angle / th
        Kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
        return np.eye(3) + np.sin(th) * Kx + (1 - np.cos(th)) * Kx @ Kx

    init_R = [rot(rng.uniform(-np.pi, np.pi, 3)) for _ in range(nb)]

    def pose(t):
        """Vertices of every body at step t (rigid motion about its own centre)."""
        out = []
        for i in range(nb):
            R = torch.from_numpy(rot(w[i] * dt * t) @ init_R[i]).to(dev)
            c = torch.from_numpy(centers[i] + v[i] * dt * t).to(dev)
            out.append(base @ R.T + c)
        return out

    scenes = [(i, j) for i in range(nb) for j in range(i + 1, nb)]
    stream = torch.cuda.Stream(device=dev)

    def run(policy):
        ctx = bvhg.Context(k=K, precision=bvhg.FILTER_FP32, device=local, stream=stream.cuda_stream)
        bodies = pose(0)
        objs = [ctx.object() for _ in range(nb)]
        for o, x in zip(objs, bodies):
            ctx.set_elements(o, x, mem=bvhg.MEM_DEVICE)
        sc = [(objs[i], objs[j]) for i, j in scenes]
        ia = np.ascontiguousarray([a for a, _ in sc], dtype=np.int32)
        ib = np.ascontiguousarray([b for _, b in sc], dtype=np.int32)
        counts = np.zeros(len(sc), dtype=np.uint64)
        cap = 1 << 22
        out = torch.empty((cap, 2), dtype=torch.int64, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total_ms, sets = 0.0, []
        for t in range(steps):
            if t:
                new = pose(t)
                for x, y in zip(bodies, new):
                    x.copy_(y)  # in place: the graph's borrowed pointers stay valid
            torch.cuda.synchronize(dev)
            mode = bvhg.REBUILD if policy(t) else bvhg.REFIT
            e0.record(stream)
            st = ctx.batch_broadphase_raw(ia.ctypes.data, ib.ctypes.data, len(sc), mode, out.data_ptr(), cap,
                                          counts.ctypes.data, bvhg.MEM_DEVICE)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            assert st == 0, st
            if t >= 2:  # the first two steps capture the REBUILD and REFIT graphs
                total_ms += e0.elapsed_time(e1)
            n = int(counts.sum())
            keys = torch.sort(out[:n, 0] * (1 << 32) + out[:n, 1])[0]
            sets.append((counts.copy(), keys))
        ctx.close()
        return total_ms / (steps - 2), sets

    ms_refit, sets_refit = run(lambda t: t == 0)
    ms_rebuild, sets_rebuild = run(lambda t: True)
    ms_r8, sets_r8 = run(lambda t: t % 8 == 0)
    same = all(np.array_equal(a[0], b[0]) and bool(torch.equal(a[1], b[1])) and
               np.array_equal(a[0], c[0]) and bool(torch.equal(a[1], c[1]))
               for a, b, c in zip(sets_refit, sets_rebuild, sets_r8))
    prims = nb * base.shape[0]
    pairs_per_step = [int(c.sum()) for c, _ in sets_rebuild]
    return {
        "metric": METRIC, "value": prims * world / (ms_refit * 1e-3) / 1e6, "unit": "Mprims/s", "n_gpus": world,
        "steps": steps, "warmup": 2, "ms_per_step": ms_refit, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded tumbling tori)",
        "config": {"workload": f"timestep: {nb} tori x {base.shape[0]} tris, {len(scenes)} body pairs batched, "
                               f"{steps} steps, FP32 filter + FP64 recheck", "k": K, "elements": prims,
                   "dt": dt, "pairs_min_max": [min(pairs_per_step), max(pairs_per_step)]},
        "refit_every_step_ms": ms_refit, "rebuild_every_step_ms": ms_rebuild, "rebuild_every_8_ms": ms_r8,
        "same_pair_sets_every_step": bool(same),
    }


def cpu_baseline_full(sphere, plate, gpu_pairs, threads=0):
    """The reference's algorithms on all host cores over the whole benchmark scene (one pass, about 4 s on 16
    cores), with the pair list kept: it is both the CPU baseline and the oracle's pair set for the GPU's."""
    from oracle import oracle as orc
    t = time.perf_counter()
    cnt, stages, want = orc.pipeline(sphere, plate, K, EPS, threads, keep_pairs=True)
    dt = time.perf_counter() - t
    n = sphere.shape[0] + plate.shape[0]
    got = np.asarray(gpu_pairs).astype(np.uint64)
    got = got[np.lexsort((got[:, 1], got[:, 0]))] if got.shape[0] else got.reshape(0, 2)
    out = {"value": n / dt / 1e6, "unit": "Mprims/s", "cores": orc.max_threads() if threads == 0 else threads,
           "kind": "port", "sample": f"the whole benchmark scene ({n} tris), 18-DOP, one pass with the pair list "
           "kept", "seconds": dt, "pairs": int(cnt), "stages_s": stages,
           "pairs_match_oracle": bool(np.array_equal(got, want))}
    # The reference's own serial element path (its headers, built into oracle/_ref when the sources were present):
    # from_vertices, top-down tree of dop_26 snapshots, potential_collision_set; 26-DOP, its only tree form.
    from oracle import ref
    from distbvh_b200 import meshes
    if ref.available():
        s6, p6 = meshes.sphere_plate(6, 256, 128)
        r = ref.Ref(26)
        t = time.perf_counter()
        rc, _ = r.tree_pairs(s6, p6, EPS, cap=0)
        dt6 = time.perf_counter() - t
        n6 = s6.shape[0] + p6.shape[0]
        out["reference_code"] = {"value": n6 / dt6 / 1e6, "unit": "Mprims/s", "cores": 1, "k": 26,
                                 "sample": f"icosphere L6 + plate 256x128 quads ({n6} tris), the reference's serial "
                                           "top-down dop_26 path", "seconds": dt6, "pairs": rc}
    return out


def run_reference(args, world, rank):
    """Reference arm: the reference's algorithms for this path on all host cores (OpenMP restatement of the Kokkos
    path: from_vertices, compute_bounds, morton, one-bit radix sort, then the serial top-down tree and a parallel
    query_tree), one pass over the whole benchmark scene per step, the pair list kept. Only the oracle and the mesh
    generators are imported: the CUDA library is never loaded here."""
    if rank != 0:
        return None
    from oracle import oracle as orc
    from distbvh_b200 import meshes
    s, p = meshes.sphere_plate(args.level, args.nx, args.ny)
    n = s.shape[0] + p.shape[0]
    for _ in range(args.warmup):
        orc.pipeline(s, p, K, EPS)
    times = []
    cnt = 0
    for _ in range(args.steps):
        t = time.perf_counter()
        cnt, _ = orc.pipeline(s, p, K, EPS)
        times.append(time.perf_counter() - t)
    ms = float(np.mean(times)) * 1e3
    value = n / (ms * 1e-3) / 1e6
    sample = f"the whole benchmark scene ({n} tris) per step"
    return {
        "metric": METRIC, "value": value, "unit": "Mprims/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded icosphere + plate)",
        "config": bench_config(args, world, n, cnt),
        "sort_digit_bits": 1,
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "Mprims/s", "cores": orc.max_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Mprims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_sweep(args, world, rank, local):
    """Sort-and-sweep (the reference's narrowphase candidate generator, src/bvh/narrowphase/kokkos.hpp:164-248)
    between two patch-sized objects: 262,144 random triangles each (centres U(0,1)^3, vertices within +-0.004),
    18-DOP, FP64, axis of largest centroid variance. A step is one bvhg_sort_and_sweep (keys, radix sort, sweep;
    pairs left on the device) over built objects; the tree broadphase on the same objects is timed beside it and
    both pair sets are compared. CPU baseline: the oracle's serial restatement of the reference's loop on the first
    32,768 elements of each object (its skip phase is quadratic)."""
    import torch
    import distbvh_b200 as bvhg
    from distbvh_b200 import meshes

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = 262144
    a = meshes.random_soup(n, 3, seed=31, size=0.004)
    b = meshes.random_soup(n, 3, seed=32, size=0.004, stream=1)
    stream = torch.cuda.Stream(device=dev)
    ctx = bvhg.Context(k=K, device=local, stream=stream.cuda_stream)
    da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    oa, ob = ctx.object(), ctx.object()
    ctx.set_elements(oa, da, mem=bvhg.MEM_DEVICE)
    ctx.set_elements(ob, db, mem=bvhg.MEM_DEVICE)
    ctx.build(oa)
    ctx.build(ob)
    cap = 1 << 22
    out = torch.empty((cap, 2), dtype=torch.int64, device=dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)

    res = {}

    def sweep():
        st, cnt, axis = ctx.sort_and_sweep_raw(oa, ob, -1, out.data_ptr(), cap, bvhg.MEM_DEVICE)
        assert st == 0, st
        res["sweep"] = (cnt, axis)

    def tree():
        st, cnt = ctx.broadphase_raw(oa, ob, out.data_ptr(), cap, bvhg.MEM_DEVICE)
        assert st == 0, st
        res["tree"] = cnt

    ms_sweep = timed(sweep)
    ms_tree = timed(tree)
    got_sweep, axis = ctx.sort_and_sweep(oa, ob, -1)
    got_tree = ctx.broadphase(oa, ob)
    same = bool(np.array_equal(np.unique(got_sweep, axis=0), np.unique(got_tree, axis=0)))
    ctx.close()
    result = {
        "metric": METRIC, "value": 2 * n * world / (ms_sweep * 1e-3) / 1e6, "unit": "Mprims/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_sweep, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded triangle soups)",
        "config": {"workload": f"sweep: sort-and-sweep of two {n}-triangle soups (vertices within +-0.004 of "
                               "U(0,1)^3 centres), 18-DOP, objects built before the timed region",
                   "k": K, "elements": 2 * n, "pairs": int(got_sweep.shape[0]), "axis": int(axis)},
        "tree_broadphase_ms": ms_tree, "same_pair_set_as_tree": same,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        m = 32768
        sa, sb = orc.kdops(a[:m], K), orc.kdops(b[:m], K)
        t0 = time.perf_counter()
        cnt = orc.sort_and_sweep(sa, sb, K, int(axis)).shape[0]
        dt = time.perf_counter() - t0
        result["cpu_baseline"] = {"value": 2 * m / dt / 1e6, "unit": "Mprims/s", "cores": 1, "kind": "port",
                                  "sample": f"the first {m} elements of each object ({cnt} pairs), the reference's "
                                            "sweep loop restated serially, slabs given"}
    return result


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
        if out is not None:
            print(json.dumps(out))
        return
    if args.workload != "sphere_plate":
        fn = {"tet_lattice": run_precision, "batch": run_batch_form, "timestep": run_timestep,
              "sweep": run_sweep}[args.workload]
        result = fn(args, world, rank, local)
        if rank == 0:
            print(json.dumps(result))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    result, sphere, plate, p64 = run_gpu(args, world, rank, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline_full(sphere, plate, p64)
            result["pairs_match_oracle"] = cb["pairs_match_oracle"]
            result["cpu_baseline"] = cb
        print(json.dumps(result))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
