#!/usr/bin/env python3
"""Benchmark of the homography grid search (one JSON line on rank 0).

Workload: the NCC single-pair configuration -- 256x256 float32 images from the seeded
blob+sinusoid generator, zero-mean NCC, 6 values on each of the 8 homography parameters
(1,679,616 grid points), argmin plus the per-point cost dump.  A step is one full search.

* ``value``  -- grid-point evaluations per second with the images already in HBM
  (CUDA events on the launching stream; L2 flushed by a 256 MiB write between steps).
* ``e2e``    -- the same metric through the public C ABI with host buffers: each step
  copies both images from pinned host memory, searches, and copies the cost dump and
  the argmin back.
* ``roofline`` -- FP32 pipe: algorithmic flops per launch (36 per pixel evaluation for
  NCC: projective map 14, bilinear 16, cost 6) over the measured launch time, against
  the FP32 FMA peak (148 SMs x 128 lanes x 2 flops x max SM clock).
* ``cpu_baseline`` -- the reference's own calcNCC (src/gpu/cudaErrorFunctions.cuh:448-507)
  built for the host, on a strided sample of the same grid, all host threads.

``--impl reference`` times that reference CPU path alone, as the reference arm.
Multi-GPU (torchrun): one pair per rank (weak scaling), no collective on the data path;
the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOPS_PER_PIXEL_EVAL = {"ZNCC": 36, "NCC_REF": 36, "SAD_AVG": 32, "MI": 34}
WORKLOADS = {
    "ncc": "ncc-single-pair 256x256 f32, zero-mean NCC, 6^8 = 1,679,616 grid points, argmin + cost dump",
    "mi": "mi-single-pair 512x512 u8 (gamma-remapped moving), MI 32x32 bins, 5^8 = 390,625 grid points",
    "sad": "sad-small 64x64 f32, SAD over the overlap (averageAbsoluteDifference), 4^8 = 65,536 grid points",
    "batch": "batched-uneven-pairs: 64 pairs, square f32 128-1024 px (log-uniform), costs SAD / ZNCC / MI-32 "
             "in turn, own ranges, 4-6 values per parameter; one persistent launch replayed from a CUDA graph",
}
WORKLOAD = WORKLOADS["ncc"]
METRIC = "homography evals/s"
UNIT = "grid-point evals/s"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one search_kernel launch on the
# full-size workload, from a one-pass ncu capture of `bench.py --no-cpu-baseline --steps 1
# --warmup 3` (the default ncc workload, ZNCC with the default taps): 2.05 MB read (images and
# staging, once), 512 B written (the 6.7 MB cost dump stays in the 126 MB L2 while the kernel
# runs).  Measured for that configuration only; the others report null.
TRAFFIC_BYTES_PER_LAUNCH = {"ncc": 2050000 + 512}


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest x over the ranks (the job's time is its slowest rank's); x itself alone."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(rank: int, base: int) -> int:
    """Seed of a rank's pair: every rank searches its own pair (weak scaling, replicas)."""
    return base + rank


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.path or not os.path.exists(self.path):
            return out
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        load = [s for s in sm if s > 0.5 * (max(sm) if sm else 1)]
        out.update(sm_mhz=statistics.median(load) if load else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=sorted(reasons), samples=len(rows))
        return out


def cpu_baseline(pair, cost_ref: str, budget_s: float = 12.0):
    """Time the reference's functor (oracle/_ref) -- or the oracle port when the reference
    build is absent -- on a strided sample of the grid, all host threads."""
    import oracle as O
    kind = "reference" if O.have_ref() else "port"
    F, M = O.Image(pair.fixed), O.Image(pair.moving)
    g = O.make_grid(*pair.grid_args())
    n = O.grid_num(g)
    threads = (O.ref().cgsref_max_threads() if kind == "reference" else os.cpu_count()) or 1

    def run(count, stride):
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_search(cost_ref, g, M, F, first=0, count=count, stride=stride, threads=threads)
        else:
            O.search(cost_ref, g, M, F, first=0, count=count, stride=stride, f64=False, threads=threads)
        return time.perf_counter() - t0

    probe = max(threads * 2, 16)
    t = run(probe, n // probe)
    per_point = t / probe
    count = int(max(probe, min(n, budget_s / max(per_point, 1e-9))))
    stride = max(1, n // count)
    count = min(count, (n + stride - 1) // stride)
    t = run(count, stride)
    return {"value": count / t, "unit": UNIT, "cores": int(threads), "kind": kind,
            "sample": f"{count} grid points of {n} (every {stride}th index), reference {cost_ref} per point, "
                      f"{t:.1f} s on {threads} host threads; value extrapolates points/s to the full grid"}


def reference_arm(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    from cugridsearch_b200 import synthetic as S
    pair = S.config1()
    per_step = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(pair, "NCC_REF", budget_s=max(2.0, args.ref_budget))
        if i >= args.warmup:
            per_step.append(r)
    vals = [r["value"] for r in per_step]
    v = statistics.median(vals)
    n_points = 6 ** 8
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n_points / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD, "grid_points": n_points, "pixels": 65536,
                       "note": "the reference has no zero-mean NCC; its calcNCC is timed on the same grid"},
            "cpu_baseline": dict(per_step[-1], value=v),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def batch_bench(args):
    """Batched uneven pairs: pairs/s of one persistent launch (graph replay), per-pair
    completion latency p50/p99 from the kernel's time stamps, and the end-to-end rate with
    the images copied in from pinned host memory and the results copied out every step."""
    import torch
    import cugridsearch_b200 as cgs
    from cugridsearch_b200 import synthetic as S

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    t_gen = time.perf_counter()
    pairs = S.config3_pairs(rank_seed(rank, S.DEFAULT_SEED), n=args.pairs)
    t_gen = time.perf_counter() - t_gen
    stream = torch.cuda.Stream(device=dev)
    host, dev_imgs, bps, results = [], [], [], []
    points = 0
    pixel_evals = 0
    for pr in pairs:
        mh, fh = torch.from_numpy(pr.moving).pin_memory(), torch.from_numpy(pr.fixed).pin_memory()
        md, fd = mh.to(dev), fh.to(dev)
        grid = cgs.CudaGrid.from_ranges(*pr.grid_args())
        res = cgs.result_buffer(dev)
        host.append((mh, fh))
        dev_imgs.append((md, fd))
        results.append(res)
        bps.append(cgs.BatchPair(pr.cost, cgs.CudaImage(md), cgs.CudaImage(fd), grid, res))
        points += grid.numElements()
        pixel_evals += grid.numElements() * pr.fixed.shape[0] * pr.fixed.shape[1]
    torch.cuda.synchronize(dev)
    batch = cgs.Batch(bps)
    tune = None
    if args.autotune > 0:
        t0 = time.perf_counter()
        best, table = batch.autotune(sample_points=args.autotune)
        tune = {"sample_points": args.autotune, "seconds": round(time.perf_counter() - t0, 2),
                "best": vars(best), "table": [[vars(p), (round(ms, 3) if np.isfinite(ms) else None), st]
                                              for p, ms, st in table]}
    plan = batch.plan
    for _ in range(args.warmup):
        batch.launch(stream)
    stream.synchronize()
    times, lat, span = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.launch(stream)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            t0, t1 = batch.pair_times()
            base = int(t0.min())
            lat.extend(((t1.astype(np.int64) - base) / 1e6).tolist())
            span.extend(((t1.astype(np.int64) - t0.astype(np.int64)) / 1e6).tolist())
    clocks = clk.summary()
    ms = max_over_ranks(statistics.median(times), world, dev)
    # end to end: images in from pinned host memory, the launch, results out
    res_h = [torch.empty(r.numel(), dtype=torch.uint8).pin_memory() for r in results]
    e2e = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            for (mh, fh), (md, fd) in zip(host, dev_imgs):
                md.copy_(mh, non_blocking=True)
                fd.copy_(fh, non_blocking=True)
        batch.launch(stream)
        with torch.cuda.stream(stream):
            for r, rh in zip(results, res_h):
                rh.copy_(r, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1))
    out = [cgs.read_result(r) for r in results]
    h2d = sum(mh.numel() * mh.element_size() + fh.numel() * fh.element_size() for mh, fh in host)
    batch.close()
    e2e_ms = max_over_ranks(statistics.median(e2e), world, dev)
    if world > 1:
        dist.destroy_process_group()
    n = len(pairs) * world  # every rank runs its own batch (weak scaling)
    points *= world
    pixel_evals *= world
    line = {"metric": "pairs/s (batched uneven pairs)", "value": n / (ms / 1e3), "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOADS["batch"], "pairs": n, "grid_points": points, "pixel_evals": pixel_evals,
                       "plan": vars(plan), "l2": "inputs exceed L2 (staged planes + dumps of all pairs)"},
            "grid_point_evals_per_s": points / (ms / 1e3), "pixel_evals_per_s": pixel_evals / (ms / 1e3),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "span_p50": float(np.percentile(span, 50)),
                           "definition": "pair finish minus the launch's first task start (globaltimer)"},
            "e2e": {"value": n / (e2e_ms / 1e3), "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": sum(r.numel() for r in res_h)},
            "gpu_launches": 2 * args.steps,
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "status_ok": all(r.status == 0 and r.valid for r in out), "generation_s": round(t_gen, 1)}
    if tune:
        line["autotune"] = tune
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cost", default="ZNCC")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--points-per-warp", type=int, default=0, help="0 = library choice")
    ap.add_argument("--ref-budget", type=float, default=6.0, help="seconds of CPU work per reference step")
    ap.add_argument("--small", action="store_true", help="3^8 grid (for profiling captures)")
    ap.add_argument("--taps", default="auto", choices=["auto", "quad", "texture"],
                    help="tap source of the fast path (auto: the library's choice)")
    ap.add_argument("--workload", default="ncc", choices=["ncc", "mi", "sad", "batch"],
                    help="ncc: the headline 256^2 ZNCC pair; mi: 512^2 u8 MI pair; sad: 64^2 SAD pair; "
                         "batch: 64 uneven pairs in one persistent launch")
    ap.add_argument("--autotune", type=int, default=0,
                    help="batch: autotune the plan on this many points per pair first (0 = default plan)")
    ap.add_argument("--pairs", type=int, default=64, help="batch: number of pairs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch":
        return batch_bench(args)

    import torch
    import torch.distributed as dist
    import cugridsearch_b200 as cgs
    from cugridsearch_b200 import synthetic as S

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    seed = rank_seed(rank, S.DEFAULT_SEED)
    if args.workload == "mi":
        pair, cost = S.config2(seed), "MI"
    elif args.workload == "sad":
        pair, cost = S.config0(seed), "SAD_AVG"
    else:
        pair, cost = S.config1(seed), args.cost
    if args.small:
        pair.count[:] = 3
    stream = torch.cuda.Stream(device=dev)
    mov_h = torch.from_numpy(pair.moving).pin_memory()
    fix_h = torch.from_numpy(pair.fixed).pin_memory()
    with torch.cuda.stream(stream):
        mov_d = mov_h.to(dev, non_blocking=True)
        fix_d = fix_h.to(dev, non_blocking=True)
    stream.synchronize()
    mov, fix = cgs.CudaImage(mov_d), cgs.CudaImage(fix_d)
    grid = cgs.CudaGrid.from_ranges(*pair.grid_args())
    n = grid.numElements()
    costs = torch.empty(n, dtype=torch.float32, device=dev)
    res = cgs.result_buffer(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    pix = pair.fixed.shape[0] * pair.fixed.shape[1] * pair.fixed.shape[2]

    def step():
        cgs.search(cost, mov, fix, grid, costs=costs, result=res, stream=stream, points_per_warp=args.points_per_warp,
                   quad_taps={"auto": None, "quad": True, "texture": False}[args.taps])

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step()
    barrier()

    # ---- device-resident timing, L2 flushed between steps
    times = []
    with ClockSampler(local) as clk:
        barrier()
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        barrier()
    clocks = clk.summary()
    total_ms = max_over_ranks(sum(times), world, dev)
    ms_per_step = total_ms / args.steps
    value = world * n * args.steps / (total_ms / 1e3)
    r = cgs.read_result(res)

    # ---- end to end through the C ABI with host buffers
    costs_h = torch.empty(n, dtype=torch.float32).pin_memory()
    res_h = torch.empty(res.numel(), dtype=torch.uint8).pin_memory()
    e2e_ms = []
    barrier()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            mov_d.copy_(mov_h, non_blocking=True)
            fix_d.copy_(fix_h, non_blocking=True)
        step()
        with torch.cuda.stream(stream):
            costs_h.copy_(costs, non_blocking=True)
            res_h.copy_(res, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    barrier()
    e2e_total = max_over_ranks(sum(e2e_ms), world, dev)
    e2e_value = world * n * args.steps / (e2e_total / 1e3)
    h2d = mov_h.numel() * mov_h.element_size() + fix_h.numel() * fix_h.element_size()
    d2h = costs_h.numel() * 4 + res_h.numel()

    # ---- roofline of the dominant kernel (search_kernel; the staging kernel is <1% of a call)
    flops = FLOPS_PER_PIXEL_EVAL.get(cost, 36) * n * pix
    achieved = flops / (ms_per_step / 1e3) / 1e12
    props = torch.cuda.get_device_properties(dev)
    sm_max = clocks.get("sm_max_mhz") or 1965.0
    peak = props.multi_processor_count * 128 * 2 * sm_max * 1e6 / 1e12
    roofline = {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4),
                "traffic": (TRAFFIC_BYTES_PER_LAUNCH.get(args.workload)
                            if cost == "ZNCC" and not args.small and args.taps == "auto" else None),
                "peak_source": "nominal FP32 FMA rate: SMs x 128 lanes x 2 flops x max SM clock "
                               "(MEASURED_PEAKS.json holds HBM and bf16 tensor peaks only)",
                "flops_per_pixel_eval": FLOPS_PER_PIXEL_EVAL.get(cost, 36),
                "pixel_evals_per_s": n * pix / (ms_per_step / 1e3)}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded blob+sinusoid generator, seed "
                                                          f"{S.DEFAULT_SEED}+rank)",
            "config": {"workload": WORKLOADS[args.workload] + (" (3^8 grid)" if args.small else ""), "cost": cost,
                       "grid_points": n, "pixels": pix, "points_per_warp": args.points_per_warp or "tuned",
                       "taps": args.taps,
                       "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_total / args.steps},
            "gpu_launches": 2 * args.steps,
            "roofline": roofline,
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "argmin": {"index": r.index, "cost": r.cost, "params": [float(x) for x in r.params]}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(pair, "NCC_REF" if cost in ("ZNCC", "NCC_REF") else cost)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
