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
             "in turn, own ranges, 4-6 values per parameter; one recorded launch sequence (persistent kernel, "
             "multi-pair span kernel, MI span searches) replayed from a CUDA graph",
}
WORKLOAD = WORKLOADS["ncc"]
METRIC = "homography evals/s"
UNIT = "grid-point evals/s"
# DRAM bytes per launch of the dominant kernel come from an ncu capture recorded in
# profiles/traffic.json together with a hash of the kernel sources it was taken on; the bench
# reports the figure only while the sources still hash the same (otherwise null).
KERNEL_SOURCES = ["cugridsearch_b200/csrc/cgs_span.cuh", "cugridsearch_b200/csrc/cgs_span_mi.cuh",
                  "cugridsearch_b200/csrc/cgs_kernels.cuh", "cugridsearch_b200/csrc/cgs_device.cuh",
                  "cugridsearch_b200/csrc/cgs_search.cu"]
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.json")


def kernel_sources_sha16() -> str:
    import hashlib
    h = hashlib.sha256()
    for f in KERNEL_SOURCES:
        with open(os.path.join(ROOT, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def recorded_traffic(workload: str):
    """(bytes per launch, provenance) of the workload's recorded capture, or (None, why)."""
    try:
        rec = json.load(open(TRAFFIC_FILE)).get(workload)
    except (OSError, ValueError):
        rec = None
    if not rec:
        return None, "no capture recorded for this workload"
    if rec.get("sources_sha16") != kernel_sources_sha16():
        return None, "the recorded capture was taken on other kernel sources"
    return int(rec["dram_bytes"]), f"ncu capture of {rec.get('kernel')} ({rec.get('command')})"


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


class RefSample:
    """The reference's functor (oracle/_ref) -- or the oracle port when the reference build is
    absent -- on a fixed strided sample of a pair's grid, on every host thread: one run of
    run() is one timed step of the reference arm."""

    def __init__(self, pair, cost_ref: str, budget_s: float):
        import oracle as O
        self.O, self.cost = O, cost_ref
        self.kind = "reference" if O.have_ref() else "port"
        self.F, self.M = O.Image(pair.fixed), O.Image(pair.moving)
        self.g = O.make_grid(*pair.grid_args())
        self.n = O.grid_num(self.g)
        self.threads = (O.ref().cgsref_max_threads() if self.kind == "reference" else os.cpu_count()) or 1
        probe = max(self.threads * 2, 16)
        per_point = self._timed(probe, self.n // probe) / probe
        count = int(max(probe, min(self.n, budget_s / max(per_point, 1e-9))))
        self.stride = max(1, self.n // count)
        self.count = min(count, (self.n + self.stride - 1) // self.stride)

    def _timed(self, count, stride):
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.O.ref_search(self.cost, self.g, self.M, self.F, first=0, count=count, stride=stride,
                              threads=self.threads)
        else:
            self.O.search(self.cost, self.g, self.M, self.F, first=0, count=count, stride=stride, f64=False,
                          threads=self.threads)
        return time.perf_counter() - t0

    def run(self) -> float:
        """Seconds of one pass over the sample."""
        return self._timed(self.count, self.stride)

    def describe(self, seconds: float) -> str:
        return (f"{self.count} grid points of {self.n} (every {self.stride}th index), reference {self.cost} per "
                f"point, {seconds:.2f} s on {self.threads} host threads")


def cpu_baseline(pair, cost_ref: str, budget_s: float = 12.0):
    """The reported CPU baseline: points/s of the reference's functor on a bounded sample."""
    smp = RefSample(pair, cost_ref, budget_s)
    t = smp.run()
    return {"value": smp.count / t, "unit": UNIT, "cores": int(smp.threads), "kind": smp.kind,
            "sample": smp.describe(t) + "; points/s of the sample"}


def reference_arm(args):
    """The reference's own CPU path on the NCC pair: each step is one pass of the reference's
    calcNCC over the same fixed strided sample of the 6^8 grid (all host threads); value =
    sample points / step time."""
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    from cugridsearch_b200 import synthetic as S
    pair = S.config1()
    smp = RefSample(pair, "NCC_REF", budget_s=max(0.5, args.ref_budget))
    times = []
    for i in range(args.warmup + args.steps):
        t = smp.run()
        if i >= args.warmup:
            times.append(t)
    t_med = statistics.median(times)
    v = smp.count / t_med
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_med,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD, "grid_points": smp.n, "pixels": 65536,
                       "step": f"one pass over a fixed strided sample of {smp.count} of the {smp.n} grid points",
                       "note": "the reference has no zero-mean NCC; its calcNCC is timed on the same grid"},
            "full_grid_ms_extrapolated": 1e3 * t_med * smp.n / smp.count,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": int(smp.threads), "kind": smp.kind,
                             "sample": smp.describe(t_med)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def measure_batch(dev, rank: int, world: int, n_pairs: int, steps: int, warmup: int, autotune: int = 0) -> dict:
    """The batched uneven pairs on one GPU: pairs/s of one batch launch (graph replay of the
    persistent kernel and the span-kernel searches, CUDA events), per-pair completion latency
    p50/p99 from the kernels' time stamps, and the end-to-end rate with the images copied in from
    pinned host memory and the results copied out every step."""
    import torch
    import cugridsearch_b200 as cgs
    from cugridsearch_b200 import synthetic as S

    t_gen = time.perf_counter()
    pairs = S.config3_pairs(rank_seed(rank, S.DEFAULT_SEED), n=n_pairs)
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
    if autotune > 0:
        t0 = time.perf_counter()
        best, table = batch.autotune(sample_points=autotune)
        tune = {"sample_points": autotune, "seconds": round(time.perf_counter() - t0, 2),
                "best": vars(best), "table": [[vars(p), (round(ms, 3) if np.isfinite(ms) else None), st]
                                              for p, ms, st in table]}
    plan = batch.plan
    launches = batch.kernel_launches
    for _ in range(warmup):
        batch.launch(stream)
    stream.synchronize()
    times, lat, span = [], [], []
    with ClockSampler(dev.index or 0) as clk:
        for _ in range(steps):
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
    res_h = [torch.empty(r.numel(), dtype=torch.uint8).pin_memory() for r in results]
    e2e = []
    for _ in range(steps):
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
    n = len(pairs) * world  # every rank runs its own batch (weak scaling)
    return {"pairs": n, "ms": ms, "pairs_per_s": n / (ms / 1e3), "grid_points": points * world,
            "pixel_evals": pixel_evals * world, "grid_point_evals_per_s": points * world / (ms / 1e3),
            "pixel_evals_per_s": pixel_evals * world / (ms / 1e3), "plan": vars(plan),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "span_p50": float(np.percentile(span, 50)),
                           "definition": "pair finish minus the launch's first task start (globaltimer)"},
            "e2e": {"value": n / (e2e_ms / 1e3), "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": sum(r.numel() for r in res_h)},
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "status_ok": all(r.status == 0 and r.valid for r in out), "generation_s": round(t_gen, 1),
            "kernel_launches_per_step": launches, "autotune": tune}


PROPOSAL_CHECKPOINT = os.path.join(ROOT, "models", "proposal_net.npz")
PROPOSAL_SERVING = dict(values=3, levels=4, spread=2.0, min_half=0.02, walks=2)


def measure_proposal(dev, n_pairs: int = 64, seed: int = 20261203 + 10 ** 7) -> dict:
    """The learned proposal against the full grid on held-out pairs of the learned-proposal
    configuration (256 px, full 6^8 zero-mean NCC grid): both paths timed with CUDA events on the
    same device-resident pairs (network, refinement launches, orchestration and fallbacks
    included), and end to end with the pairs copied in from pinned host memory; corner errors
    against the generator's ground truth and against the full grid's argmin."""
    import torch
    from cugridsearch_b200 import proposal as P

    fe, me, gt = P.config4_batch_cached(seed, n_pairs, dev)
    fh, mh = fe.cpu().pin_memory(), me.cpu().pin_memory()
    net = P.ProposalNet(max_batch=256)
    net.load(PROPOSAL_CHECKPOINT)
    full = P.full_grid(256, 6)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        e1.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    P.refine_serve(net, fe, me, full, **PROPOSAL_SERVING)  # warm-up on the same pairs
    with ClockSampler(dev.index or 0) as clk:
        (truth, tcost), t_full = timed(lambda: P.grid_argmins(fe, me, full))
        prop_runs = [timed(lambda: P.refine_serve(net, fe, me, full, **PROPOSAL_SERVING)) for _ in range(3)]
        r, t_prop = sorted(prop_runs, key=lambda v: v[1])[1]  # the median run

        def e2e():
            fe.copy_(fh, non_blocking=True)
            me.copy_(mh, non_blocking=True)
            return P.refine_serve(net, fe, me, full, **PROPOSAL_SERVING)
        e2e_runs = [timed(e2e) for _ in range(3)]
        r2, t_e2e = sorted(e2e_runs, key=lambda v: v[1])[1]
    clocks = clk.summary()
    net.close()
    g = gt.numpy()
    err_gt = P.corner_error(r.params, g, 256)
    err_full_gt = P.corner_error(truth, g, 256)
    err_vs_full = P.corner_error(r.params, truth, 256)
    gap = r.costs - tcost
    return {"pairs": n_pairs, "checkpoint": os.path.relpath(PROPOSAL_CHECKPOINT, ROOT), "serving": PROPOSAL_SERVING,
            "full_grid_pairs_per_s": n_pairs / t_full, "proposal_pairs_per_s": n_pairs / t_prop,
            "speedup": t_full / t_prop, "fallback_rate": float(r.fallback.mean()),
            "corner_error_vs_ground_truth_px": {"proposal_mean": float(err_gt.mean()),
                                                "proposal_p90": float(np.percentile(err_gt, 90)),
                                                "full_grid_mean": float(err_full_gt.mean())},
            "corner_error_vs_full_grid_px": {"mean": float(err_vs_full.mean()),
                                             "p90": float(np.percentile(err_vs_full, 90))},
            "cost_not_above_full_grid": float(np.mean(gap <= 0.0)), "cost_gap_mean": float(gap.mean()),
            "points_fraction": r.points / (n_pairs * full.numElements()),
            "timing_runs_s": {"proposal": [round(v[1], 4) for v in prop_runs], "statistic": "median of 3 runs",
                              "e2e": [round(v[1], 4) for v in e2e_runs],
                              "e2e_fallbacks": [int(v[0].fallback.sum()) for v in e2e_runs]},
            "e2e": {"value": n_pairs / t_e2e, "unit": "pairs/s",
                    "h2d_bytes_per_step": int(fh.numel() * 4 + mh.numel() * 4),
                    "d2h_bytes_per_step": int(r2.d2h_bytes)},
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "status_ok": bool(np.all(np.isfinite(r.costs))),
            "workload": "learned-proposal: held-out 256x256 f32 pairs (config-4 generator), rotation +-20 deg, "
                        "translation +-32 px; full grid 6^8 zero-mean NCC; proposal = CNN centre and radii, then "
                        "coarse-to-fine local grids of 3 values per axis, full-grid fallback above the coarse probe"}


def batch_bench(args):
    """The batched workload as the bench line itself (--workload batch)."""
    import torch

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    m = measure_batch(dev, rank, world, args.pairs, args.steps, args.warmup, args.autotune)
    if world > 1:
        dist.destroy_process_group()
    line = {"metric": "pairs/s (batched uneven pairs)", "value": m["pairs_per_s"], "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOADS["batch"], "pairs": m["pairs"], "grid_points": m["grid_points"],
                       "pixel_evals": m["pixel_evals"], "plan": m["plan"],
                       "l2": "inputs exceed L2 (staged planes + dumps of all pairs)"},
            "grid_point_evals_per_s": m["grid_point_evals_per_s"], "pixel_evals_per_s": m["pixel_evals_per_s"],
            "latency_ms": m["latency_ms"], "e2e": m["e2e"], "gpu_launches": m["kernel_launches_per_step"] * args.steps,
            "clocks": m["clocks"],
            "status_ok": m["status_ok"], "generation_s": m["generation_s"]}
    if m["autotune"]:
        line["autotune"] = m["autotune"]
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
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the same-functor (calcNCC) and batched-pairs objects of the default line")
    ap.add_argument("--points-per-warp", type=int, default=0, help="0 = library choice")
    ap.add_argument("--ref-budget", type=float, default=2.0, help="seconds of CPU work per reference step")
    ap.add_argument("--small", action="store_true", help="3^8 grid (for profiling captures)")
    ap.add_argument("--grid-counts", default=None,
                    help="values per axis, comma-separated, in place of the workload's (profiling captures)")
    ap.add_argument("--per-sample-decisions", action="store_true",
                    help="ZNCC and MI on the per-sample decision kernel instead of the span kernels")
    ap.add_argument("--taps", default="auto", choices=["auto", "quad", "texture"],
                    help="tap source of the fast path (auto: the library's choice)")
    ap.add_argument("--workload", default="ncc", choices=["ncc", "mi", "sad", "batch"],
                    help="ncc: the headline 256^2 ZNCC pair; mi: 512^2 u8 MI pair; sad: 64^2 SAD pair; "
                         "batch: 64 uneven pairs in one batch launch")
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
    if args.grid_counts:
        pair.count[:] = [float(v) for v in args.grid_counts.split(",")]
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
                   quad_taps={"auto": None, "quad": True, "texture": False}[args.taps],
                   per_sample_decisions=args.per_sample_decisions)

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

    span_kernel = (((cost == "ZNCC" and args.taps != "texture") or (cost == "MI" and args.taps == "auto")) and
                   not args.per_sample_decisions and pair.fixed.shape[2] == 1)
    # ---- roofline of the dominant kernel (the search kernel; staging and the FP64 verification
    # pass are well under 1% of a call)
    traffic, traffic_src = (recorded_traffic(args.workload)
                            if ((args.workload == "ncc" and cost == "ZNCC") or (args.workload == "mi" and cost == "MI"))
                            and not args.small and not args.grid_counts and not args.per_sample_decisions
                            and args.taps == "auto" else (None, "no capture recorded for this configuration"))
    flops = FLOPS_PER_PIXEL_EVAL.get(cost, 36) * n * pix
    achieved = flops / (ms_per_step / 1e3) / 1e12
    props = torch.cuda.get_device_properties(dev)
    sm_max = clocks.get("sm_max_mhz") or 1965.0
    peak = props.multi_processor_count * 128 * 2 * sm_max * 1e6 / 1e12
    roofline = {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4),
                "traffic": traffic,
                "traffic_source": traffic_src,
                "peak_source": "nominal FP32 FMA rate: SMs x 128 lanes x 2 flops x max SM clock "
                               "(MEASURED_PEAKS.json holds HBM and bf16 tensor peaks only)",
                "flops_per_pixel_eval": FLOPS_PER_PIXEL_EVAL.get(cost, 36),
                "pixel_evals_per_s": n * pix / (ms_per_step / 1e3)}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded blob+sinusoid generator, seed "
                                                          f"{S.DEFAULT_SEED}+rank)",
            "config": {"workload": WORKLOADS[args.workload] + (" (3^8 grid)" if args.small else "") +
                                   (f" (grid {args.grid_counts})" if args.grid_counts else ""), "cost": cost,
                       "grid_points": n, "pixels": pix, "points_per_warp": args.points_per_warp or "tuned",
                       "taps": args.taps,
                       "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_total / args.steps},
            # per search: staging, (the span kernels' staging step,) search, verification band, re-scoring
            "gpu_launches": (5 if span_kernel else 4) * args.steps,
            "roofline": roofline,
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "argmin": {"index": r.index, "cost": r.cost, "params": [float(x) for x in r.params]},
            "fp64_verify": {"verified": r.verified, "candidates": r.candidates, "index_fp64": r.index_fp64,
                            "argmin_agrees": bool(r.valid and r.index == r.index_fp64), "cost_fp64": r.cost_fp64,
                            "err_fp64": r.err_fp64, "max_err_fp64": r.max_err_fp64,
                            "definition": "grid points within 2e-5 x max(1, |best|) of the FP32 minimum re-scored "
                                          "on the device with the reference's exact sampling and FP64 sums"}}
    reduced = args.small or bool(args.grid_counts)
    if world == 1 and args.workload == "ncc" and cost == "ZNCC" and not reduced and not args.no_extras:
        # the reference arm's functor (calcNCC, the reference's exact sampling) on the same pair and grid
        def step_ref():
            cgs.search("NCC_REF", mov, fix, grid, costs=costs, result=res, stream=stream)
        step_ref()
        ts = []
        for _ in range(3):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_ref()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        t_ref = statistics.median(ts)
        line["same_functor"] = {"cost": "NCC_REF", "sampling": "exact (the reference's operation sequence)",
                                "value": n / (t_ref / 1e3), "unit": UNIT, "ms_per_step": t_ref, "steps": 3,
                                "note": "the reference arm's functor (calcNCC) on the same pair and grid"}
        # the batched uneven pairs: one warm-up and one timed graph replay
        line["batch"] = measure_batch(dev, rank, world, args.pairs, steps=1, warmup=1)
        line["batch"]["workload"] = WORKLOADS["batch"]
        line["batch"].pop("autotune", None)
        # the learned proposal against the full grid (second half of the metric)
        if os.path.exists(PROPOSAL_CHECKPOINT):
            line["proposal"] = measure_proposal(dev)
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
