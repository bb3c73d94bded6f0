"""The learned proposal: a CNN (``cgs_net_*`` in libcgs_b200.so) that predicts where a pair's
grid-search argmin lies, the local grid it implies (``cgs_proposal_grid``), and the serving
path that searches that grid and falls back to the full grid when the proposal's best cost
is worse than a coarse probe of the full grid.

The reference has no learned component; its drivers search the full grid, optionally
shrinking the range around the argmin level by level (src/gpu/cudaGridSearch_main_mi.cu:
312-363).  Here the full grid stays the arbiter: labels are the full grid's own argmins, and a
pair whose proposal cannot beat the coarse probe is searched in full.

Parameters are exchanged in grid-range units: ``u = 2 (p - start) / (end - start) - 1`` per
axis (-1 at the grid's start, +1 at its end).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import check

N_OUT = 16


def _torch():
    import torch
    return torch


def _stream(stream) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream) if hasattr(s, "cuda_stream") else int(s)


def to_units(params, start, end) -> np.ndarray:
    """Parameters -> grid-range units (-1 .. 1 over [start, end]); collapsed axes give 0."""
    p, a, b = (np.asarray(v, np.float64) for v in (params, start, end))
    span = np.where(b != a, b - a, 1.0)
    return np.where(b != a, 2.0 * (p - a) / span - 1.0, 0.0)


def from_units(u, start, end) -> np.ndarray:
    u, a, b = (np.asarray(v, np.float64) for v in (u, start, end))
    return a + (u + 1.0) * 0.5 * (b - a)


class ProposalNet:
    """The proposal CNN on the current CUDA device (one ``cgs_net`` handle)."""

    def __init__(self, max_batch: int = 256, seed: int = 0):
        L = _abi.load()
        h = C.c_void_p(None)
        check(L.cgs_net_create(int(max_batch), int(seed), C.byref(h)))
        self._h = h
        self.max_batch = int(max_batch)
        self.n_params = int(L.cgs_net_param_count())

    # -- parameters
    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        check(_abi.load().cgs_net_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        check(_abi.load().cgs_net_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def grads(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        check(_abi.load().cgs_net_get_grads(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def save(self, path: str) -> None:
        np.savez_compressed(path, params=self.params())

    def load(self, path: str) -> None:
        self.set_params(np.load(path)["params"])

    # -- passes
    def forward(self, fixed, moving, stream=None):
        """fixed, moving: CUDA float32 tensors (n, side, side), side a multiple of 128.
        Returns a (n, 16) CUDA tensor: 8 centres then 8 log-radii (grid-range units)."""
        torch = _torch()
        n, side = int(fixed.shape[0]), int(fixed.shape[-1])
        out = torch.empty((n, N_OUT), dtype=torch.float32, device=fixed.device)
        check(_abi.load().cgs_net_forward(self._h, fixed.data_ptr(), moving.data_ptr(), n, side, out.data_ptr(),
                                          _stream(stream)))
        return out

    def backward(self, labels, stream=None):
        """Gradients of the mean loss for the last forward; labels (n, 8) CUDA float32.
        Returns the loss as a 1-element CUDA tensor."""
        torch = _torch()
        loss = torch.empty(1, dtype=torch.float32, device=labels.device)
        check(_abi.load().cgs_net_backward(self._h, labels.data_ptr(), loss.data_ptr(), _stream(stream)))
        return loss

    def adam_step(self, lr: float, stream=None) -> None:
        check(_abi.load().cgs_net_adam_step(self._h, float(lr), _stream(stream)))

    def train_step(self, fixed, moving, labels, lr: float, stream=None):
        self.forward(fixed, moving, stream)
        loss = self.backward(labels, stream)
        self.adam_step(lr, stream)
        return loss

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _abi.load().cgs_net_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def grid_window(full, first, count):
    """The window of `full` with count[a] values from index first[a] on each axis (a CudaGrid
    whose values are the full grid's)."""
    from . import CudaGrid
    f = (C.c_int32 * 8)(*[int(v) for v in first] + [0] * (8 - len(first)))
    c = (C.c_int32 * 8)(*[int(v) for v in count] + [1] * (8 - len(count)))
    g = CudaGrid(full.g.dims)
    check(_abi.load().cgs_grid_window(C.byref(full.g), f, c, C.byref(g.g)))
    return g


def proposal_window(full, out16, min_values: int = 3, max_values: int = 5):
    """(first, count) per axis of the window a proposal implies (cgs_proposal_window)."""
    o = (C.c_float * 16)(*[float(v) for v in np.asarray(out16, np.float32)])
    f, c = (C.c_int32 * 8)(), (C.c_int32 * 8)()
    check(_abi.load().cgs_proposal_window(C.byref(full.g), o, int(min_values), int(max_values), f, c))
    d = full.g.dims
    return np.array(list(f)[:d], np.int64), np.array(list(c)[:d], np.int64)


def proposal_grid(full, out16, min_values: int = 3, max_values: int = 5):
    """The local grid (a CudaGrid) of one proposal."""
    return grid_window(full, *proposal_window(full, out16, min_values, max_values))


def coarse_grid(full, values: int = 3):
    """A coarse probe of the full grid: on each axis `values` full-grid values a whole number of
    steps apart (indices 0, s, 2s, .. with s = (count - 1) // (values - 1)).  Its points are
    full-grid points, so its best cost bounds the full grid's best from above."""
    from . import CudaGrid
    d = full.g.dims
    counts = [int(full.g.count[a]) for a in range(d)]
    inc = np.cumprod([1] + counts[:-1])
    g = CudaGrid(d)
    for a in range(d):
        n = counts[a]
        k = max(1, min(values, n))
        step = (n - 1) // (k - 1) if k > 1 else 0
        g.g.start[a] = full.g.start[a]
        g.g.end[a] = float(full.getGridPoint(int((k - 1) * step * inc[a]))[a]) if k > 1 else full.g.start[a]
        g.g.count[a] = float(k)
    g.update()
    return g


@dataclass
class ServeResult:
    params: np.ndarray   # (n, 8) chosen grid points
    costs: np.ndarray    # (n,) their costs
    fallback: np.ndarray # (n,) True where the full grid was searched
    points: int          # grid points evaluated in total (proposal + probe + fallbacks)
    d2h_bytes: int = 0   # device-to-host bytes read back (network outputs, per-launch results)


def full_grid(side: int = 256, values: int = 6):
    """The full grid of the learned-proposal configuration at `side` pixels."""
    from . import CudaGrid
    from .synthetic import config4_ranges
    lo, hi = config4_ranges(side)
    return CudaGrid.from_ranges([float(v) for v in lo], [float(v) for v in hi], [values] * 8)


def _batch_search(cost, fixed, moving, grids, device, dump=None):
    """One batch launch over pairs i with grid grids[i]: (params (n, 8), costs (n,),
    valid (n,), points evaluated).  dump: indices of the pairs whose whole cost arrays are
    wanted; they are then returned as a fifth element (dict index -> numpy array)."""
    import torch
    from . import Batch, BatchPair, CudaImage, read_result
    # the results in one device block (one copy back), pair i's at bytes [i st, i st + rb), each
    # slot 128-byte aligned as a result buffer of its own would be
    rb = C.sizeof(_abi.CgsArgmin)
    st = (rb + 127) // 128 * 128
    block = torch.empty(len(grids) * st, dtype=torch.uint8, device=device)
    res = [block[i * st:i * st + rb] for i in range(len(grids))]
    dumps = {i: torch.empty(grids[i].numElements(), dtype=torch.float32, device=device) for i in (dump or ())}
    pairs = [BatchPair(cost, CudaImage(moving[i]), CudaImage(fixed[i]), g, res[i], dumps.get(i))
             for i, g in enumerate(grids)]
    with Batch(pairs) as b:
        b.launch()
        torch.cuda.synchronize(device)
    host = block.cpu()
    out = [read_result(host[i * st:i * st + rb]) for i in range(len(grids))]
    params = np.stack([o.params for o in out]).astype(np.float64)
    costs = np.array([o.cost for o in out], np.float64)
    valid = np.array([o.valid and o.status == 0 for o in out])
    pts = int(sum(g.numElements() for g in grids))
    if dump is not None:
        return params, costs, valid, pts, {i: t.cpu().numpy() for i, t in dumps.items()}
    return params, costs, valid, pts


def grid_argmins(fixed, moving, grid, cost: str = "ZNCC", chunk: int = 256):
    """The grid-search argmin of every pair (the full grid's answer), in chunks of pairs per
    batch launch.  fixed, moving: CUDA float32 (n, side, side).  Returns (params, costs)."""
    n = int(fixed.shape[0])
    ps, cs = [], []
    for i in range(0, n, chunk):
        j = min(n, i + chunk)
        p, c, _, _ = _batch_search(cost, fixed[i:j], moving[i:j], [grid] * (j - i), fixed.device)
        ps.append(p)
        cs.append(c)
    return np.concatenate(ps), np.concatenate(cs)


def _axis_indices(index: int, counts) -> np.ndarray:
    """Per-axis indices of a flat grid index (axis 0 fastest)."""
    out = []
    for c in counts:
        out.append(index % c)
        index //= c
    return np.array(out, np.int64)


def serve(net: ProposalNet, fixed, moving, full, cost: str = "ZNCC", min_values: int = 3, max_values: int = 5,
          probe_values: int = 3, walks: int = 6, starts: int = 2) -> ServeResult:
    """The learned-proposal path for a batch of pairs.

    1. The network proposes a window of the full grid per pair (cgs_proposal_window).  One
       batch launch searches every pair's window and a coarse probe of the full grid
       (full-grid points, so its best bounds the full grid's best from above).
    2. With starts = k > 1, k - 1 more walkers per pair start from min_values-wide windows
       centred on the probe's k - 1 best points.
    3. A walker whose window's best lies strictly inside the window on every axis (or on a
       window edge that is the grid's edge) stops there: a certified local minimum of the grid.
       A best on an inner window edge moves the window to centre on it, at most `walks` times.
       Every pass over the pending walkers of all pairs is one batch launch.
    4. A pair's answer is the best certified point (or the probe's best, if lower); a pair
       without any certified point is searched on the full grid (the fallback)."""
    n = int(fixed.shape[0])
    d = full.g.dims
    counts = np.array([int(c) for c in full.getAxisSampleCounts()], np.int64)
    step = int(getattr(net, "max_batch", n) or n)
    out = np.concatenate([net.forward(fixed[i:i + step], moving[i:i + step]).cpu().numpy()
                          for i in range(0, n, step)])
    probe = coarse_grid(full, probe_values)
    params = np.zeros((n, d))
    costs = np.full(n, np.inf)
    certified = np.zeros(n, bool)
    # walkers: [pair, first, count, walks left]
    walkers = [[i, *proposal_window(full, out[i], min_values, max_values), walks] for i in range(n)]
    start = np.array([full.g.start[a] for a in range(d)], np.float64)
    fres = np.array([full.g.resolution[a] for a in range(d)], np.float64)
    pts = 0
    first_pass = True
    while walkers:
        grids = [grid_window(full, w[1], w[2]) for w in walkers]
        idx = [w[0] for w in walkers]
        if first_pass:
            grids += [probe] * n
            idx += list(range(n))
        nw = len(walkers)
        if first_pass and starts > 1:
            p, c, v, k, dumps = _batch_search(cost, fixed[idx], moving[idx], grids, fixed.device,
                                              dump=range(nw, nw + n))
        else:
            p, c, v, k = _batch_search(cost, fixed[idx], moving[idx], grids, fixed.device)
        pts += k
        nxt = []
        for j in range(nw):
            i, first, cnt, left = walkers[j]
            if not v[j]:
                continue
            if c[j] < costs[i]:
                params[i], costs[i] = p[j], c[j]
            g = grids[j]
            lo = np.array([g.g.start[a] for a in range(d)], np.float64)
            res = np.array([g.g.resolution[a] for a in range(d)], np.float64)
            loc = np.where(cnt > 1, np.rint((p[j] - lo) / np.where(res != 0, res, 1.0)), 0).astype(np.int64)
            on_edge = ((loc == 0) & (first > 0)) | ((loc == cnt - 1) & (first + cnt < counts))
            if not on_edge.any():
                certified[i] = True
            elif left > 0:
                nxt.append([i, np.clip(first + loc - (cnt - 1) // 2, 0, counts - cnt), cnt, left - 1])
        if first_pass:
            pp, pc, pv = p[nw:], c[nw:], v[nw:]
            for i in range(n):
                if pv[i] and pc[i] < costs[i]:
                    params[i], costs[i] = pp[i], pc[i]
            if starts > 1:
                # the probe's best points (lowest index first on ties), as full-grid indices
                width = np.minimum(min_values, counts)
                pcounts = np.array([int(cc) for cc in probe.getAxisSampleCounts()], np.int64)
                pstep = np.where(pcounts > 1, (counts - 1) // np.maximum(pcounts - 1, 1), 0)
                for i in range(n):
                    pd = dumps[nw + i]
                    cand = np.where(np.isfinite(pd), pd, np.inf)
                    order = np.argsort(cand, kind="stable")[: starts - 1]
                    for q in order:
                        if not np.isfinite(cand[q]):
                            break
                        centre = _axis_indices(int(q), pcounts) * pstep
                        nxt.append([i, np.clip(centre - (width - 1) // 2, 0, counts - width), width.copy(), walks])
            first_pass = False
        walkers = nxt
    fallback = ~certified
    if fallback.any():
        fi = np.flatnonzero(fallback)
        pf, cf, _, k = _batch_search(cost, fixed[fi], moving[fi], [full] * len(fi), fixed.device)
        pts += k
        params[fi], costs[fi] = pf, cf
    return ServeResult(params, costs, fallback, pts)


def refine_serve(net: ProposalNet, fixed, moving, full, cost: str = "ZNCC", values: int = 3, levels: int = 4,
                 spread: float = 2.0, min_half: float = 0.02, probe_values: int = 3, walks: int = 2,
                 start=None) -> ServeResult:
    """The learned proposal with local refinement grids (the configuration's local grid around
    the proposal), for a batch of pairs.

    1. The network's centre and radii (grid-range units) give each pair a local grid of `values`
       values per axis over centre +- spread x radius (at least min_half of the range, clipped
       to the full grid's range).  One batch launch searches every pair's local grid and a
       coarse probe of the full grid (`probe_values` full-grid values per axis).
    2. Coarse to fine, as the reference's driver loop (src/gpu/cudaGridSearch_main_mi.cu:
       312-363): each further launch re-centres every pair's grid on its best point with half the
       range, `levels` times; a best point on an edge of the local grid that is not the full
       grid's edge re-centres it without halving (at most `walks` times per pair).
    3. A pair's answer is its best refined point; where that costs more than the probe's best
       the pair is searched on the full grid instead (the fallback).
    The refined points lie between the full grid's values, so the answer can be closer to the
    true registration than the full grid's own argmin.  start: (n, 8) parameters that replace
    the network's centres, with min_half as the first half-range (an experiment's control: the
    refinement started at the generator's ground truth)."""
    from . import CudaGrid
    n = int(fixed.shape[0])
    d = full.g.dims
    lo = np.array([full.g.start[a] for a in range(d)], np.float64)
    hi = np.array([full.g.end[a] for a in range(d)], np.float64)
    step = int(getattr(net, "max_batch", n) or n)
    out = np.concatenate([net.forward(fixed[i:i + step], moving[i:i + step]).cpu().numpy()
                          for i in range(0, n, step)]).astype(np.float64)
    centre = from_units(np.clip(out[:, :d], -1.0, 1.0), lo, hi)
    half = np.clip(spread * np.exp(np.clip(out[:, 8:8 + d], -12.0, 4.0)), min_half, 1.0) * (hi - lo) / 2.0
    if start is not None:
        centre = np.asarray(start, np.float64)[:, :d]
        half = np.full((n, d), min_half) * (hi - lo) / 2.0

    def local(c, h):
        a, b = np.maximum(lo, c - h), np.minimum(hi, c + h)
        return CudaGrid.from_ranges(a, np.where(b > a, b, a), np.where(b > a, float(values), 1.0))

    probe = coarse_grid(full, probe_values)
    params = np.zeros((n, d))
    costs = np.full(n, np.inf)
    grids = [local(centre[i], half[i]) for i in range(n)]
    rbytes = C.sizeof(_abi.CgsArgmin)
    d2h = out.size * 4 + 2 * n * rbytes
    p, c, v, pts = _batch_search(cost, fixed[np.r_[0:n, 0:n]], moving[np.r_[0:n, 0:n]], grids + [probe] * n,
                                 fixed.device)
    probe_cost = np.where(v[n:], c[n:], np.inf)
    left_levels = np.full(n, levels)
    left_walks = np.full(n, walks)

    def grid_rows(gs):
        # each grid's start, resolution and sample counts as the library computed them
        starts = np.array([g.g.start[:d] for g in gs], np.float64)
        steps = np.array([g.g.resolution[:d] for g in gs], np.float64)
        counts = np.array([g.g.count[:d] for g in gs], np.float64).astype(np.int64)
        return starts, steps, counts

    active = np.arange(n)
    cur_p, cur_c, cur_v = p[:n], c[:n], v[:n]
    ga, gr, gc = grid_rows(grids)
    span = hi - lo
    while True:
        # every active pair at once: keep its best point, then walk (best point on an inner
        # edge of its local grid), halve (levels left) or stop
        better = cur_v & (cur_c < costs[active])
        params[active[better]] = cur_p[better]
        costs[active[better]] = cur_c[better]
        alive = cur_v & np.isfinite(costs[active])
        loc = np.where(gc > 1, np.rint((params[active] - ga) / np.where(gr != 0, gr, 1.0)), 0).astype(np.int64)
        edge = ((loc == 0) & (ga > lo + 1e-9 * span)) | ((loc == gc - 1) & (ga + gr * (gc - 1) < hi - 1e-9 * span))
        walk = alive & edge.any(axis=1) & (left_walks[active] > 0)
        halve = alive & ~walk & (left_levels[active] > 0)
        left_walks[active[walk]] -= 1
        left_levels[active[halve]] -= 1
        half[active[halve]] = half[active[halve]] / 2.0
        nxt = active[walk | halve]
        if not nxt.size:
            break
        ngrids = [local(params[i], half[i]) for i in nxt]
        active = nxt
        cur_p, cur_c, cur_v, k = _batch_search(cost, fixed[active], moving[active], ngrids, fixed.device)
        ga, gr, gc = grid_rows(ngrids)
        pts += k
        d2h += len(ngrids) * rbytes
    fallback = ~(costs <= probe_cost)
    if fallback.any():
        fi = np.flatnonzero(fallback)
        pf, cf, _, k = _batch_search(cost, fixed[fi], moving[fi], [full] * len(fi), fixed.device)
        pts += k
        d2h += len(fi) * rbytes
        params[fi], costs[fi] = pf, cf
    return ServeResult(params, costs, fallback, pts, d2h)


def corner_error(p_a, p_b, side: int = 256) -> np.ndarray:
    """Mean distance (px) between the image corners mapped by the homographies of parameter
    vectors p_a and p_b (centred parametrisation at side / 2), per row."""
    from .synthetic import homography
    pa, pb = np.atleast_2d(p_a), np.atleast_2d(p_b)
    corners = np.array([[0, 0, 1], [side - 1, 0, 1], [0, side - 1, 1], [side - 1, side - 1, 1]], np.float64).T
    out = []
    for a, b in zip(pa, pb):
        qa = homography(a, "centred", side / 2.0, side / 2.0) @ corners
        qb = homography(b, "centred", side / 2.0, side / 2.0) @ corners
        qa, qb = qa[:2] / qa[2], qb[:2] / qb[2]
        out.append(float(np.mean(np.hypot(*(qa - qb)))))
    return np.array(out)


def downsample(x, s: int):
    """s x s box average of a (n, side, side) CUDA stack (the network's own input rule)."""
    import torch
    n, h, w = x.shape
    return x.reshape(n, h // s, s, w // s, s).mean(dim=(2, 4)).contiguous()


def train(net: ProposalNet, fixed, moving, labels_u, epochs: int, batch: int = 256, lr: float = 1e-3,
          seed: int = 0, log=None) -> list[float]:
    """Adam on the Laplace loss over (fixed, moving, labels) CUDA tensors; returns per-epoch
    mean losses."""
    import torch
    n = int(fixed.shape[0])
    g = torch.Generator(device="cpu").manual_seed(seed)
    lab = torch.as_tensor(np.asarray(labels_u, np.float32), device=fixed.device)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(fixed.device)
        tot = torch.zeros(1, device=fixed.device)
        steps = 0
        for i in range(0, n - batch + 1, batch):
            ix = perm[i:i + batch]
            tot += net.train_step(fixed[ix].contiguous(), moving[ix].contiguous(), lab[ix].contiguous(), lr)
            steps += 1
        hist.append(float(tot) / max(1, steps))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.4f}")
    return hist


def experiment(n_train: int, n_eval: int, epochs: int, seed: int, out_dir: str, label_side: int = 128,
               min_values: int = 3, max_values: int = 5, batch: int = 256, checkpoint: str | None = None,
               variants=None, init: str | None = None, labels: str = "grid", lr: float = 1e-3,
               full_grid_cache: str | None = None, mode: str = "lattice", scene: bool = False, log=print) -> dict:
    """The learned-proposal configuration end to end on the current GPU: generate training pairs
    (256 px), label them -- labels="grid": the full 6^8 ZNCC grid's argmin on the pairs box-averaged
    to label_side; labels="truth": the generator's ground-truth parameters, no search -- train, then
    on held-out 256 px pairs compare the served proposal path with the full grid (the arbiter):
    corner error, cost gap, fallback rate and pairs/s of both (CUDA events).  full_grid_cache: an .npz
    holding the full grid's argmins of the same held-out pairs (written here when absent); with
    it, the full grid is timed on the first 64 pairs only."""
    import json
    import os
    import time

    import torch
    dev = torch.device("cuda")
    os.makedirs(out_dir, exist_ok=True)
    t0 = time.time()
    full_l = full_grid(label_side, 6)
    lo_l, hi_l = full_l.matrix()[0], full_l.matrix()[1]
    fs, ms, us = [], [], []
    s = 256 // label_side
    chunk = 512
    t_label = 0.0
    net = ProposalNet(max_batch=batch, seed=seed)
    hist, t_train = [float("nan")], 0.0
    if checkpoint:  # a network trained earlier on the same generator: evaluation only
        net.load(checkpoint)
        n_train = 0
    elif init:  # start training from these parameters
        net.load(init)
    lo_e, hi_e = full_grid(256, 6).matrix()[0], full_grid(256, 6).matrix()[1]
    for i in range(0, n_train, chunk):
        k = min(chunk, n_train - i)
        f, m, gt = config4_batch_cached(seed + i, k, dev, scene)
        fd, md = downsample(f, s), downsample(m, s)
        torch.cuda.synchronize()
        if labels == "truth":
            us.append(to_units(gt.numpy(), lo_e, hi_e).astype(np.float32))
        else:
            tl = time.time()
            p, _ = grid_argmins(fd, md, full_l)
            t_label += time.time() - tl
            us.append(to_units(p, lo_l, hi_l).astype(np.float32))
        fs.append(fd)
        ms.append(md)
        if (i // chunk) % 16 == 0 or i + k == n_train:
            log(f"labelled {i + k}/{n_train} ({t_label:.0f} s in the grid search)")
    ckpt = checkpoint
    if n_train:
        F, M, U = torch.cat(fs), torch.cat(ms), np.concatenate(us)
        del fs, ms
        np.save(os.path.join(out_dir, "labels.npy"), U)
        tt = time.time()
        hist = train(net, F, M, U, epochs=epochs, batch=batch, lr=lr, seed=seed, log=log)
        torch.cuda.synchronize()
        t_train = time.time() - tt
        ckpt = os.path.join(out_dir, "proposal_net.npz")
        net.save(ckpt)
        del F, M
    # evaluation at 256 px: the full grid (the arbiter) once, then each serving variant
    full = full_grid(256, 6)
    fe, me, gte = config4_batch_cached(seed + 10 ** 7, n_eval, dev, scene)
    ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cached = None
    if full_grid_cache and os.path.exists(full_grid_cache):
        z = np.load(full_grid_cache)
        if int(z["n_eval"]) == n_eval and int(z["seed"]) == seed and bool(z.get("scene", False)) == scene:
            cached = z
    if cached is not None:
        truth, tcost = cached["truth"], cached["cost"]
        k = min(64, n_eval)
        ev[0].record()
        grid_argmins(fe[:k], me[:k], full)
        ev[1].record()
        torch.cuda.synchronize()
        t_full = ev[0].elapsed_time(ev[1]) / 1e3 * n_eval / k
    else:
        ev[0].record()
        truth, tcost = grid_argmins(fe, me, full)
        ev[1].record()
        torch.cuda.synchronize()
        t_full = ev[0].elapsed_time(ev[1]) / 1e3
        if full_grid_cache:
            np.savez(full_grid_cache, truth=truth, cost=tcost, n_eval=n_eval, seed=seed, scene=scene)
    # how often the label resolution's argmin is the evaluation resolution's
    lab_e, _ = grid_argmins(downsample(fe, 256 // label_side), downsample(me, 256 // label_side), full_l)
    same = np.all(np.isclose(to_units(lab_e, lo_l, hi_l), to_units(truth, full.matrix()[0], full.matrix()[1]),
                             atol=1e-4), axis=1)
    res = {"n_train": n_train, "n_eval": n_eval, "epochs": epochs, "label_side": label_side, "labels": labels,
           "scene": scene,
           "label_matches_eval_argmin": float(same.mean()), "loss_first": hist[0], "loss_last": hist[-1],
           "label_seconds": round(t_label, 1), "train_seconds": round(t_train, 1),
           "full_grid_pairs_per_s": n_eval / t_full,
           "gt_corner_error_full_grid_px": float(corner_error(truth, gte.numpy(), 256).mean()),
           "mode": mode,
           "checkpoint": ckpt, "variants": []}
    for var in variants or [(min_values, max_values, 6, 2)]:
        if mode == "refine":
            vals, lev, spread, mh, walks = var[:5]
            kw = dict(values=int(vals), levels=int(lev), spread=float(spread), min_half=float(mh), walks=int(walks))
            fn, desc = refine_serve, {"mode": "refine", **kw}
            if len(var) > 5 and var[5]:  # control: refinement started at the ground truth
                gt_np = gte.numpy()
                desc["start"] = "ground truth"
                fn = (lambda net_, f_, m_, full_, **k_: refine_serve(
                    net_, f_, m_, full_, start=gt_np[:f_.shape[0]], **k_))
        else:
            mn, mx, walks, starts = var
            kw = dict(min_values=mn, max_values=mx, walks=walks, starts=starts)
            fn, desc = serve, {"mode": "lattice", **kw}
        fn(net, fe[:8], me[:8], full, **kw)  # warm-up
        ev[0].record()
        r = fn(net, fe, me, full, **kw)
        ev[1].record()
        torch.cuda.synchronize()
        t_serve = ev[0].elapsed_time(ev[1]) / 1e3
        err = corner_error(r.params, truth, 256)
        gap = r.costs - tcost
        gerr = corner_error(r.params, gte.numpy(), 256)
        perr = np.abs(to_units(r.params, full.matrix()[0], full.matrix()[1]) -
                      to_units(gte.numpy(), full.matrix()[0], full.matrix()[1])).mean(axis=0)
        res["variants"].append({
            **desc, "proposal_pairs_per_s": n_eval / t_serve, "speedup": t_full / t_serve,
            "gt_corner_error_mean_px": float(gerr.mean()), "gt_corner_error_p90_px": float(np.percentile(gerr, 90)),
            "cost_not_above_full_grid": float(np.mean(gap <= 0.0)),
            "gt_param_error_units": [round(float(v), 5) for v in perr],
            "fallback_rate": float(r.fallback.mean()), "corner_error_mean_px": float(err.mean()),
            "corner_error_p90_px": float(np.percentile(err, 90)), "agree_within_0_5px": float(np.mean(err <= 0.5)),
            "cost_gap_mean": float(np.mean(gap)), "cost_gap_max": float(np.max(gap)),
            "points_fraction": r.points / (n_eval * full.numElements())})
        log(json.dumps(res["variants"][-1]))
    res["wall_seconds"] = round(time.time() - t0, 1)
    with open(os.path.join(out_dir, "proposal_eval.json"), "w") as fh:
        json.dump(res, fh, indent=1)
    net.close()
    return res


def config4_batch_cached(seed: int, n: int, device, scene: bool = False):
    """config4_batch in chunks of at most 256 pairs (bounded generator memory)."""
    import torch
    from .synthetic import config4_batch
    fs, ms, gs = [], [], []
    for i in range(0, n, 256):
        f, m, g = config4_batch(seed + i, min(256, n - i), device, scene=scene)
        fs.append(f)
        ms.append(m)
        gs.append(g)
    return torch.cat(fs), torch.cat(ms), torch.cat(gs)


def forward_timing(batch: int = 256, reps: int = 20, seed: int = 7) -> dict:
    """Forward passes and training steps of the network on random 128 x 128 pairs (CUDA events,
    after warm-up): the ms per forward and per training step at `batch` pairs."""
    import torch
    dev = torch.device("cuda")
    g = torch.Generator(device="cpu").manual_seed(seed)
    f = (torch.rand(batch, 128, 128, generator=g) * 255).to(dev).contiguous()
    m = (torch.rand(batch, 128, 128, generator=g) * 255).to(dev).contiguous()
    lab = (torch.rand(batch, 8, generator=g) * 2 - 1).to(dev).contiguous()
    net = ProposalNet(max_batch=batch, seed=seed)
    try:
        for _ in range(3):
            net.forward(f, m)
        ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev[0].record()
        for _ in range(reps):
            net.forward(f, m)
        ev[1].record()
        ev[1].synchronize()
        fwd = ev[0].elapsed_time(ev[1]) / reps
        ev[0].record()
        for _ in range(reps):
            net.train_step(f, m, lab, 1e-6)
        ev[1].record()
        ev[1].synchronize()
        step = ev[0].elapsed_time(ev[1]) / reps
        net.params()  # raises if a tensor-core pass gave up waiting
    finally:
        net.close()
    return {"batch": batch, "forward_ms": fwd, "train_step_ms": step}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train and evaluate the learned proposal (one GPU)")
    ap.add_argument("--train", type=int, default=8192)
    ap.add_argument("--eval", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--out", default="proposal_run")
    ap.add_argument("--min-values", type=int, default=3)
    ap.add_argument("--max-values", type=int, default=5)
    ap.add_argument("--checkpoint", default=None, help="evaluate this trained network instead of training")
    ap.add_argument("--init", default=None, help="start training from this network's parameters")
    ap.add_argument("--label-side", type=int, default=128, help="image side the labels are searched at")
    ap.add_argument("--mode", default="lattice", choices=["lattice", "refine"],
                    help="lattice: walkers on windows of the full grid; refine: coarse-to-fine local grids")
    ap.add_argument("--variants", default=None,
                    help="serving variants separated by ';': lattice min_values,max_values,walks,starts; "
                         "refine values,levels,spread,min_half,walks")
    ap.add_argument("--labels", default="grid", choices=["grid", "truth"],
                    help="grid: full-grid argmins at --label-side; truth: the generator's parameters")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--scene", action="store_true",
                    help="moving images see the fixed image's mirror continuation past its edges (no black borders)")
    ap.add_argument("--full-grid-cache", default=None,
                    help=".npz of the full grid's argmins of the held-out pairs (reused when it matches --eval "
                         "and --seed, else written)")
    ap.add_argument("--net-timing", action="store_true",
                    help="only time the network's forward pass and training step on random pairs")
    a = ap.parse_args()
    if a.net_timing:
        print(json.dumps(forward_timing()))
        raise SystemExit(0)
    spec = a.variants or ("3,3,6,1;3,3,6,2;3,5,6,1;3,5,6,2" if a.mode == "lattice" else "3,4,2,0.02,2;3,5,2,0.02,2")
    vs = [tuple(float(x) for x in v.split(",")) for v in spec.split(";") if v]
    if a.mode == "lattice":
        vs = [tuple(int(x) for x in v) for v in vs]
    print(json.dumps(experiment(a.train, a.eval, a.epochs, a.seed, a.out, label_side=a.label_side,
                                min_values=a.min_values, max_values=a.max_values, checkpoint=a.checkpoint,
                                variants=vs, init=a.init, labels=a.labels, lr=a.lr,
                                full_grid_cache=a.full_grid_cache, mode=a.mode, scene=a.scene)))
