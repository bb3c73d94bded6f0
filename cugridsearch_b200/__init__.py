"""cugridsearch_b200 -- B200 (sm_100a) homography grid search behind the cuGridSearch API.

The compute runs in ``libcgs_b200.so`` (hand-written CUDA for sm_100a, C ABI in
``include/cugridsearch_b200.h``).  This module is the Python host mirror of the
reference's template API (``src/gpu/cudaGridSearch.cuh``, ``include/cudaTensor.cuh``):

=========================================  ===============================================
reference                                  here
=========================================  ===============================================
``CudaGrid<float, D>`` + setters           :class:`CudaGrid`
``CudaImage<T, C>`` (caller-owned data)     :class:`CudaImage` (wraps a CUDA tensor)
``CudaTensor<float, D>`` result + find_extrema  :class:`CudaTensor`
``CudaGridSearcher<F, G, D>::search*``      :class:`CudaGridSearcher`
device functor pointer (``calcNCC`` ...)    cost names: :data:`calcNCC` etc.
=========================================  ===============================================

Device memory and streams come from PyTorch tensors; nothing here computes a cost.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import COSTS, CgsArgmin, CgsBatchPlan, CgsError, CgsGrid, CgsImage, CgsOptions, CgsPair, CgsTuneEntry, check

__all__ = [
    "CudaGrid", "CudaImage", "CudaTensor", "CudaGridSearcher", "Argmin", "search", "argmin",
    "COSTS", "CgsError", "library", "refine", "homography", "transform_image", "fuse_aligned",
    "filter_image", "quantize_image", "averageAbsoluteDifference", "averageAbsoluteDifferenceH",
    "sumOfAbsoluteDifferences", "sumOfAbsoluteDifferences_by_reference", "calcSQD", "calcNCC",
    "calcSQDAlt", "calcNCCAlt", "calcMIAlt", "ZNCC", "MI", "Batch", "BatchPair", "BatchPlan",
]

# Cost selectors named after the reference functors (the device function pointer the
# reference passes to search_by_value).
averageAbsoluteDifference = "SAD_AVG"          # cudaErrorFunctions.cuh:31-87
averageAbsoluteDifferenceH = "SAD_AVG_H"       # cudaErrorFunctions.cuh:194-224
sumOfAbsoluteDifferences = "SAD_SUM_T"         # cudaErrorFunctions.cuh:89-114 (by value)
sumOfAbsoluteDifferences_by_reference = "SAD_SUM_T_REF"  # cudaErrorFunctions.cuh:171-192
calcSQD = "SQD_REF"                            # cudaErrorFunctions.cuh:378-446
calcNCC = "NCC_REF"                            # cudaErrorFunctions.cuh:448-507
calcSQDAlt = "SQD_ALT"                         # cudaErrorFunctions.cuh:226-300
calcNCCAlt = "NCC_ALT"                         # cudaErrorFunctions.cuh:302-376
calcMIAlt = "MI_ALT"                           # cudaErrorFunction_mi.cuh:117-255
ZNCC = "ZNCC"
MI = "MI"


def library() -> C.CDLL:
    return _abi.load()


def _torch():
    import torch  # device memory and streams only
    return torch


def _stream_handle(stream) -> int:
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)


@dataclass
class Argmin:
    """A search's result (cgs_argmin): the FP32 argmin and, from the FP64 verification pass, the
    FP64 cost of that index, its error, the FP64 argmin among the re-scored band and the largest
    FP32 - FP64 difference there (verified = number of points re-scored; 0: no pass ran)."""
    cost: float
    index: int
    params: np.ndarray
    valid: bool
    status: int = 0
    verified: int = 0
    candidates: int = 0
    index_fp64: int = -1
    cost_fp64: float = float("nan")
    err_fp64: float = float("nan")
    max_err_fp64: float = 0.0

    @staticmethod
    def from_struct(r: CgsArgmin) -> "Argmin":
        return Argmin(float(r.cost), int(r.index), np.array(list(r.params), dtype=np.float32), bool(r.valid),
                      int(r.status), int(r.verified), int(r.candidates), int(r.index_fp64), float(r.cost_fp64),
                      float(r.err_fp64), float(r.max_err_fp64))


class CudaGrid:
    """CudaGrid<float, D> (src/gpu/cudaGridSearch.cuh:74-231): rows {start, end,
    resolution, count}; every setter calls update() as the reference's do (:198-215)."""

    def __init__(self, dims: int = 8):
        if not 1 <= dims <= 8:
            raise ValueError("dims must be 1..8")
        self.g = CgsGrid()
        self.g.dims = dims
        for a in range(8):
            self.g.count[a] = 1.0

    @classmethod
    def from_ranges(cls, start, end, count) -> "CudaGrid":
        """setStartPoint, setEndPoint, setNumSamples.  Each setter's update recomputes every axis
        from its start, end and count alone, and the counts are set last, so one update after
        all three rows leaves the same grid as the three updates."""
        g = cls(len(start))
        d = g.g.dims
        for row, vals in ((g.g.start, start), (g.g.end, end), (g.g.count, count)):
            if len(vals) != d:
                raise ValueError(f"expected {d} values")
            row[:d] = np.asarray(vals, np.float64).astype(np.float32).tolist()  # rounded to FP32 as the setters do
        g.update()
        return g

    def getDimension(self) -> int:
        return int(self.g.dims)

    def _set_row(self, row, vals):
        if len(vals) != self.g.dims:
            raise ValueError(f"expected {self.g.dims} values")
        for a, v in enumerate(vals):
            row[a] = float(np.float32(v))
        self.update()

    def setStartPoint(self, vals):
        self._set_row(self.g.start, vals)

    def setEndPoint(self, vals):
        self._set_row(self.g.end, vals)

    def setNumSamples(self, vals):
        self._set_row(self.g.count, vals)

    def update(self, changed_axis: int = -1):
        check(_abi.load().cgs_grid_update(C.byref(self.g), changed_axis))

    def getAxisSampleCounts(self) -> np.ndarray:
        return np.array(list(self.g.count)[: self.g.dims], dtype=np.float32)

    def resolution(self) -> np.ndarray:
        return np.array(list(self.g.resolution)[: self.g.dims], dtype=np.float32)

    def numElements(self) -> int:
        n = C.c_uint64(0)
        check(_abi.load().cgs_grid_num_elements(C.byref(self.g), C.byref(n)))
        return int(n.value)

    def getGridPoint(self, index: int) -> np.ndarray:
        out = (C.c_float * 8)()
        check(_abi.load().cgs_grid_point(C.byref(self.g), int(index), out))
        return np.array(list(out)[: self.g.dims], dtype=np.float32)

    def matrix(self) -> np.ndarray:
        """The 4 x D device matrix layout of the reference (rows start/end/res/count)."""
        d = self.g.dims
        return np.array([list(self.g.start)[:d], list(self.g.end)[:d], list(self.g.resolution)[:d],
                         list(self.g.count)[:d]], dtype=np.float32)


class CudaImage:
    """CudaImage<T, C> (include/cudaTensor.cuh:507-596) over a caller-owned CUDA tensor of
    shape (H, W) or (H, W, C), dtype float32, uint8, float64 or uint16, HWC row-major."""

    def __init__(self, tensor):
        torch = _torch()
        if not isinstance(tensor, torch.Tensor) or not tensor.is_cuda:
            raise TypeError("CudaImage wraps a CUDA tensor (device memory is caller-owned)")
        if tensor.dim() == 2:
            tensor = tensor.unsqueeze(-1)
        if tensor.dim() != 3 or not tensor.is_contiguous():
            raise ValueError("expected a contiguous (H, W) or (H, W, C) tensor")
        pix = {torch.float32: _abi.PIXEL_F32, torch.uint8: _abi.PIXEL_U8, torch.float64: _abi.PIXEL_F64,
               torch.uint16: _abi.PIXEL_U16}.get(tensor.dtype)
        if pix is None:
            raise TypeError("pixel type must be float32, uint8, float64 or uint16")
        self.tensor = tensor
        h, w, c = tensor.shape
        self.img = CgsImage(tensor.data_ptr(), h, w, c, pix)

    def height(self) -> int:
        return int(self.img.height)

    def width(self) -> int:
        return int(self.img.width)

    def channels(self) -> int:
        return int(self.img.channels)


class CudaTensor:
    """CudaTensor<float, D> result tensor (include/cudaTensor.cuh:108-361) on a CUDA tensor."""

    def __init__(self, tensor):
        torch = _torch()
        if tensor.dtype != torch.float32 or not tensor.is_cuda or not tensor.is_contiguous():
            raise TypeError("expected a contiguous float32 CUDA tensor")
        self.tensor = tensor

    def size(self) -> int:
        return int(self.tensor.numel())

    def find_extrema(self, stream=None) -> tuple[float, int]:
        """find_extrema (include/cudaTensor.cuh:215-265): (min value, flat index)."""
        torch = _torch()
        out = torch.empty(C.sizeof(CgsArgmin), dtype=torch.uint8, device=self.tensor.device)
        s = _stream_handle(stream)
        check(_abi.load().cgs_argmin_f32(self.tensor.data_ptr(), self.tensor.numel(), out.data_ptr(), s))
        host = out.cpu().numpy().tobytes()
        r = CgsArgmin.from_buffer_copy(host)
        return float(r.cost), int(r.index)


def _options(cost: str, mi_bins: int = 0, overlap_gate: float = 0.0, points_per_warp: int = 0,
             warps_per_block: int = 0, natural_order: bool = False, exact_samples: bool | None = None,
             quad_taps: bool | None = None, per_sample_decisions: bool = False, verify: bool = True) -> CgsOptions:
    if cost not in COSTS:
        raise ValueError(f"unknown cost {cost!r}")
    flags = _abi.FLAG_NATURAL_ORDER if natural_order else 0
    if not verify:
        flags |= _abi.FLAG_NO_VERIFY
    if per_sample_decisions:
        flags |= _abi.FLAG_PER_SAMPLE_DECISIONS
    if quad_taps is True:
        flags |= _abi.FLAG_QUAD_TAPS
    elif quad_taps is False:
        flags |= _abi.FLAG_TEXTURE_TAPS
    if exact_samples is True:
        flags |= _abi.FLAG_EXACT_SAMPLES
    elif exact_samples is False:
        flags |= _abi.FLAG_FAST_SAMPLES
    return CgsOptions(COSTS[cost], mi_bins, overlap_gate, points_per_warp, warps_per_block, flags)


def search(cost: str, moving: CudaImage, fixed: CudaImage, grid: CudaGrid, costs=None, stream=None,
           mi_bins: int = 0, overlap_gate: float = 0.0, points_per_warp: int = 0, warps_per_block: int = 0,
           natural_order: bool = False, exact_samples: bool | None = None, result=None,
           quad_taps: bool | None = None, per_sample_decisions: bool = False, verify: bool = True) -> Argmin | None:
    """Run one fused search.  With ``result`` (a CUDA uint8 tensor of sizeof(cgs_argmin)
    bytes) the call is asynchronous and returns None; otherwise it synchronises and
    returns the :class:`Argmin`.  ``exact_samples``: None = the cost's default (exact for
    the reference functors, fast for ZNCC / MI), True / False force a mode.  ``quad_taps``:
    None = the library's choice, True = pre-gathered 16-byte quads, False = texture gathers.
    ``per_sample_decisions``: run single-channel ZNCC and MI on the per-sample decision kernel
    instead of the span kernels (CGS_FLAG_PER_SAMPLE_DECISIONS).  ``verify``: run the FP64 verification pass
    (the Argmin's *_fp64 fields); False sets CGS_FLAG_NO_VERIFY."""
    opt = _options(cost, mi_bins, overlap_gate, points_per_warp, warps_per_block, natural_order, exact_samples,
                   quad_taps, per_sample_decisions, verify)
    cptr = costs.data_ptr() if costs is not None else None
    s = _stream_handle(stream)
    L = _abi.load()
    if result is not None:
        check(L.cgs_search(C.byref(moving.img), C.byref(fixed.img), C.byref(grid.g), C.byref(opt), cptr,
                           result.data_ptr(), s))
        return None
    r = CgsArgmin()
    check(L.cgs_search_sync(C.byref(moving.img), C.byref(fixed.img), C.byref(grid.g), C.byref(opt), cptr,
                            C.byref(r), s))
    return Argmin.from_struct(r)


def refine(cost: str, moving: CudaImage, fixed: CudaImage, grid: CudaGrid, depth: int, stream=None,
           mi_bins: int = 0, overlap_gate: float = 0.0, exact_samples: bool | None = None):
    """Coarse-to-fine search (cgs_search_refine): `depth` searches, each on the previous grid
    shrunk about its argmin as the reference's driver does (src/gpu/cudaGridSearch_main_mi.cu:
    312-363).  Returns (per-level Argmins, the last level's CudaGrid)."""
    opt = _options(cost, mi_bins, overlap_gate, exact_samples=exact_samples)
    levels = (CgsArgmin * int(depth))()
    last = CudaGrid(grid.g.dims)
    check(_abi.load().cgs_search_refine(C.byref(moving.img), C.byref(fixed.img), C.byref(grid.g), C.byref(opt),
                                        int(depth), levels, C.byref(last.g), _stream_handle(stream)))
    return [Argmin.from_struct(r) for r in levels], last


def homography(params, cx: float = 0.0, cy: float = 0.0, centred: bool = True) -> np.ndarray:
    """parametersToHomography (centred at (cx, cy)) or the uncentred form: the 8 entries
    h11..h32 (float32) of the reference's float arithmetic."""
    p = (C.c_float * 8)(*[float(np.float32(v)) for v in params])
    out = (C.c_float * 8)()
    check(_abi.load().cgs_homography(p, float(cx), float(cy), int(bool(centred)), out))
    return np.array(list(out), np.float32)


def transform_image(H, image: CudaImage, out: CudaImage, rows: int | None = None, cols: int | None = None,
                    stream=None) -> None:
    """transformImage: out(y, x) = image sampled at the inverse map of H, where inside."""
    h = (C.c_float * 8)(*[float(np.float32(v)) for v in H])
    rows = out.height() if rows is None else rows
    cols = out.width() if cols is None else cols
    check(_abi.load().cgs_transform_image(h, int(rows), int(cols), C.byref(image.img), C.byref(out.img),
                                          _stream_handle(stream)))


def fuse_aligned(estimated_H, true_H, reference: CudaImage, moving: CudaImage, fused: CudaImage, channel: int = 0,
                 stream=None) -> None:
    """fuseAlignedImages: 3-channel overlay (moving under the estimate, reference, moving
    under the true homography)."""
    he = (C.c_float * 8)(*[float(np.float32(v)) for v in estimated_H])
    ht = (C.c_float * 8)(*[float(np.float32(v)) for v in true_H])
    check(_abi.load().cgs_fuse_aligned(he, ht, C.byref(reference.img), C.byref(moving.img), C.byref(fused.img),
                                       int(channel), _stream_handle(stream)))


def filter_image(filt: CudaImage, image: CudaImage, out: CudaImage, actions=None, stream=None) -> None:
    """CudaImage::filter: correlate FILTER channels (action 1) with `filt`, copy COPY channels
    (action 0); by default every channel is filtered."""
    c = image.channels()
    acts = (C.c_int32 * c)(*([1] * c if actions is None else [int(a) for a in actions]))
    check(_abi.load().cgs_filter_image(C.byref(filt.img), C.byref(image.img), C.byref(out.img), acts,
                                       _stream_handle(stream)))


def quantize_image(image: CudaImage, mod: float, stream=None) -> None:
    """transformPixel: in-place intensity quantisation of a uint8 image."""
    check(_abi.load().cgs_quantize_image(C.byref(image.img), float(mod), _stream_handle(stream)))


def argmin(values, stream=None) -> Argmin:
    torch = _torch()
    out = torch.empty(C.sizeof(CgsArgmin), dtype=torch.uint8, device=values.device)
    check(_abi.load().cgs_argmin_f32(values.data_ptr(), values.numel(), out.data_ptr(), _stream_handle(stream)))
    return Argmin.from_struct(CgsArgmin.from_buffer_copy(out.cpu().numpy().tobytes()))


def mi_histogram(moving: CudaImage, fixed: CudaImage, params, bins: int = 32, stream=None) -> np.ndarray:
    """Joint (fixed bin, moving bin) counts of the MI cost at one parameter vector."""
    torch = _torch()
    h = torch.empty(bins * bins, dtype=torch.int32, device=moving.tensor.device)
    p = (C.c_float * 8)(*[float(np.float32(v)) for v in params])
    check(_abi.load().cgs_mi_histogram(C.byref(moving.img), C.byref(fixed.img), p, bins, h.data_ptr(),
                                       _stream_handle(stream)))
    return h.cpu().numpy().view(np.uint32).reshape(bins, bins)


def covariance(grid: CudaGrid, costs, stream=None) -> np.ndarray:
    """CudaGridSearcher::covariance_by_value on a cost tensor (cgs_covariance): the
    dims x dims curvature matrix around the grid minimum, summed in double."""
    torch = _torch()
    d = grid.g.dims
    out = torch.empty(d * d, dtype=torch.float64, device=costs.device)
    check(_abi.load().cgs_covariance(C.byref(grid.g), costs.data_ptr(), costs.numel(), out.data_ptr(),
                                     _stream_handle(stream)))
    return out.cpu().numpy().reshape(d, d)


def result_buffer(device=None):
    """A device buffer for one asynchronous cgs_argmin result."""
    torch = _torch()
    return torch.empty(C.sizeof(CgsArgmin), dtype=torch.uint8, device=device or "cuda")


def read_result(buf) -> Argmin:
    return Argmin.from_struct(CgsArgmin.from_buffer_copy(buf.cpu().numpy().tobytes()))


class CudaGridSearcher:
    """CudaGridSearcher<float, float, D> (src/gpu/cudaGridSearch.cuh:540-855).

    Every search variant evaluates the same function of each grid point, so all of them
    run the one fused kernel; the launch-shape arguments of the stream/block variants
    (STREAM_BLOCK_DIM, numCores, numThreads) are accepted and ignored.  The result tensor
    receives the per-point costs, as the reference's does."""

    def __init__(self, grid: CudaGrid, result: CudaTensor | None):
        self._grid = grid
        self._result = result
        self.last: Argmin | None = None

    def _run(self, fn: str, moving: CudaImage, fixed: CudaImage, **kw) -> Argmin:
        costs = self._result.tensor if self._result is not None else None
        if costs is not None and costs.numel() < self._grid.numElements():
            raise ValueError("result tensor is smaller than the grid")
        self.last = search(fn, moving, fixed, self._grid, costs=costs, **kw)
        return self.last

    def search(self, fn, moving, fixed, **kw):
        return self._run(fn, moving, fixed, **kw)

    def search_by_value(self, fn, moving, fixed, **kw):
        return self._run(fn, moving, fixed, **kw)

    def search_by_value_block(self, fn, numThreads, moving, fixed, **kw):
        return self._run(fn, moving, fixed, **kw)

    def search_by_value_stream(self, fn, STREAM_BLOCK_DIM, numCores, moving, fixed, **kw):
        return self._run(fn, moving, fixed, **kw)

    def search_by_reference(self, fn, moving, fixed, **kw):
        return self._run(fn, moving, fixed, **kw)

    def search_by_reference_stream(self, fn, STREAM_BLOCK_DIM, numCores, moving, fixed, **kw):
        return self._run(fn, moving, fixed, **kw)

    def covariance_by_value(self, covar_matrix=None) -> np.ndarray:
        """Curvature matrix around the minimum of the result tensor (D x D); added into
        covar_matrix when one is given, as the reference adds into its buffer."""
        if self._result is None:
            raise ValueError("covariance_by_value needs the result tensor")
        n = self._grid.numElements()
        cov = covariance(self._grid, self._result.tensor.reshape(-1)[:n])
        if covar_matrix is not None:
            covar_matrix += cov.astype(covar_matrix.dtype).reshape(covar_matrix.shape)
            return covar_matrix
        return cov


@dataclass
class BatchPlan:
    """Launch plan of the batch kernel (cgs_batch_plan): grid points per warp (1, 2, 4, 8),
    warps per block (4, 8, 16) and whether a block's warps share points (block_split: MI
    histograms per block) or own them (MI histograms per warp)."""
    points_per_warp: int = 2
    warps_per_block: int = 16
    block_split: int = 0

    def to_c(self) -> CgsBatchPlan:
        return CgsBatchPlan(self.points_per_warp, self.warps_per_block, self.block_split, 0)

    @staticmethod
    def from_c(p: CgsBatchPlan) -> "BatchPlan":
        return BatchPlan(int(p.points_per_warp), int(p.warps_per_block), int(p.block_split))


@dataclass
class BatchPair:
    """One pair of a batch: images, grid, cost options, an optional cost dump and a device
    result buffer (see :func:`result_buffer`)."""
    cost: str
    moving: CudaImage
    fixed: CudaImage
    grid: CudaGrid
    result: object
    costs: object = None
    mi_bins: int = 0
    overlap_gate: float = 0.0
    exact_samples: bool | None = None
    per_sample_decisions: bool = False

    def to_c(self) -> CgsPair:
        opt = _options(self.cost, self.mi_bins, self.overlap_gate, exact_samples=self.exact_samples,
                       per_sample_decisions=self.per_sample_decisions)
        return CgsPair(self.moving.img, self.fixed.img, self.grid.g, opt,
                       self.costs.data_ptr() if self.costs is not None else None, self.result.data_ptr())


class Batch:
    """Many pairs in one recorded launch sequence (cgs_batch_*): a persistent kernel over the
    pairs' tasks, then the span-kernel searches of the ZNCC and MI pairs that :func:`search`
    runs on span kernels; the pairs' images, dumps and results are bound at creation;
    :meth:`launch` replays the recorded CUDA graph."""

    def __init__(self, pairs: list[BatchPair], plan: BatchPlan | None = None):
        self.pairs = list(pairs)  # keeps the tensors alive
        arr = (CgsPair * len(self.pairs))(*[p.to_c() for p in self.pairs])
        h = C.c_void_p(None)
        cp = C.byref(plan.to_c()) if plan is not None else None
        check(_abi.load().cgs_batch_create(arr, len(self.pairs), cp, C.byref(h)))
        self._h = h

    def launch(self, stream=None) -> None:
        check(_abi.load().cgs_batch_launch(self._h, _stream_handle(stream)))

    @property
    def plan(self) -> BatchPlan:
        p = CgsBatchPlan()
        check(_abi.load().cgs_batch_get_plan(self._h, C.byref(p)))
        return BatchPlan.from_c(p)

    @plan.setter
    def plan(self, plan: BatchPlan) -> None:
        check(_abi.load().cgs_batch_set_plan(self._h, C.byref(plan.to_c())))

    def autotune(self, sample_points: int = 4096) -> tuple[BatchPlan, list[tuple[BatchPlan, float, int]]]:
        """Times all 24 plans on the first ``sample_points`` points of every pair, applies the
        fastest and returns it with every (plan, ms, status) measurement."""
        entries = (CgsTuneEntry * 32)()
        n = C.c_int32(0)
        best = CgsBatchPlan()
        check(_abi.load().cgs_batch_autotune(self._h, int(sample_points), entries, 32, C.byref(n), C.byref(best)))
        table = [(BatchPlan.from_c(e.plan), float(e.ms), int(e.status)) for e in entries[: n.value]]
        return BatchPlan.from_c(best), table

    def pair_times(self) -> tuple[np.ndarray, np.ndarray]:
        """(start, end) device time stamps in ns of each pair's first and last task in the
        last launch (waits for it)."""
        n = len(self.pairs)
        a, b = (C.c_uint64 * n)(), (C.c_uint64 * n)()
        check(_abi.load().cgs_batch_pair_times(self._h, a, b))
        return np.array(list(a), dtype=np.uint64), np.array(list(b), dtype=np.uint64)

    @property
    def kernel_launches(self) -> int:
        """Kernel launches of one :meth:`launch` (the recorded graph's kernel nodes)."""
        n = C.c_int32(0)
        check(_abi.load().cgs_batch_kernel_launches(self._h, C.byref(n)))
        return int(n.value)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _abi.load().cgs_batch_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
