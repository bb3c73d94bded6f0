"""The span kernels: zero-mean NCC with row decisions and shared-memory windows (cgs_span.cuh),
and MI with row decisions and queued exact samples (cgs_span_mi.cuh).

It is the default for single-channel ZNCC on the fast sampling path.  Checked here against the
per-sample decision kernel (CGS_FLAG_PER_SAMPLE_DECISIONS, itself oracle-checked in
test_gpu_parity.py) and against the FP64 oracle:

* same finite/infinite pattern (the same overlap decisions gate the costs) and costs within the
  FP32 summation tolerance, on ragged sizes (moving image smaller or larger than the fixed one,
  widths that are not multiples of the tile width);
* bit-identical costs for 2 and 4 points per warp and for the locality and the reference order;
* every tile shape (64, 128 or 256 columns by 8, 16 or 32 rows) within tolerance;
* maps whose rows run along the moving image's edges (no rotation, unit scale, whole-pixel
  translations: whole rows and columns on the overlap's boundary take the exact path) against
  the per-sample kernel and the oracle;
* windows too large for a stage (forced small with CGS_SPAN_CAP) read global memory instead, with
  bit-identical costs;
* the self-checking build (CGS_SPAN_CHECK=1) finds every fast sample's quad inside its window;
* MI: costs bit-identical to the per-sample kernel's (the histogram counts are exact in both and
  the cost is formed by the same function), on ragged u8 and f32 pairs, every band height, and
  rows along the image edges.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import close_costs
from cugridsearch_b200 import synthetic as S

pytestmark = pytest.mark.gpu


class _env:
    """Set tuning variables of the library for the duration of a block."""

    def __init__(self, **kv):
        self.kv = {k: str(v) for k, v in kv.items()}

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        os.environ.update(self.kv)

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _run(cuda, pair, cost="ZNCC", **kw):
    import torch
    import cugridsearch_b200 as cgs
    mov = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.moving)).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.fixed)).to(cuda))
    grid = cgs.CudaGrid.from_ranges(*pair.grid_args())
    costs = torch.full((grid.numElements(),), 7.0e30, dtype=torch.float32, device=cuda)
    res = cgs.search(cost, mov, fix, grid, costs=costs, **kw)
    torch.cuda.synchronize()
    assert res.status == 0
    return res, costs.cpu().numpy()


def _per_sample(cuda, pair, cost="ZNCC"):
    import cugridsearch_b200 as cgs
    import cugridsearch_b200._abi as abi
    import torch
    mov = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.moving)).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.fixed)).to(cuda))
    grid = cgs.CudaGrid.from_ranges(*pair.grid_args())
    n = grid.numElements()
    costs = torch.full((n,), 7.0e30, dtype=torch.float32, device=cuda)
    import ctypes as C
    opts = abi.CgsOptions(abi.COSTS[cost], 32, 0.0, 0, 0, abi.FLAG_PER_SAMPLE_DECISIONS)
    r = abi.CgsArgmin()
    abi.check(abi.load().cgs_search_sync(C.byref(mov.img), C.byref(fix.img), C.byref(grid.g), C.byref(opts),
                                         costs.data_ptr(), C.byref(r), torch.cuda.current_stream().cuda_stream))
    return r, costs.cpu().numpy()


def _agree(a, b, rel=1e-5):
    fin = np.isfinite(b)
    np.testing.assert_array_equal(np.isfinite(a), fin)
    d = np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1.0)
    assert d.max(initial=0.0) <= rel, d.max()


CASES = [(64, 64), (96, 80), (100, 128), (45, 37), (160, 160)]


@pytest.mark.parametrize("size,msize", CASES)
def test_span_matches_per_sample_kernel_and_oracle(cuda, lib, size, msize):
    pair = S.small_pair(300 + size, size=size, count=3, cost="ZNCC", msize=msize)
    with _env(CGS_SPAN_CHECK=1):
        res, c = _run(cuda, pair)
    r0, c0 = _per_sample(cuda, pair)
    _agree(c, c0)
    g = O.make_grid(*pair.grid_args())
    c32, c64 = O.search("ZNCC", g, O.Image(pair.moving), O.Image(pair.fixed))
    bad = close_costs(c, c32, c64, "ZNCC")
    assert not bad.any(), int(bad.sum())
    fin = np.where(np.isfinite(c), c, np.inf)
    assert res.index == int(np.argmin(fin)) and res.cost == c[res.index]


def test_span_tunings_bit_identical(cuda, lib):
    pair = S.small_pair(311, size=96, count=3, cost="ZNCC", msize=90)
    base, c0 = _run(cuda, pair)
    for kw in ({"points_per_warp": 2}, {"natural_order": True}, {"points_per_warp": 2, "natural_order": True}):
        r, c = _run(cuda, pair, **kw)
        np.testing.assert_array_equal(c.view(np.uint32), c0.view(np.uint32))
        assert r.index == base.index


@pytest.mark.parametrize("tx", [2, 4, 8])
@pytest.mark.parametrize("th", [8, 16, 32])
def test_span_tile_shapes(cuda, lib, tx, th):
    pair = S.small_pair(317, size=136, count=3, cost="ZNCC", msize=128)
    _, c0 = _per_sample(cuda, pair)
    with _env(CGS_SPAN_TX=tx, CGS_SPAN_TH=th, CGS_SPAN_CHECK=1):
        _, c = _run(cuda, pair)
    _agree(c, c0)


def test_span_global_fallback_bit_identical(cuda, lib):
    pair = S.config4()
    pair.count[:] = 3
    with _env(CGS_SPAN_CHECK=1):
        _, c0 = _run(cuda, pair)
        with _env(CGS_SPAN_CAP=1024):  # most windows no longer fit: those tiles read global memory
            _, c1 = _run(cuda, pair)
    np.testing.assert_array_equal(c1.view(np.uint32), c0.view(np.uint32))
    _, cp = _per_sample(cuda, pair)
    _agree(c0, cp)


def test_span_config1_self_check(cuda, lib):
    """The benchmark pair through the self-checking build: no fast sample's quad leaves its
    window, and the costs equal the plain build's bit for bit."""
    pair = S.config1()
    _, c0 = _run(cuda, pair)
    with _env(CGS_SPAN_CHECK=1):
        _, c1 = _run(cuda, pair)
    np.testing.assert_array_equal(c1.view(np.uint32), c0.view(np.uint32))


def test_span_rows_along_the_edges(cuda, lib):
    """Translations by whole pixels (and a half pixel), no rotation, unit scale: mapped
    coordinates land exactly on the moving image's first and last rows and columns, so whole
    rows of the band take the reference's exact sequence."""
    pair = S.small_pair(331, size=72, count=3, cost="ZNCC", msize=64)
    pair.lo[:] = [0.0, 1.0, 1.0, 0.0, -8.0, -8.0, 0.0, 0.0]
    pair.hi[:] = [0.0, 1.0, 1.0, 0.0, 8.0, 8.0, 0.0, 0.0]
    pair.count[:] = [1, 1, 1, 1, 33, 33, 1, 1]
    with _env(CGS_SPAN_CHECK=1):
        res, c = _run(cuda, pair)
    _, c0 = _per_sample(cuda, pair)
    _agree(c, c0)
    g = O.make_grid(*pair.grid_args())
    c32, c64 = O.search("ZNCC", g, O.Image(pair.moving), O.Image(pair.fixed))
    bad = close_costs(c, c32, c64, "ZNCC")
    assert not bad.any(), int(bad.sum())


MI_CASES = [(64, 64, True), (96, 80, True), (100, 128, True), (45, 37, True), (72, 64, False)]


@pytest.mark.parametrize("size,msize,u8", MI_CASES)
def test_mi_span_equals_per_sample_kernel(cuda, lib, size, msize, u8):
    pair = S.small_pair(400 + size, size=size, count=3, cost="MI", u8=u8, msize=msize)
    with _env(CGS_SPAN_CHECK=1):
        res, c = _run(cuda, pair, "MI")
    r0, c0 = _per_sample(cuda, pair, "MI")
    np.testing.assert_array_equal(c.view(np.uint32), c0.view(np.uint32))
    assert res.index == r0.index
    g = O.make_grid(*pair.grid_args())
    c32, c64 = O.search("MI", g, O.Image(pair.moving), O.Image(pair.fixed), O.opts(32))
    bad = close_costs(c, c32, c64, "MI")
    assert not bad.any(), int(bad.sum())


@pytest.mark.parametrize("th", [8, 16, 32])
def test_mi_span_band_heights(cuda, lib, th):
    pair = S.small_pair(421, size=80, count=3, cost="MI", u8=True, msize=76)
    _, c0 = _per_sample(cuda, pair, "MI")
    with _env(CGS_SPAN_TH=th, CGS_SPAN_CHECK=1):
        _, c = _run(cuda, pair, "MI")
    np.testing.assert_array_equal(c.view(np.uint32), c0.view(np.uint32))


def test_mi_span_rows_along_the_edges(cuda, lib):
    pair = S.small_pair(433, size=72, count=3, cost="MI", u8=True, msize=64)
    pair.lo[:] = [0.0, 1.0, 1.0, 0.0, -8.0, -8.0, 0.0, 0.0]
    pair.hi[:] = [0.0, 1.0, 1.0, 0.0, 8.0, 8.0, 0.0, 0.0]
    pair.count[:] = [1, 1, 1, 1, 33, 33, 1, 1]
    with _env(CGS_SPAN_CHECK=1):
        _, c = _run(cuda, pair, "MI")
    _, c0 = _per_sample(cuda, pair, "MI")
    np.testing.assert_array_equal(c.view(np.uint32), c0.view(np.uint32))


def test_mi_span_config2_self_check(cuda, lib):
    """The MI benchmark pair (512^2 u8) on a 3^8 grid: the self-checking build reports no quad
    outside the image and equals the plain build and the per-sample kernel bit for bit."""
    pair = S.config2()
    pair.count[:] = 3
    _, c0 = _run(cuda, pair, "MI")
    with _env(CGS_SPAN_CHECK=1):
        _, c1 = _run(cuda, pair, "MI")
    np.testing.assert_array_equal(c1.view(np.uint32), c0.view(np.uint32))
    _, cp = _per_sample(cuda, pair, "MI")
    np.testing.assert_array_equal(c0.view(np.uint32), cp.view(np.uint32))
