"""The FP64 verification pass of cgs_search (cgs_verify.cu) against the CPU oracle.

The pass re-scores, with the reference's exact sampling and FP64 sums, the grid points whose FP32
cost lies within 2e-5 x max(1, |best|) of the minimum and reports, in the result: the FP64 cost of
the reported index (cost_fp64) and its error (err_fp64), the FP64 argmin among the re-scored points
(index_fp64) and the largest FP32 - FP64 difference among them.  Checked here:

* cost_fp64 equals the CPU oracle's FP64 cost of the reported index to FP64 summation order (1e-12
  relative), for every cost the pass supports, one and three channels, and the benchmark pair;
* err_fp64 is |cost - cost_fp64| and within the FP32 tolerance (1e-5 of the cost scale);
* index_fp64 is the FP64 argmin of the whole grid (the oracle's, ties within 1e-12 aside);
* without the pass (verify=False) and for the scanline functors the fields read "not verified".
"""
import math

import numpy as np
import pytest

import oracle as O
from conftest import COST_SCALE
from cugridsearch_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _run(cuda, pair, cost, grid_args=None, **kw):
    import torch
    import cugridsearch_b200 as cgs
    mov = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.moving)).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.fixed)).to(cuda))
    grid = cgs.CudaGrid.from_ranges(*(grid_args or pair.grid_args()))
    costs = torch.empty(grid.numElements(), dtype=torch.float32, device=cuda)
    res = cgs.search(cost, mov, fix, grid, costs=costs, **kw)
    return res, costs.cpu().numpy()


def _oracle64(pair, cost, grid_args=None, idx=None, mi_bins=32):
    g = O.make_grid(*(grid_args or pair.grid_args()))
    F, M = O.Image(pair.fixed), O.Image(pair.moving)
    if idx is None:
        _, c64 = O.search(cost, g, M, F, O.opts(mi_bins), f32=False)
        return c64
    _, c64 = O.search(cost, g, M, F, O.opts(mi_bins), first=int(idx), count=1, f32=False, threads=1)
    return float(c64[0])


def _check(res, gpu, c64_all, cost):
    assert res.valid and res.verified >= 1 and res.candidates >= res.verified
    ref = c64_all[res.index]
    scale = max(abs(ref), 1.0)
    assert abs(res.cost_fp64 - ref) <= 1e-12 * scale, (res.cost_fp64, ref)
    assert res.err_fp64 == pytest.approx(abs(res.cost - res.cost_fp64), abs=1e-12 * scale)
    assert res.err_fp64 <= 1e-5 * max(abs(ref), COST_SCALE[cost])
    assert res.max_err_fp64 >= res.err_fp64
    fin = np.where(np.isfinite(c64_all), c64_all, np.inf)
    best = int(np.argmin(fin))
    assert res.index_fp64 == best or abs(fin[res.index_fp64] - fin[best]) <= 1e-12 * max(abs(fin[best]), 1.0)


CASES = ["SAD_AVG", "SQD_REF", "NCC_REF", "ZNCC", "MI"]


@pytest.mark.parametrize("channels", [1, 3])
@pytest.mark.parametrize("cost", CASES)
def test_verify_matches_oracle_fp64(cuda, lib, cost, channels):
    u8 = cost == "MI"
    pair = S.small_pair(501, size=48, count=3, cost=cost, u8=u8, channels=channels, msize=44)
    res, gpu = _run(cuda, pair, cost)
    _check(res, gpu, _oracle64(pair, cost), cost)


@pytest.mark.parametrize("cost", ["SAD_AVG_H", "SAD_SUM_T", "SAD_SUM_T_REF"])
def test_verify_raw_and_translation_costs(cuda, lib, cost):
    pair = S.small_pair(503, size=32, count=3, cost="SAD_AVG")
    if cost == "SAD_AVG_H":
        ga = ([0.95, -0.05, -3.0, -0.05, 0.95, -3.0, -1e-3, -1e-3], [1.05, 0.05, 3.0, 0.05, 1.05, 3.0, 1e-3, 1e-3],
              [3] * 8)
    else:
        ga = ([-6.0, -6.0], [6.0, 6.0], [25, 19])
    res, gpu = _run(cuda, pair, cost, grid_args=ga)
    _check(res, gpu, _oracle64(pair, cost, grid_args=ga), cost)


def test_verify_benchmark_pair(cuda, lib):
    """The NCC pair of the benchmark (256^2, 6^8 zero-mean NCC, fast sampling): the reported FP32
    argmin's FP64 cost against the oracle, and the FP64 argmin of the band at least as good."""
    pair = S.config1()
    res, gpu = _run(cuda, pair, "ZNCC")
    assert res.valid and res.verified >= 1
    ref = _oracle64(pair, "ZNCC", idx=res.index)
    assert abs(res.cost_fp64 - ref) <= 1e-12 * max(abs(ref), 1.0)
    assert res.err_fp64 <= 1e-5
    alt = _oracle64(pair, "ZNCC", idx=res.index_fp64)
    assert alt <= ref + 1e-12


def test_verify_off_and_unsupported(cuda, lib):
    pair = S.small_pair(505, size=32, count=3, cost="ZNCC")
    res, _ = _run(cuda, pair, "ZNCC", verify=False)
    assert res.verified == 0 and res.candidates == 0 and res.index_fp64 == -1 and math.isnan(res.cost_fp64)
    res2, _ = _run(cuda, pair, "NCC_ALT")
    assert res2.verified == 0 and res2.index_fp64 == -1
