"""GPU parity: the sm_100a kernels through the C ABI against the CPU oracle.

The oracle's FP32 functions are bit-exact restatements of the reference functors (pinned
in test_oracle.py against the reference source built for the host), and its FP64
functions take the same samples with exact sums.  Per-point costs must satisfy
|gpu - fp64| <= |ref32 - fp64| + 1e-5 * max(|fp64|, scale); sentinels (123123, NaN,
+inf) must match exactly; the argmin must equal the reference's wherever the best cost
is separated from the runner-up by more than that tolerance.
"""
import numpy as np
import pytest

import oracle as O
from conftest import close_costs, separated_argmin
from cugridsearch_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _gpu_search(cuda, pair, cost, dims_grid=None, **kw):
    import torch
    import cugridsearch_b200 as cgs
    mov = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.moving)).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(np.ascontiguousarray(pair.fixed)).to(cuda))
    lo, hi, cnt = dims_grid if dims_grid is not None else pair.grid_args()
    grid = cgs.CudaGrid.from_ranges(lo, hi, cnt)
    n = grid.numElements()
    costs = torch.full((n,), 7.0e30, dtype=torch.float32, device=cuda)
    res = cgs.search(cost, mov, fix, grid, costs=costs, **kw)
    torch.cuda.synchronize()
    return res, costs.cpu().numpy(), grid


def _oracle(pair, cost, dims_grid=None, mi_bins=32, gate=0.0):
    lo, hi, cnt = dims_grid if dims_grid is not None else pair.grid_args()
    g = O.make_grid(lo, hi, cnt)
    F, M = O.Image(pair.fixed), O.Image(pair.moving)
    return O.search(cost, g, M, F, O.opts(mi_bins, gate))


def _check(res, costs, c32, c64, cost, grid):
    bad = close_costs(costs, c32, c64, cost)
    assert not bad.any(), (f"{cost}: {int(bad.sum())} of {len(bad)} points out of tolerance; first "
                           f"{np.flatnonzero(bad)[:5]} gpu={costs[bad][:5]} ref={c32[bad][:5]} f64={c64[bad][:5]}")
    i, sep, near = separated_argmin(c32, c64, cost)
    if i < 0:
        assert not res.valid and res.index == -1
        return
    assert res.valid
    if sep:
        assert res.index == i, f"{cost}: argmin {res.index} != reference {i}"
    else:
        assert res.index in set(near.tolist())
    # the reported argmin is the lowest-index minimum of the dumped costs
    fin = np.where(np.isfinite(costs), costs, np.inf)
    assert res.index == int(np.argmin(fin))
    assert res.cost == costs[res.index]
    np.testing.assert_array_equal(res.params[: grid.getDimension()], grid.getGridPoint(res.index))


EIGHT_PARAM = ["SAD_AVG", "SQD_REF", "NCC_REF", "ZNCC", "MI", "SQD_ALT", "NCC_ALT", "MI_ALT"]


def _pair(seed, size, cost, **kw):
    p = S.small_pair(seed, size=size, count=3, cost=cost, **kw)
    if cost == "MI_ALT":  # calcMIAlt's translations are fractions of the image
        p.lo[4:6], p.hi[4:6] = -0.15, 0.15
    return p


@pytest.mark.parametrize("u8", [False, True])
@pytest.mark.parametrize("cost", EIGHT_PARAM)
def test_eight_param_costs_match_oracle(cuda, lib, cost, u8):
    pair = _pair(101, 32, cost, u8=u8)
    res, costs, grid = _gpu_search(cuda, pair, cost)
    c32, c64 = _oracle(pair, cost)
    _check(res, costs, c32, c64, cost, grid)


@pytest.mark.parametrize("cost", ["SAD_AVG", "NCC_REF", "ZNCC", "MI", "SQD_REF", "SQD_ALT", "NCC_ALT", "MI_ALT"])
def test_ragged_sizes_and_channels(cuda, lib, cost):
    # fixed 29 wide, moving 23 wide: odd row pitches, the W-1 < x < W alias, last-row pad
    pair = _pair(7, 29, cost, msize=23, channels=3)
    res, costs, grid = _gpu_search(cuda, pair, cost)
    c32, c64 = _oracle(pair, cost)
    _check(res, costs, c32, c64, cost, grid)


def test_raw_homography_sad(cuda, lib):
    pair = S.small_pair(3, size=32, count=3, cost="SAD_AVG_H")
    lo = [0.95, -0.05, -3.0, -0.05, 0.95, -3.0, -1e-3, -1e-3]
    hi = [1.05, 0.05, 3.0, 0.05, 1.05, 3.0, 1e-3, 1e-3]
    dg = (lo, hi, [3] * 8)
    res, costs, grid = _gpu_search(cuda, pair, "SAD_AVG_H", dims_grid=dg)
    c32, c64 = _oracle(pair, "SAD_AVG_H", dims_grid=dg)
    _check(res, costs, c32, c64, "SAD_AVG_H", grid)


@pytest.mark.parametrize("cost", ["SAD_SUM_T", "SAD_SUM_T_REF"])
def test_translation_sad(cuda, lib, cost):
    # 2-D translation grid like the reference's example 1/2
    pair = S.small_pair(5, size=24, count=3, cost="SAD_AVG")
    dg = ([-6.0, -6.0], [6.0, 6.0], [49, 37])
    res, costs, grid = _gpu_search(cuda, pair, cost, dims_grid=dg)
    c32, c64 = _oracle(pair, cost, dims_grid=dg)
    _check(res, costs, c32, c64, cost, grid)


@pytest.mark.parametrize("bins", [16, 32, 64])
def test_mi_bins(cuda, lib, bins):
    pair = S.small_pair(11, size=32, count=3, cost="MI", u8=True)
    res, costs, grid = _gpu_search(cuda, pair, "MI", mi_bins=bins)
    c32, c64 = _oracle(pair, "MI", mi_bins=bins)
    _check(res, costs, c32, c64, "MI", grid)


@pytest.mark.parametrize("cost", ["ZNCC", "MI"])
def test_overlap_gate(cuda, lib, cost):
    pair = S.small_pair(13, size=32, count=3, cost=cost)
    res, costs, grid = _gpu_search(cuda, pair, cost, overlap_gate=0.9)
    c32, c64 = _oracle(pair, cost, gate=0.9)
    assert np.isinf(c64).any() and np.isfinite(c64).any()
    _check(res, costs, c32, c64, cost, grid)


@pytest.mark.parametrize("cost", ["SAD_AVG", "ZNCC", "MI"])
def test_order_and_tiling_do_not_change_results(cuda, lib, cost):
    """Locality order vs the reference order, and every points-per-warp and warps-per-block
    setting, give bit-identical costs (each point's sums are formed the same way wherever it
    runs)."""
    pair = S.small_pair(17, size=32, count=3, cost=cost)
    base, c0, _ = _gpu_search(cuda, pair, cost, natural_order=True)
    for g in (1, 2, 4):
        if cost == "MI" and g == 4:
            continue
        for nw in (8, 16):
            r, c, _ = _gpu_search(cuda, pair, cost, points_per_warp=g, warps_per_block=nw)
            np.testing.assert_array_equal(c, c0)
            assert r.index == base.index and r.cost == base.cost


def test_repeatable(cuda, lib):
    pair = S.small_pair(19, size=32, count=3, cost="ZNCC")
    r1, c1, _ = _gpu_search(cuda, pair, "ZNCC")
    for _ in range(3):
        r2, c2, _ = _gpu_search(cuda, pair, "ZNCC")
        np.testing.assert_array_equal(c1, c2)
        assert r1.index == r2.index


def test_argmin_f32(cuda, lib):
    import torch
    import cugridsearch_b200 as cgs
    rng = np.random.default_rng(0)
    v = rng.normal(size=1_000_003).astype(np.float32)
    v[[5, 17, 999_999]] = -10.0          # ties: lowest index wins
    v[[1, 2]] = np.nan
    t = torch.from_numpy(v).to(cuda)
    r = cgs.argmin(t)
    assert r.valid and r.index == 5 and r.cost == -10.0
    val, idx = cgs.CudaTensor(t).find_extrema()
    assert idx == 5 and val == -10.0
    t2 = torch.full((100,), float("nan"), device=cuda)
    r2 = cgs.argmin(t2)
    assert not r2.valid and r2.index == -1


@pytest.mark.parametrize("u8", [True, False])
@pytest.mark.parametrize("bins", [32, 64])
def test_mi_histogram_counts_exact(cuda, lib, u8, bins):
    """Joint-histogram counts equal the oracle's (the reference's arithmetic) exactly."""
    import torch
    import cugridsearch_b200 as cgs
    pair = S.small_pair(23, size=48, count=3, cost="MI", u8=u8)
    mov = cgs.CudaImage(torch.from_numpy(pair.moving).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(pair.fixed).to(cuda))
    F, M = O.Image(pair.fixed), O.Image(pair.moving)
    rng = np.random.default_rng(5)
    for k in range(12):
        params = pair.gt if k == 0 else rng.uniform(pair.lo, pair.hi).astype(np.float32)
        h = cgs.mi_histogram(mov, fix, params, bins=bins)
        ho, n = O.histogram("MI", params, M, F, O.opts(bins))
        np.testing.assert_array_equal(h, ho)
        assert int(h.sum()) == n


@pytest.mark.parametrize("cost", ["MI", "SAD_AVG", "NCC_REF", "ZNCC", "SQD_REF", "SAD_AVG_H"])
def test_fast_path_decisions_match_exact_path(cuda, lib, cost):
    """The guarded fast sampling mode makes the same decisions as the exact mode: MI costs are
    bit-identical (identical histograms), other costs agree to rounding on smooth images."""
    pair = S.small_pair(29, size=96, count=3, cost=cost, u8=(cost == "MI"))
    dg = None
    if cost == "SAD_AVG_H":
        dg = ([0.95, -0.05, -4.0, -0.05, 0.95, -4.0, -1e-4, -1e-4], [1.05, 0.05, 4.0, 0.05, 1.05, 4.0, 1e-4, 1e-4],
              [3] * 8)
    rf, cf, _ = _gpu_search(cuda, pair, cost, dims_grid=dg, exact_samples=False)
    re, ce, _ = _gpu_search(cuda, pair, cost, dims_grid=dg, exact_samples=True)
    if cost == "MI":
        np.testing.assert_array_equal(cf, ce)
    else:
        fin = np.isfinite(ce)
        np.testing.assert_array_equal(np.isfinite(cf), fin)
        assert np.max(np.abs(cf[fin] - ce[fin]) / np.maximum(np.abs(ce[fin]), 1.0)) < 2e-6
    assert rf.index == re.index or abs(rf.cost - re.cost) <= 2e-6 * max(1.0, abs(re.cost))


@pytest.mark.parametrize("fast", [True, False])
@pytest.mark.parametrize("cost", ["SAD_AVG", "SAD_AVG_H", "SQD_REF", "NCC_REF", "ZNCC", "MI"])
def test_quad_taps_identical(cuda, lib, cost, fast):
    """Taps from pre-gathered quads (CGS_FLAG_QUAD_TAPS) give the same costs, bit for bit, as
    texture gathers or scalar loads, in both sampling modes, on ragged three-channel images
    (the W - 1 < x < W alias and the last-row pad) -- and the oracle's tolerance holds."""
    channels = 1 if cost == "SAD_AVG_H" else 3
    pair = S.small_pair(29, size=29, count=3, cost=cost, msize=23, channels=channels)
    base, c0, _ = _gpu_search(cuda, pair, cost, exact_samples=not fast, quad_taps=False)
    res, c1, grid = _gpu_search(cuda, pair, cost, exact_samples=not fast, quad_taps=True)
    np.testing.assert_array_equal(c1.view(np.uint32), c0.view(np.uint32))
    assert res.index == base.index
    c32, c64 = _oracle(pair, cost)
    _check(res, c1, c32, c64, cost, grid)
