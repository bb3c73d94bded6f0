"""The allocation-free entry point, cgs_search_noalloc.

Callers that cannot allocate device memory while they run (a loop that reserves its memory
budget up front, or a process where a caching allocator already holds nearly all free
memory) use cgs_search_noalloc, whose scratch is a fixed array inside the library.  These
tests call it through the C ABI, twice in a row (the array keeps the previous call's
contents), and compare each result with cgs_search's on the same inputs.  This file is
collected last so that a run stopping at the first failure has run every other test first;
it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from cugridsearch_b200 import synthetic as S

pytestmark = pytest.mark.gpu

REL = 1e-6  # both entry points form every sum identically; allow a last-bit difference


def _run(lib, fn, mov, fix, grid, opts, costs, res, stream):
    status = getattr(lib, fn)(C.byref(mov.img), C.byref(fix.img), C.byref(grid.g), C.byref(opts),
                              costs.data_ptr(), res.data_ptr(), stream)
    assert status == 0, lib.cgs_last_error().decode()


# Every cost the allocation-free entry point runs, single- and three-channel where the cost
# takes several channels.  Each case's second pair has a moving image smaller than the fixed
# one, so samples reach the moving image's last column and row (the reference's flat-index
# neighbour at W - 1 < x < W and the zero row past the image).
CASES = [(c, ch) for c in ("SAD_AVG", "SQD_REF", "NCC_REF", "ZNCC", "MI") for ch in (1, 3)] + \
        [("SAD_AVG_H", 1), ("SAD_SUM_T", 1), ("SAD_SUM_T_REF", 1)]


def _case_pairs(cost, channels):
    u8 = cost == "MI"
    base = "SAD_AVG" if cost in ("SAD_SUM_T", "SAD_SUM_T_REF") else cost
    pairs = [S.small_pair(41, size=64, count=4, cost=base, u8=u8, channels=channels),
             S.small_pair(42, size=48, count=4, cost=base, u8=u8, channels=channels, msize=37)]
    grids = []
    for p in pairs:
        if cost == "SAD_AVG_H":
            grids.append(([0.95, -0.05, -4.0, -0.05, 0.95, -4.0, -1e-4, -1e-4],
                          [1.05, 0.05, 4.0, 0.05, 1.05, 4.0, 1e-4, 1e-4], [3] * 8))
        elif cost in ("SAD_SUM_T", "SAD_SUM_T_REF"):
            grids.append(([-6.0, -6.0], [6.0, 6.0], [25, 19]))
        else:
            grids.append(p.grid_args())
    return pairs, grids


@pytest.mark.parametrize("cost,channels", CASES)
def test_noalloc_matches_search_on_two_calls(cuda, lib, cost, channels):
    import torch
    import cugridsearch_b200 as cgs
    import cugridsearch_b200._abi as abi
    stream = torch.cuda.current_stream().cuda_stream
    pairs, grids = _case_pairs(cost, channels)
    for k, (pair, ga) in enumerate(zip(pairs, grids)):  # two calls in a row, different inputs
        mov = cgs.CudaImage(torch.from_numpy(pair.moving).to(cuda))
        fix = cgs.CudaImage(torch.from_numpy(pair.fixed).to(cuda))
        grid = cgs.CudaGrid.from_ranges(*ga)
        n = grid.numElements()
        opts = abi.CgsOptions(abi.COSTS[cost], 32, 0.0, 0, 0, 0)
        ref_costs = torch.full((n,), 7e30, device=cuda)
        ref_res = cgs.result_buffer(cuda)
        _run(lib, "cgs_search", mov, fix, grid, opts, ref_costs, ref_res, stream)
        na_costs = torch.full((n,), 7e30, device=cuda)
        na_res = cgs.result_buffer(cuda)
        _run(lib, "cgs_search_noalloc", mov, fix, grid, opts, na_costs, na_res, stream)
        torch.cuda.synchronize()
        a, b = ref_costs.cpu().numpy(), na_costs.cpu().numpy()
        fin = np.isfinite(a)
        np.testing.assert_array_equal(fin, np.isfinite(b))
        assert np.all(np.abs(a[fin] - b[fin]) <= REL * np.maximum(np.abs(a[fin]), 1.0)), f"call {k}"
        ra, rb = cgs.read_result(ref_res), cgs.read_result(na_res)
        assert rb.valid and rb.status == 0
        assert rb.index == ra.index or abs(rb.cost - ra.cost) <= REL * max(1.0, abs(ra.cost))


@pytest.mark.parametrize("cost", ["SQD_ALT", "NCC_ALT", "MI_ALT"])
def test_noalloc_rejects_scanline_costs(cuda, lib, cost):
    """The scanline functors have no allocation-free kernel: the call is refused with
    CGS_ERROR_UNSUPPORTED and a message naming the reason, and nothing runs."""
    import torch
    import cugridsearch_b200 as cgs
    import cugridsearch_b200._abi as abi
    pair = S.small_pair(44, size=32, count=3, cost=cost)
    mov = cgs.CudaImage(torch.from_numpy(pair.moving).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(pair.fixed).to(cuda))
    grid = cgs.CudaGrid.from_ranges(*pair.grid_args())
    opts = abi.CgsOptions(abi.COSTS[cost], 32, 0.0, 0, 0, 0)
    res = cgs.result_buffer(cuda)
    status = lib.cgs_search_noalloc(C.byref(mov.img), C.byref(fix.img), C.byref(grid.g), C.byref(opts), None,
                                    res.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert status == 2
    assert b"scanline" in lib.cgs_last_error()


def test_noalloc_allocates_nothing_and_rejects_oversize(cuda, lib):
    import torch
    import cugridsearch_b200 as cgs
    import cugridsearch_b200._abi as abi
    stream = torch.cuda.current_stream().cuda_stream
    pair = S.small_pair(43, size=64, count=4, cost="ZNCC")
    mov = cgs.CudaImage(torch.from_numpy(pair.moving).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(pair.fixed).to(cuda))
    grid = cgs.CudaGrid.from_ranges(*pair.grid_args())
    n = grid.numElements()
    opts = abi.CgsOptions(abi.COSTS["ZNCC"], 32, 0.0, 0, 0, 0)
    costs = torch.empty((n,), device=cuda)
    res = cgs.result_buffer(cuda)
    _run(lib, "cgs_search_noalloc", mov, fix, grid, opts, costs, res, stream)  # first call: set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        _run(lib, "cgs_search_noalloc", mov, fix, grid, opts, costs, res, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, "device memory changed across allocation-free calls"
    # 1536 x 1536 f32 pair: staged copies need about 19 MB > the 16 MiB array
    big = torch.zeros((1536, 1536), dtype=torch.float32, device=cuda)
    bm = cgs.CudaImage(big)
    status = lib.cgs_search_noalloc(C.byref(bm.img), C.byref(bm.img), C.byref(grid.g), C.byref(opts),
                                    None, res.data_ptr(), stream)
    assert status == 1 and b"too large" in lib.cgs_last_error()
