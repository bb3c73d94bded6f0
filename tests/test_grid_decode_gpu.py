"""The library's grid arithmetic against the reference's own CudaGrid running on the GPU.

The reference decodes grid points only on the device (CudaGrid::indexToGridPoint,
src/gpu/cudaGridSearch.cuh:160-187, compiled with nvcc's default flags, which contract
start + i * res into one fused multiply-add) and updates the grid on the device
(updateProcess, :235-272).  The oracle harness builds that code unchanged for sm_100a
(oracle/ref_harness.cu); here its grid points and resolutions are compared bit for bit with
the library's host-side cgs_grid_point / cgs_grid_update, which every search result's
parameters come from.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GRIDS = [
    ([-0.1745, 0.9, 0.9, -0.05, -24, -24, -1e-4, -1e-4], [0.1745, 1.1, 1.1, 0.05, 24, 24, 1e-4, 1e-4], [6] * 8),
    ([-0.2, 0.8, 0.8, -0.1, -2, -2, -1e-3, -1e-3], [0.2, 1.2, 1.2, 0.1, 2, 2, 1e-3, 1e-3], [3] * 8),
    ([-0.33, 0.71, 0.93, -0.07, -7.3, -5.1, -3e-4, -2e-4], [0.41, 1.37, 1.19, 0.11, 9.7, 3.3, 4e-4, 1e-4],
     [5, 4, 7, 3, 9, 6, 2, 3]),
    ([-3, -3], [3, 3], [1000, 1000]),
    ([-3, -3], [3, 3], [103, 111]),
    ([-2.5, -1.75], [4.25, 3.5], [7.5, 9]),  # fractional count, as the reference's drivers allow
]


@pytest.mark.skipif(not O.have_ref(), reason="reference harness not built")
@pytest.mark.parametrize("k", range(len(GRIDS)))
def test_grid_points_bit_exact_with_reference_device_decode(cuda, lib, k):
    import cugridsearch_b200 as cgs
    start, end, count = GRIDS[k]
    grid = cgs.CudaGrid.from_ranges(start, end, count)
    n = grid.numElements()
    rng = np.random.default_rng(k)
    idx = np.unique(np.concatenate([[0, n - 1], rng.integers(0, n, 300)])).astype(np.int64)
    pts, mat = O.ref_device_grid_points(start, end, count, idx)
    d = len(start)
    np.testing.assert_array_equal(mat[2], np.array(list(grid.g.resolution)[:d], np.float32))
    np.testing.assert_array_equal(mat[3], np.array(list(grid.g.count)[:d], np.float32))
    mine = np.array([grid.getGridPoint(int(i))[:d] for i in idx], dtype=np.float32)
    np.testing.assert_array_equal(mine, pts)
