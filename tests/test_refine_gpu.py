"""Coarse-to-fine search (cgs_search_refine) against the reference driver's loop restated on the
CPU with the oracle (src/gpu/cudaGridSearch_main_mi.cu:312-363): each level's argmin, decoded
point and next grid.  A level's argmin is compared only where the oracle's best cost is
separated from the runner-up by more than the parity tolerance; the loop stops comparing at
the first tied level (both sides are then free to go different ways)."""
import numpy as np
import pytest

import oracle as O
from conftest import separated_argmin
from cugridsearch_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _oracle_levels(name, pair, depth):
    start, end, count = pair.grid_args()
    M, F = O.Image(pair.moving), O.Image(pair.fixed)
    start = np.array(start, np.float32)
    end = np.array(end, np.float32)
    out = []
    for _ in range(depth):
        g = O.make_grid(start, end, count)
        c32, c64 = O.search(name, g, M, F)
        i, sep, _ = separated_argmin(c32, c64, name)
        p = O.grid_point(g, i)[: len(start)]
        out.append((i, sep, p.copy(), np.array(list(g.start)[:8], np.float32), np.array(list(g.end)[:8], np.float32)))
        quarter = (end - start) / np.float32(4)
        start = (p - quarter).astype(np.float32)
        end = (p + (end - start) / np.float32(4)).astype(np.float32)
    return out


@pytest.mark.parametrize("name", ["NCC_REF", "ZNCC", "SAD_AVG"])
def test_refine_matches_reference_loop(cuda, lib, name):
    import torch
    import cugridsearch_b200 as cgs
    pair = S.small_pair(303, size=32, count=3, cost=name)
    mov = cgs.CudaImage(torch.from_numpy(pair.moving).to(cuda))
    fix = cgs.CudaImage(torch.from_numpy(pair.fixed).to(cuda))
    grid = cgs.CudaGrid.from_ranges(*pair.grid_args())
    depth = 3
    levels, last = cgs.refine(name, mov, fix, grid, depth)
    ref = _oracle_levels(name, pair, depth)
    for lv, (r, (i, sep, p, st, en)) in enumerate(zip(levels, ref)):
        assert r.valid and r.status == 0
        if not sep:
            break
        assert r.index == i, (lv, r.index, i)
        np.testing.assert_array_equal(r.params, p)
    else:
        # every level agreed: the final grid is the oracle's last level grid
        np.testing.assert_array_equal(last.matrix()[0], ref[-1][3])
        np.testing.assert_array_equal(last.matrix()[1], ref[-1][4])
