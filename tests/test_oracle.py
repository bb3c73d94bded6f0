"""Pinning the CPU oracle (CPU only).

1. Against the committed golden vectors, which the reference's own functor source produced
   (tests/golden/make_golden.py): the oracle's FP32 functions reproduce every stored cost
   bit for bit.  This pin holds on machines without the reference.
2. Against the reference itself (oracle/_ref, where available): bit-exact on random
   parameters, for the costs and for the homography helpers.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from cugridsearch_b200 import synthetic as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))
CASES = MANIFEST["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_reproduces_reference_golden_vectors(case):
    z = np.load(os.path.join(GOLDEN, case["name"] + ".npz"))
    M, F = O.Image(z["moving"]), O.Image(z["fixed"])
    g = O.make_grid(case["start"], case["end"], case["count"])
    assert O.grid_num(g) == case["grid_points"]
    idx = z["indices"]
    stride = case["stride"]
    c32, _ = O.search(case["cost"], g, M, F, first=0, count=len(idx), stride=stride, f64=False)
    np.testing.assert_array_equal(c32, z["costs"])
    if stride == 1:
        fin = np.where(np.isfinite(c32), c32, np.inf)
        assert int(np.argmin(fin)) == int(z["argmin"])


def test_example_translation_minimum_is_at_zero_shift():
    # example 1 searches A against itself: the best translation is the grid point nearest 0
    case = next(c for c in CASES if c["name"] == "ex1_A_A_translation_sad")
    g = O.make_grid(case["start"], case["end"], case["count"])
    pt = O.grid_point(g, case["argmin"])
    assert abs(pt[0]) < 0.01 and abs(pt[1]) < 0.01


ref_needed = pytest.mark.skipif(not O.have_ref(), reason="reference harness not built here")


@ref_needed
@pytest.mark.parametrize("dtype", [np.float32, np.uint8, np.float64])
@pytest.mark.parametrize("cost", ["SAD_AVG", "SAD_AVG_H", "SAD_SUM_T", "SAD_SUM_T_REF", "SQD_REF", "NCC_REF",
                                  "SQD_ALT", "NCC_ALT", "MI_ALT"])
def test_oracle_bit_exact_against_reference(cost, dtype):
    rng = np.random.default_rng(hash((cost, str(dtype))) % 2**32)
    for (h, w, hm, wm, c) in [(21, 26, 19, 23, 1), (16, 16, 16, 16, 3)]:
        if c == 3 and cost in ("SAD_AVG_H", "SAD_SUM_T", "SAD_SUM_T_REF"):
            continue
        if dtype == np.uint8:
            f = rng.integers(0, 256, (h, w, c)).astype(dtype)
            m = rng.integers(0, 256, (hm, wm, c)).astype(dtype)
        else:
            f = rng.uniform(0, 255, (h, w, c)).astype(dtype)
            m = rng.uniform(0, 255, (hm, wm, c)).astype(dtype)
        F, M = O.Image(f), O.Image(m)
        for _ in range(60):
            if cost == "SAD_AVG_H":
                p = np.array([1, 0, 0, 0, 1, 0, 0, 0], np.float32) + rng.uniform(-0.1, 0.1, 8).astype(np.float32)
                p[[2, 5]] = rng.uniform(-4, 4, 2)
                p[6:] = rng.uniform(-2e-3, 2e-3, 2)
            else:
                p = np.array([rng.uniform(-0.3, 0.3), rng.uniform(0.8, 1.2), rng.uniform(0.8, 1.2),
                              rng.uniform(-0.1, 0.1), rng.uniform(-6, 6), rng.uniform(-6, 6),
                              rng.uniform(-2e-3, 2e-3), rng.uniform(-2e-3, 2e-3)], np.float32)
                if cost == "MI_ALT":
                    p[4:6] = rng.uniform(-0.2, 0.2, 2)
                    p[6:] *= 0.01
            a, _ = O.cost(cost, p, M, F)
            b = O.ref_cost(cost, p, M, F)
            assert a == b or (np.isnan(a) and np.isnan(b)), (cost, p, a, b)


@ref_needed
def test_homography_helpers_bit_exact():
    import ctypes as C
    rng = np.random.default_rng(3)
    L, R = O.lib(), O.ref()
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    for _ in range(2000):
        p = np.array([rng.uniform(-3, 3), rng.uniform(0.2, 3), rng.uniform(0.2, 3), rng.uniform(-1, 1),
                      rng.uniform(-100, 100), rng.uniform(-100, 100), rng.uniform(-1e-2, 1e-2),
                      rng.uniform(-1e-2, 1e-2)], np.float32)
        cx, cy = np.float32(rng.integers(1, 600) / 2), np.float32(rng.integers(1, 600) / 2)
        h1, h2 = np.zeros(8, np.float32), np.zeros(8, np.float32)
        L.og_params_to_h(fp(p), cx, cy, fp(h1))
        R.cgsref_params_to_h(fp(p), cx, cy, fp(h2))
        np.testing.assert_array_equal(h1, h2)
        mw, mh, fw, fh = [int(v) for v in rng.integers(2, 700, 4)]
        L.og_params_to_h_norm(fp(p), mw, mh, fw, fh, fp(h1))
        R.cgsref_params_to_h_norm(fp(p), mw, mh, fw, fh, fp(h2))
        np.testing.assert_array_equal(h1, h2)
        x, y = [int(v) for v in rng.integers(0, 700, 2)]
        a, b = C.c_float(), C.c_float()
        c_, d_ = C.c_float(), C.c_float()
        L.og_new_coord(fp(h1), x, y, C.byref(a), C.byref(b))
        R.cgsref_new_coord(fp(h1), x, y, C.byref(c_), C.byref(d_))
        np.testing.assert_array_equal(np.array([a.value, b.value], np.float32),
                                      np.array([c_.value, d_.value], np.float32))  # NaN == NaN here


def test_fp64_oracle_agrees_with_fp32_to_rounding():
    pair = S.small_pair(77, size=32, count=3, cost="NCC_REF")
    g = O.make_grid(*pair.grid_args())
    c32, c64 = O.search("NCC_REF", g, O.Image(pair.moving), O.Image(pair.fixed))
    fin = np.isfinite(c64)
    assert np.max(np.abs(c32[fin] - c64[fin])) < 1e-5
