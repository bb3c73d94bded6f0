"""The drop-in template headers on the CPU (include/cugridsearch/; no GPU needed).

The functor bodies of the drop-in headers run when a caller invokes a functor directly
(on the host, like the reference's "Min Value check") and on the device for instantiations
the library has no fused kernel for.  Here they are compiled for the host
(tests/native/dropin_host.cu) and pinned:
  * the reference functors bit for bit against the reference's own functor source
    (oracle/_ref) -- or, where the reference is absent, against the oracle, which is itself
    pinned bit for bit to the reference and to the golden vectors;
  * calcZNCC / calcMI against the oracle's FP64 definitions;
  * the block-cooperative functors (computed here by one thread) against the oracle's
    equivalent formulas, within FP32 summation-order tolerance.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "tests", "native")
SO = os.path.join(NATIVE, "_build", "libdropin_host.so")
PIX = {np.dtype(np.float32): 0, np.dtype(np.uint8): 1, np.dtype(np.float64): 2, np.dtype(np.uint16): 3}
CODES = dict(O.COSTS, SAD_STREAM=100, NCC_STREAM=101, NCC_STREAM_ALT=102, SQD_STREAM=103, MI_STREAM=104,
             MI_STREAM_ALT=105)

_lib = None


def dropin():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            from cugridsearch_b200 import build
            build.build()
            subprocess.run(["make", "-s", "-C", NATIVE, SO], check=True)
        L = C.CDLL(SO)
        L.dropin_eval.restype = C.c_float
        L.dropin_eval.argtypes = [C.c_int, C.POINTER(C.c_float), C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                  C.c_int, C.c_int, C.c_int]
        L.dropin_params_to_h.argtypes = [C.POINTER(C.c_float), C.c_float, C.c_float, C.POINTER(C.c_float)]
        _lib = L
    return _lib


def ev(name, p, M: O.Image, F: O.Image) -> float:
    p = np.ascontiguousarray(p, dtype=np.float32)
    h, w, c = F.arr.shape
    mh, mw, _ = M.arr.shape
    return dropin().dropin_eval(CODES[name], p.ctypes.data_as(C.POINTER(C.c_float)), PIX[M.arr.dtype],
                                M.padded.ctypes.data, mh, mw, F.padded.ctypes.data, h, w, c)


def random_params(rng, cost):
    if cost == "SAD_AVG_H":
        p = np.array([1, 0, 0, 0, 1, 0, 0, 0], np.float32) + rng.uniform(-0.1, 0.1, 8).astype(np.float32)
        p[[2, 5]] = rng.uniform(-4, 4, 2)
        p[6:] = rng.uniform(-2e-3, 2e-3, 2)
        return p
    p = np.array([rng.uniform(-0.3, 0.3), rng.uniform(0.8, 1.2), rng.uniform(0.8, 1.2), rng.uniform(-0.1, 0.1),
                  rng.uniform(-6, 6), rng.uniform(-6, 6), rng.uniform(-2e-3, 2e-3), rng.uniform(-2e-3, 2e-3)],
                 np.float32)
    if cost == "MI_ALT":
        p[4:6] = rng.uniform(-0.2, 0.2, 2)
        p[6:] *= 0.01
    return p


def images(rng, dtype, shape_f, shape_m):
    if dtype == np.uint8:
        return (O.Image(rng.integers(0, 256, shape_m).astype(dtype)), O.Image(rng.integers(0, 256, shape_f).astype(dtype)))
    return (O.Image(rng.uniform(0, 255, shape_m).astype(dtype)), O.Image(rng.uniform(0, 255, shape_f).astype(dtype)))


def test_dropin_homography_matches_reference_helper():
    rng = np.random.default_rng(7)
    for _ in range(200):
        p = random_params(rng, "NCC_REF")
        cx, cy = np.float32(rng.uniform(5, 300)), np.float32(rng.uniform(5, 300))
        a = np.zeros(8, np.float32)
        b = np.zeros(8, np.float32)
        dropin().dropin_params_to_h(p.ctypes.data_as(C.POINTER(C.c_float)), cx, cy, a.ctypes.data_as(C.POINTER(C.c_float)))
        if O.have_ref():
            O.ref().cgsref_params_to_h(p.ctypes.data_as(C.POINTER(C.c_float)), cx, cy, b.ctypes.data_as(C.POINTER(C.c_float)))
        else:
            O.lib().og_params_to_h(p.ctypes.data_as(C.POINTER(C.c_float)), cx, cy, b.ctypes.data_as(C.POINTER(C.c_float)))
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("dtype", [np.float32, np.uint8, np.float64])
@pytest.mark.parametrize("cost", ["SAD_AVG", "SAD_AVG_H", "SAD_SUM_T", "SAD_SUM_T_REF", "SQD_REF", "NCC_REF",
                                  "SQD_ALT", "NCC_ALT", "MI_ALT"])
def test_dropin_functors_bit_exact_against_reference(cost, dtype):
    """The drop-in body of each reference functor returns the reference's FP32 value."""
    rng = np.random.default_rng(abs(hash((cost, str(dtype), "dropin"))) % 2**32)
    for (h, w, hm, wm, c) in [(21, 26, 19, 23, 1), (16, 16, 16, 16, 3)]:
        if c == 3 and cost in ("SAD_AVG_H", "SAD_SUM_T", "SAD_SUM_T_REF"):
            continue
        M, F = images(rng, dtype, (h, w, c), (hm, wm, c))
        for _ in range(25):
            p = random_params(rng, cost)
            a = ev(cost, p, M, F)
            b = O.ref_cost(cost, p, M, F) if O.have_ref() else O.cost(cost, p, M, F)[0]
            assert a == b or (np.isnan(a) and np.isnan(b)), (cost, p, a, b)


@pytest.mark.parametrize("cost", ["ZNCC", "MI"])
def test_dropin_zncc_mi_match_oracle_fp64(cost):
    rng = np.random.default_rng(11 if cost == "ZNCC" else 12)
    for dtype in (np.float32, np.uint8):
        M, F = images(rng, dtype, (24, 28, 1), (22, 25, 1))
        for _ in range(30):
            p = random_params(rng, cost)
            a = ev(cost, p, M, F)
            b, _ = O.cost(cost, p, M, F, o=O.opts(mi_bins=32), f64=True)
            if not np.isfinite(b):
                assert a == b
            else:
                assert abs(a - b) <= 1e-6 * max(1.0, abs(b)), (p, a, b)


def _nmi(hist):
    h = hist.astype(np.float64)
    n = h.sum()
    if n == 0:
        return np.nan
    pxy = h / n
    px, py = pxy.sum(1), pxy.sum(0)
    nz = pxy > 0
    mi = (pxy[nz] * (np.log2(pxy[nz]) - np.log2(np.outer(px, py)[nz]))).sum()
    hx = -(px[px > 0] * np.log2(px[px > 0])).sum()
    hy = -(py[py > 0] * np.log2(py[py > 0])).sum()
    return -2 * mi / (hx + hy)


def test_dropin_block_functors_match_their_formulas():
    """The reference's block-cooperative functors, computed by one thread: each agrees with
    the oracle's evaluation of the same formula (row-partial FP32 sums vs FP64)."""
    rng = np.random.default_rng(5)
    M, F = images(rng, np.float32, (20, 24, 1), (20, 24, 1))
    checked = {k: 0 for k in ("SAD_STREAM", "NCC_STREAM", "SQD_STREAM", "NCC_STREAM_ALT", "MI_STREAM")}
    for _ in range(40):
        p = random_params(rng, "NCC_REF")
        # translation mean |m - f| over the overlap (count 0 -> 0)
        s, n = O.cost("SAD_SUM_T", p, M, F, f64=True)
        a = ev("SAD_STREAM", p, M, F)
        assert abs(a - s / max(n, 1)) <= 1e-5 * max(1.0, abs(s / max(n, 1)))
        checked["SAD_STREAM"] += 1
        ncc, n = O.cost("NCC_REF", p, M, F, f64=True)
        if n > 0:
            assert abs(ev("NCC_STREAM", p, M, F) - ncc) <= 1e-5
            checked["NCC_STREAM"] += 1
        sqd, n = O.cost("SQD_REF", p, M, F, f64=True)
        if n > 0:
            assert abs(ev("SQD_STREAM", p, M, F) - sqd) <= 1e-5 * max(1e-3, abs(sqd))
            checked["SQD_STREAM"] += 1
        else:
            assert np.isnan(ev("SQD_STREAM", p, M, F))
        alt, _ = O.cost("NCC_ALT", p, M, F, f64=True)
        b = ev("NCC_STREAM_ALT", p, M, F)
        if alt == 123123.0:
            assert b == 0.0
        else:
            assert abs(b - alt) <= 1e-5
            checked["NCC_STREAM_ALT"] += 1
        hist, n = O.histogram("MI", p, M, F, O.opts(mi_bins=64))
        if n > 0:
            assert abs(ev("MI_STREAM", p, M, F) - _nmi(hist)) <= 1e-4
            checked["MI_STREAM"] += 1
        v = ev("MI_STREAM_ALT", p, M, F)
        assert v == 123123.0 or (-1.0001 <= v <= 1e-6)
    assert all(v > 5 for v in checked.values()), checked
