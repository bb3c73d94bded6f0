"""A program written against the reference's template API, on the GPU.

tests/native/dropin_main.cu declares __device__ functor pointers exactly as the reference's
drivers do (src/gpu/cudaGridSearch_main_mi.cu:78-81, cudaGridSearch_example1.cu:36-44,
example2.cu:40-41), fetches them with cudaMemcpyFromSymbol and runs CudaGridSearcher,
CudaTensor::find_extrema and CudaGrid::getGridPoint from the drop-in headers.  Checked here:
  * which path ran: known functors with a library kernel take the fused kernel; the
    block-cooperative functors and known functors on pixel types without a kernel take
    the direct-call kernel; a caller's own functor takes the function-pointer kernel;
  * the cost tensor against the oracle (FP64, parity tolerance) or, for the direct and
    pointer paths, against the drop-in bodies evaluated on the host;
  * find_extrema / getGridPoint against the tensor and the oracle's grid decode;
  * covariance_by_value against the oracle's FP64 restatement.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import close_costs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "tests", "native")
BIN = os.path.join(NATIVE, "_build", "dropin_main")

R8 = dict(lo=[-0.1, 0.9, 0.9, -0.05, -3, -3, -5e-4, -5e-4], hi=[0.1, 1.1, 1.1, 0.05, 3, 3, 5e-4, 5e-4])
RH = dict(lo=[0.95, -0.05, -2, -0.05, 0.95, -2, -5e-4, -5e-4], hi=[1.05, 0.05, 2, 0.05, 1.05, 2, 5e-4, 5e-4])
RM = dict(lo=[-0.1, 0.9, 0.9, -0.05, -0.1, -0.1, -5e-6, -5e-6], hi=[0.1, 1.1, 1.1, 0.05, 0.1, 0.1, 5e-6, 5e-6])


def _pair(rng, dtype, c=1, size=(20, 24), msize=(21, 23), smooth=True):
    yy, xx = np.mgrid[0:64, 0:64].astype(np.float64)
    base = 120 + 60 * np.sin(xx / 5.0) * np.cos(yy / 7.0) + 30 * np.cos((xx + 2 * yy) / 9.0)

    def img(h, w, off):
        a = base[off:off + h, off:off + w]
        a = np.repeat(a[:, :, None], c, axis=2) + rng.normal(0, 4, (h, w, c))
        a = np.clip(a, 0, 255)
        return a.astype(dtype) if dtype != np.uint8 else np.round(a).astype(np.uint8)

    return img(msize[0], msize[1], 2), img(size[0], size[1], 0)


CASES = [
    # name, functor, pixel, channels, dims, ranges, count, method, expected path, oracle cost
    ("ncc", "ncc", "f32", 1, 8, R8, 3, "value", "fused", "NCC_REF"),
    ("sqd", "sqd", "f32", 1, 8, R8, 3, "block", "fused", "SQD_REF"),
    ("sad", "sad", "f32", 1, 8, dict(lo=[-0.1, 0.9, 0.9, -0.05, -3, -3, -5e-4, -5e-4],
                                     hi=[0.1, 1.1, 1.1, 0.05, 3, 3, 5e-4, 5e-4]), 3, "stream", "fused", "SAD_AVG"),
    ("sadh", "sadh", "f32", 1, 8, RH, 3, "value", "fused", "SAD_AVG_H"),
    ("ncc_alt", "ncc_alt", "f32", 1, 8, R8, 3, "value", "fused", "NCC_ALT"),
    ("sqd_alt", "sqd_alt", "f32", 1, 8, R8, 3, "value", "fused", "SQD_ALT"),
    ("mi_alt", "mi_alt", "f32", 1, 8, RM, 3, "value", "fused", "MI_ALT"),
    ("zncc", "zncc", "f32", 1, 8, R8, 3, "value", "fused", "ZNCC"),
    ("mi", "mi", "f32", 1, 8, R8, 3, "value", "fused", "MI"),
    ("mi16", "mi16", "f32", 1, 8, R8, 3, "value", "fused", "MI16"),
    ("u8_ncc", "ncc", "u8", 3, 8, R8, 3, "value", "fused", "NCC_REF"),
    ("u8_mi_alt", "mi_alt", "u8", 3, 8, RM, 3, "value", "fused", "MI_ALT"),
    ("u8_mi", "mi", "u8", 3, 8, R8, 3, "value", "fused", "MI"),
    ("ncc_stream", "ncc_stream", "f32", 1, 8, R8, 2, "stream", "direct", "NCC_STREAM"),
    ("sqd_stream", "sqd_stream", "f32", 1, 8, R8, 2, "stream", "direct", "SQD_STREAM"),
    ("ncc_stream_alt", "ncc_stream_alt", "f32", 1, 8, R8, 2, "stream", "direct", "NCC_STREAM_ALT"),
    ("mi_stream", "mi_stream", "f32", 1, 8, R8, 2, "stream", "direct", "MI_STREAM"),
    ("mi_stream_alt", "mi_stream_alt", "f32", 1, 8, R8, 2, "stream", "direct", "MI_STREAM_ALT"),
    ("user", "user_ncc", "f32", 1, 8, R8, 2, "value", "pointer", "USER"),
    ("i16_ncc", "ncc", "i16", 1, 8, R8, 2, "value", "direct", "NCC_REF"),
    ("sad_t", "sad_t", "f64", 1, 2, dict(lo=[-3, -3], hi=[3, 3]), (103, 111), "value", "fused", "SAD_SUM_T"),
    ("sad_t_ref", "sad_t", "f64", 1, 2, dict(lo=[-3, -3], hi=[3, 3]), (103, 111), "ref", "fused", "SAD_SUM_T_REF"),
    ("sad_stream", "sad_stream", "f64", 1, 2, dict(lo=[-3, -3], hi=[3, 3]), (57, 61), "stream", "direct",
     "SAD_STREAM"),
    ("cov", "ncc", "f32", 1, 8, R8, 3, "cov", "fused", "NCC_REF"),
]
DT = {"f32": np.float32, "f64": np.float64, "u8": np.uint8, "i16": np.int16}


@pytest.fixture(scope="module")
def outputs(tmp_path_factory, cuda, lib):
    if not os.path.exists(BIN):
        subprocess.run(["make", "-s", "-C", NATIVE, BIN], check=True)
    d_in = tmp_path_factory.mktemp("dropin_in")
    d_out = tmp_path_factory.mktemp("dropin_out")
    rng = np.random.default_rng(20261203)
    inputs = {}
    lines = []
    for (name, fn, pix, c, dims, rg, count, method, _, _) in CASES:
        mov, fix = _pair(rng, DT[pix], c)
        mov.tofile(d_in / f"{name}_mov.bin")
        fix.tofile(d_in / f"{name}_fix.bin")
        cnt = list(count) if isinstance(count, tuple) else [count] * dims
        inputs[name] = (mov, fix, rg["lo"], rg["hi"], cnt)
        vals = [name, fn, pix, c, dims, mov.shape[0], mov.shape[1], fix.shape[0], fix.shape[1], method]
        vals += [repr(float(v)) for v in rg["lo"]] + [repr(float(v)) for v in rg["hi"]] + [str(v) for v in cnt]
        lines.append(" ".join(str(v) for v in vals))
    (d_in / "cases.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([BIN, str(d_in), str(d_out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = {}
    for case in CASES:
        name = case[0]
        txt = (d_out / f"{name}.txt").read_text().split()
        out[name] = (txt, np.fromfile(d_out / f"{name}_costs.bin", dtype=np.float32))
    return inputs, out


def _host_dropin(name, pts, M, F):
    from test_dropin_cpu import ev
    return np.array([ev(name, p, M, F) for p in pts], dtype=np.float64)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_dropin_program(outputs, case):
    name, fn, pix, c, dims, rg, count, method, path, ocost = case
    inputs, out = outputs
    mov, fix, lo, hi, cnt = inputs[name]
    txt, gpu = out[name]
    assert txt[0] == path, f"{name} ran on the {txt[0]} path"
    g = O.make_grid(lo, hi, cnt)
    n = O.grid_num(g)
    assert gpu.size == n
    if pix == "i16":  # no oracle pixel type: the same values as float32
        mov, fix = mov.astype(np.float32), fix.astype(np.float32)
    M, F = O.Image(mov), O.Image(fix)
    pts = np.array([O.grid_point(g, i) for i in range(n)], dtype=np.float32)
    if ocost in O.COSTS or ocost == "MI16":
        oc = "MI" if ocost == "MI16" else ocost
        o = O.opts(mi_bins=16 if ocost == "MI16" else 32)
        c32, c64 = O.search(oc, g, M, F, o=o)
        if path == "fused":
            bad = close_costs(gpu, c32, c64, oc)
        else:  # the functor body compiled for the device (FMA contraction): FP32 rounding apart
            bad = close_costs(gpu, c32, c64, oc, rel=1e-4)
        assert not bad.any(), f"{int(bad.sum())} of {n} costs out of tolerance"
    elif ocost == "USER":
        _, c64 = O.search("NCC_REF", g, M, F)
        np.testing.assert_allclose(gpu, 0.5 * c64, rtol=1e-4, atol=1e-5)
    else:  # block-cooperative functors: their single-thread body on the host
        ref = _host_dropin(ocost, pts, M, F)
        special = ~np.isfinite(ref) | (ref == 123123.0)
        ok = np.isclose(gpu, ref, rtol=1e-4, atol=1e-5) | (np.isnan(gpu) & np.isnan(ref)) | (gpu == ref)
        if ocost in ("NCC_STREAM_ALT", "MI_STREAM_ALT"):
            # scanline sampling: the entry-point formulas cancel heavily, so a last-bit
            # difference of the device's cos / sin can move a row's samples (the program is
            # built with -fmad=false: with contraction, half of these costs moved by up to
            # 1e-3 relative -- the reference's own device and host builds disagree as much)
            assert ok.mean() >= 0.98, f"{int((~ok).sum())} of {n} differ"
        else:
            assert ok.all(), f"{int((~ok).sum())} of {n} differ"
        assert np.array_equal(np.isnan(gpu[special]), np.isnan(ref[special]))
    # find_extrema: lowest value, lowest index among equals; getGridPoint of that index
    idx, best = int(txt[1]), float(txt[2])
    fin = np.where(np.isfinite(gpu), gpu, np.inf)
    if np.isfinite(fin).any():
        assert idx == int(np.argmin(fin)) and np.float32(best) == gpu[idx]
    point = np.array([float(v) for v in txt[3:3 + dims]], dtype=np.float32)
    np.testing.assert_array_equal(point, O.grid_point(g, idx)[:dims])
    if method == "cov":
        cov = np.array([float(v) for v in txt[3 + dims:]], dtype=np.float64).reshape(dims, dims)
        want, _ = O.covariance(g, gpu)
        np.testing.assert_allclose(cov, want, rtol=2e-6, atol=1e-6 * max(1.0, np.abs(want).max()))
