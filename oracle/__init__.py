"""CPU oracle for the homography grid search -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this package; the product (``cugridsearch_b200``) never does.

Two libraries are wrapped:

* ``_build/libcgs_oracle.so`` -- the plain-C restatement of the reference cost
  functors (``cgs_oracle.c``), with FP32 (reference arithmetic) and FP64-accumulation
  variants.  Always buildable with gcc.
* ``_ref/libcgs_ref.so`` -- the reference's own functor source
  (``src/gpu/cudaErrorFunctions.cuh``, ``cudaErrorFunction_mi.cuh``) compiled for the
  host by ``ref_harness.cu``.  Built where the reference checkout exists and shipped
  prebuilt elsewhere; :func:`have_ref` says whether it is available.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libcgs_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcgs_ref.so")
# The reference checkout, when this machine has one: named by the caller (build(ref_dir=...)) or
# by CGS_REFERENCE_DIR; there is no default location.
REF_SRC = os.environ.get("CGS_REFERENCE_DIR", "")

COSTS = {
    "SAD_AVG": 0, "SAD_AVG_H": 1, "SAD_SUM_T": 2, "SAD_SUM_T_REF": 3, "SQD_REF": 4,
    "NCC_REF": 5, "SQD_ALT": 6, "NCC_ALT": 7, "MI_ALT": 8, "ZNCC": 9, "MI": 10,
}
PIX = {np.dtype(np.float32): 0, np.dtype(np.uint8): 1, np.dtype(np.float64): 2, np.dtype(np.uint16): 3}

_lock = threading.Lock()
_lib = None
_ref = None


class OgImage(C.Structure):
    _fields_ = [("data", C.c_void_p), ("height", C.c_int32), ("width", C.c_int32),
                ("channels", C.c_int32), ("pix", C.c_int32)]


class OgOpts(C.Structure):
    _fields_ = [("mi_bins", C.c_int32), ("overlap_gate", C.c_float)]


class OgGrid(C.Structure):
    _fields_ = [("dims", C.c_int32), ("start", C.c_float * 8), ("end", C.c_float * 8),
                ("resolution", C.c_float * 8), ("count", C.c_float * 8)]


def build(ref_dir: str | None = None) -> None:
    """Build the oracle, and the reference harness when a reference checkout is given
    (``ref_dir``, else CGS_REFERENCE_DIR) and present."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref_dir = ref_dir or REF_SRC
    if ref_dir and os.path.isdir(os.path.join(ref_dir, "src", "gpu")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_dir}"], check=True)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(ORACLE_SO):
                subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
            L = C.CDLL(ORACLE_SO)
            P = C.POINTER
            L.og_cost_f32.restype = C.c_float
            L.og_cost_f32.argtypes = [C.c_int, P(C.c_float), P(OgImage), P(OgImage), P(OgOpts), P(C.c_int64)]
            L.og_cost_f64.restype = C.c_double
            L.og_cost_f64.argtypes = [C.c_int, P(C.c_float), P(OgImage), P(OgImage), P(OgOpts), P(C.c_int64)]
            L.og_histogram.restype = C.c_int64
            L.og_histogram.argtypes = [C.c_int, P(C.c_float), P(OgImage), P(OgImage), P(OgOpts), P(C.c_uint32)]
            L.og_grid_update.argtypes = [P(OgGrid), C.c_int]
            L.og_grid_num_elements.restype = C.c_int64
            L.og_grid_num_elements.argtypes = [P(OgGrid)]
            L.og_grid_increments.argtypes = [P(OgGrid), P(C.c_int32)]
            L.og_grid_point.argtypes = [P(OgGrid), C.c_int64, C.c_int, P(C.c_float)]
            L.og_params_to_h.argtypes = [P(C.c_float), C.c_float, C.c_float, P(C.c_float)]
            L.og_params_to_h_uncentred.argtypes = [P(C.c_float), P(C.c_float)]
            L.og_params_to_h_norm.argtypes = [P(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_float)]
            L.og_new_coord.argtypes = [P(C.c_float), C.c_int, C.c_int, P(C.c_float), P(C.c_float)]
            L.og_bilinear_probe.argtypes = [P(OgImage), C.c_float, C.c_float, C.c_int, P(C.c_float)]
            L.og_covariance.argtypes = [P(OgGrid), P(C.c_float), C.c_int64, P(C.c_double), P(C.c_float)]
            L.og_search.restype = C.c_int
            L.og_search.argtypes = [C.c_int, P(OgGrid), C.c_int, P(OgImage), P(OgImage), P(OgOpts),
                                    C.c_int64, C.c_int64, C.c_int64, P(C.c_float), P(C.c_double), C.c_int]
            _lib = L
    return _lib


def have_ref() -> bool:
    if os.path.exists(REF_SO):
        return True
    if REF_SRC and os.path.isdir(os.path.join(REF_SRC, "src", "gpu")):
        try:
            subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)
        except Exception:
            return False
        return os.path.exists(REF_SO)
    return False


def ref():
    global _ref
    with _lock:
        if _ref is None:
            L = C.CDLL(REF_SO)
            P = C.POINTER
            L.cgsref_eval.restype = C.c_float
            L.cgsref_eval.argtypes = [C.c_int, P(C.c_float), C.c_int, C.c_void_p, C.c_int, C.c_int,
                                      C.c_void_p, C.c_int, C.c_int, C.c_int]
            L.cgsref_params_to_h.argtypes = [P(C.c_float), C.c_float, C.c_float, P(C.c_float)]
            L.cgsref_params_to_h_norm.argtypes = [P(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_float)]
            L.cgsref_new_coord.argtypes = [P(C.c_float), C.c_int, C.c_int, P(C.c_float), P(C.c_float)]
            L.cgsref_bilinear.restype = C.c_float
            L.cgsref_bilinear.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float]
            L.cgsref_search.restype = C.c_int
            L.cgsref_search.argtypes = [C.c_int, C.c_int, P(C.c_float), P(C.c_float), P(C.c_float), C.c_int,
                                        C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                        C.c_int, C.c_int64, C.c_int64, C.c_int64, P(C.c_float), C.c_int]
            L.cgsref_max_threads.restype = C.c_int
            L.cgsref_device_grid_points.restype = C.c_int
            L.cgsref_device_grid_points.argtypes = [C.c_int, P(C.c_float), P(C.c_float), P(C.c_float),
                                                    P(C.c_int64), C.c_int, P(C.c_float), P(C.c_float)]
            _ref = L
    return _ref


# ----------------------------------------------------------------------------- helpers

def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def as_hwc(img: np.ndarray) -> np.ndarray:
    img = np.ascontiguousarray(img)
    if img.ndim == 2:
        img = img[:, :, None]
    if img.dtype not in PIX:
        raise TypeError(f"unsupported pixel type {img.dtype}")
    return img


class Image:
    """Host image in CudaImage layout (HWC row-major) for the oracle libraries."""

    def __init__(self, img: np.ndarray):
        self.arr = as_hwc(img)
        h, w, c = self.arr.shape
        self.og = OgImage(self.arr.ctypes.data, h, w, c, PIX[self.arr.dtype])
        # zero-padded copy for the reference harness: one extra row plus one pixel
        pad = np.zeros((h + 1) * w * c + c, dtype=self.arr.dtype)
        pad[: h * w * c] = self.arr.reshape(-1)
        self.padded = pad


def opts(mi_bins: int = 32, overlap_gate: float = 0.0) -> OgOpts:
    return OgOpts(mi_bins, overlap_gate)


def cost(name: str, params, mov: Image, fix: Image, o: OgOpts | None = None, f64: bool = False):
    p = np.ascontiguousarray(params, dtype=np.float32)
    n = C.c_int64(0)
    o = o or opts()
    fn = lib().og_cost_f64 if f64 else lib().og_cost_f32
    v = fn(COSTS[name], _fptr(p), C.byref(mov.og), C.byref(fix.og), C.byref(o), C.byref(n))
    return v, n.value


def histogram(name: str, params, mov: Image, fix: Image, o: OgOpts | None = None) -> tuple[np.ndarray, int]:
    o = o or opts()
    bins = 64 if name == "MI_ALT" else o.mi_bins
    h = np.zeros(bins * bins, dtype=np.uint32)
    p = np.ascontiguousarray(params, dtype=np.float32)
    n = lib().og_histogram(COSTS[name], _fptr(p), C.byref(mov.og), C.byref(fix.og), C.byref(o),
                           h.ctypes.data_as(C.POINTER(C.c_uint32)))
    return h.reshape(bins, bins), int(n)


def make_grid(start, end, count) -> OgGrid:
    """Grid set up as CudaGrid::setStartPoint/EndPoint/NumSamples do (each calls update())."""
    d = len(start)
    g = OgGrid()
    g.dims = d
    for a in range(d):
        g.start[a] = float(start[a]); g.end[a] = float(end[a]); g.count[a] = float(count[a])
    lib().og_grid_update(C.byref(g), -1)
    return g


def grid_num(g: OgGrid) -> int:
    return int(lib().og_grid_num_elements(C.byref(g)))


def grid_point(g: OgGrid, index: int, use_fma: bool = True) -> np.ndarray:
    out = np.zeros(8, dtype=np.float32)
    lib().og_grid_point(C.byref(g), int(index), int(use_fma), _fptr(out))
    return out


def search(name: str, g: OgGrid, mov: Image, fix: Image, o: OgOpts | None = None, first: int = 0,
           count: int | None = None, stride: int = 1, f32: bool = True, f64: bool = True,
           threads: int = 0, use_fma: bool = True):
    """Costs of the grid points first, first+stride, ... (count of them) on the CPU."""
    o = o or opts()
    if count is None:
        count = (grid_num(g) - first + stride - 1) // stride
    c32 = np.zeros(count, dtype=np.float32) if f32 else None
    c64 = np.zeros(count, dtype=np.float64) if f64 else None
    rc = lib().og_search(COSTS[name], C.byref(g), int(use_fma), C.byref(mov.og), C.byref(fix.og), C.byref(o),
                         first, count, stride,
                         _fptr(c32) if f32 else None,
                         c64.ctypes.data_as(C.POINTER(C.c_double)) if f64 else None, threads)
    if rc != 0:
        raise ValueError("og_search rejected its arguments")
    return c32, c64


def covariance(g: OgGrid, costs: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(double-accumulated, reference float-accumulated) covariance of a cost array."""
    c = np.ascontiguousarray(costs, dtype=np.float32)
    d = g.dims
    o64 = np.zeros(d * d, dtype=np.float64)
    o32 = np.zeros(d * d, dtype=np.float32)
    lib().og_covariance(C.byref(g), _fptr(c), c.size, o64.ctypes.data_as(C.POINTER(C.c_double)), _fptr(o32))
    return o64.reshape(d, d), o32.reshape(d, d)


def ref_cost(name: str, params, mov: Image, fix: Image) -> float:
    p = np.ascontiguousarray(params, dtype=np.float32)
    h, w, c = fix.arr.shape
    mh, mw, _ = mov.arr.shape
    return ref().cgsref_eval(COSTS[name], _fptr(p), PIX[mov.arr.dtype], mov.padded.ctypes.data, mh, mw,
                             fix.padded.ctypes.data, h, w, c)


def ref_device_grid_points(start, end, count, indices):
    """Grid points decoded by the reference's own CudaGrid on the GPU (dims 2 or 8, counts >= 2):
    (points[n, dims], matrix[4, dims] = start, end, resolution, count after the updates)."""
    d = len(start)
    st, en, ct = (np.ascontiguousarray(v, dtype=np.float32) for v in (start, end, count))
    idx = np.ascontiguousarray(indices, dtype=np.int64)
    out = np.zeros((len(idx), d), dtype=np.float32)
    mat = np.zeros((4, d), dtype=np.float32)
    rc = ref().cgsref_device_grid_points(d, _fptr(st), _fptr(en), _fptr(ct),
                                         idx.ctypes.data_as(C.POINTER(C.c_int64)), len(idx), _fptr(out), _fptr(mat))
    if rc != 0:
        raise RuntimeError(f"cgsref_device_grid_points failed ({rc})")
    return out, mat


def ref_search(name: str, g: OgGrid, mov: Image, fix: Image, first: int = 0, count: int | None = None,
               stride: int = 1, threads: int = 0, use_fma: bool = True) -> np.ndarray:
    if count is None:
        count = (grid_num(g) - first + stride - 1) // stride
    out = np.zeros(count, dtype=np.float32)
    h, w, c = fix.arr.shape
    mh, mw, _ = mov.arr.shape
    start = np.array(list(g.start), dtype=np.float32)
    res = np.array(list(g.resolution), dtype=np.float32)
    cnt = np.array(list(g.count), dtype=np.float32)
    ref().cgsref_search(COSTS[name], g.dims, _fptr(start), _fptr(res), _fptr(cnt), int(use_fma),
                        PIX[mov.arr.dtype], mov.padded.ctypes.data, mh, mw, fix.padded.ctypes.data, h, w, c,
                        first, count, stride, _fptr(out), threads)
    return out
