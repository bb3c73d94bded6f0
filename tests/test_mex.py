"""The MATLAB entry point (cugridsearch_b200/mex/cudaGridSearch_mex.cpp) through an
in-process stand-in for MATLAB's mx runtime (tests/native/mex_stub; MATLAB is not installed).

CPU: argument checking -- every malformed call raises through mexErrMsgIdAndTxt before any
device work.  GPU: the MEX call agrees with the library's own search on the same images
(MATLAB column-major images are transposed to the CudaImage layout; the cost volume comes
back as a count(1) x ... x count(D) single array in the reference's index order)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "tests", "native")
SO = os.path.join(NATIVE, "_build", "libcgs_mex_test.so")
CLS = {np.dtype(np.float64): 6, np.dtype(np.float32): 7, np.dtype(np.uint8): 9, np.dtype(np.uint16): 11,
       np.dtype(np.int32): 12}
NP = {6: np.float64, 7: np.float32, 9: np.uint8, 11: np.uint16}

_lib = None


def mexlib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            from cugridsearch_b200 import build
            build.build()
            subprocess.run(["make", "-s", "-C", NATIVE, SO], check=True)
        L = C.CDLL(SO)
        L.fake_mx_numeric.restype = C.c_void_p
        L.fake_mx_numeric.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64), C.c_void_p]
        L.fake_mx_string.restype = C.c_void_p
        L.fake_mx_string.argtypes = [C.c_char_p]
        L.fake_mx_destroy.argtypes = [C.c_void_p]
        L.fake_mx_class.argtypes = [C.c_void_p]
        L.fake_mx_ndim.argtypes = [C.c_void_p]
        L.fake_mx_dim.restype = C.c_uint64
        L.fake_mx_dim.argtypes = [C.c_void_p, C.c_int]
        L.fake_mx_data.restype = C.c_void_p
        L.fake_mx_data.argtypes = [C.c_void_p]
        L.fake_mex_call.restype = C.c_char_p
        L.fake_mex_call.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
        _lib = L
    return _lib


def to_mx(v):
    L = mexlib()
    if isinstance(v, str):
        return L.fake_mx_string(v.encode())
    a = v if isinstance(v, np.ndarray) else np.asarray(v, dtype=np.float64)  # MATLAB literals are double
    if a.ndim == 0 or a.ndim == 1:
        a = a.reshape(1, -1)  # MATLAB row vector
    dims = (C.c_uint64 * a.ndim)(*a.shape)
    f = np.asfortranarray(a)  # MATLAB stores column-major
    return L.fake_mx_numeric(CLS[a.dtype], a.ndim, dims, f.ctypes.data)


def from_mx(p):
    L = mexlib()
    cls = L.fake_mx_class(p)
    shape = tuple(L.fake_mx_dim(p, i) for i in range(L.fake_mx_ndim(p)))
    n = int(np.prod(shape))
    dt = np.dtype(NP[cls])
    raw = C.string_at(L.fake_mx_data(p), n * dt.itemsize)
    return np.frombuffer(raw, dtype=dt).reshape(shape, order="F").copy()


def mex(nlhs, *args):
    """Calls mexFunction; returns the outputs, or raises RuntimeError with MATLAB's message."""
    L = mexlib()
    prhs = (C.c_void_p * len(args))(*[to_mx(a) for a in args])
    plhs = (C.c_void_p * max(nlhs, 1))()
    err = L.fake_mex_call(nlhs, plhs, len(args), prhs)
    for p in prhs:
        L.fake_mx_destroy(p)
    if err:
        raise RuntimeError(err.decode())
    out = [from_mx(plhs[i]) for i in range(nlhs)]
    for i in range(nlhs):
        L.fake_mx_destroy(plhs[i])
    return out


GRID8 = ([-0.1, 0.9, 0.9, -0.05, -3, -3, -5e-4, -5e-4], [0.1, 1.1, 1.1, 0.05, 3, 3, 5e-4, 5e-4], [3] * 8)


def _imgs(dtype, shape=(20, 24), c=1, seed=0):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:shape[0] + 2, 0:shape[1] + 2]
    base = 120 + 60 * np.sin(xx / 5.0) * np.cos(yy / 7.0)
    f = base[:shape[0], :shape[1]]
    m = base[1:shape[0] + 1, 2:shape[1] + 2]
    if c > 1:
        f = np.repeat(f[:, :, None], c, 2)
        m = np.repeat(m[:, :, None], c, 2)
    f = f + rng.normal(0, 3, f.shape)
    m = m + rng.normal(0, 3, m.shape)
    if dtype == np.uint8:
        return np.clip(np.round(f), 0, 255).astype(dtype), np.clip(np.round(m), 0, 255).astype(dtype)
    return f.astype(dtype), m.astype(dtype)


@pytest.mark.parametrize("args, msg", [
    ((), "usage"),
    (("x", "y", 1, 2, 3, "NCC_REF"), "fixed must be double, single, uint8 or uint16"),
    ((np.zeros((4, 4)), np.zeros((4, 4), np.float32), [0], [1], [2], "NCC_REF"), "same class"),
    ((np.zeros((4, 4)), np.zeros((4, 4, 3)), [0], [1], [2], "NCC_REF"), "same number of channels"),
    ((np.zeros((4, 4)), np.zeros((4, 4)), [0, 0], [1], [2], "NCC_REF"), "same length"),
    ((np.zeros((4, 4)), np.zeros((4, 4)), [0], [1], [2], "nope"), "unknown cost 'nope'"),
    ((np.zeros((4, 4)), np.zeros((4, 4)), [0], [1], [2], 5.0), "costName must be a string"),
    ((np.zeros((4, 4)), np.zeros((4, 4)), np.zeros(9), np.zeros(9), np.zeros(9), "NCC_REF"), "1 to 8"),
    ((np.zeros((4, 4), np.int32), np.zeros((4, 4), np.int32), [0], [1], [2], "NCC_REF"), "must be double"),
])
def test_mex_rejects_bad_calls(args, msg):
    with pytest.raises(RuntimeError, match="cudaGridSearch:error") as e:
        mex(4, *args)
    assert msg in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("cost, dtype, c", [("NCC_REF", np.float32, 1), ("calcMIAlt", np.uint8, 3), ("MI", np.uint8, 3),
                                            ("ZNCC", np.float64, 1), ("averageAbsoluteDifference", np.uint16, 1)])
def test_mex_matches_library_search(cuda, lib, cost, dtype, c):
    import torch
    import cugridsearch_b200 as cgs
    fix, mov = _imgs(dtype, c=c)
    start, end, count = GRID8
    if cost == "calcMIAlt":
        start, end = list(start), list(end)
        start[4:6], end[4:6] = [-0.1, -0.1], [0.1, 0.1]
    idx, best, params, costs = mex(4, fix, mov, np.array(start), np.array(end), np.array(count, float), cost)
    name = {"calcMIAlt": "MI_ALT", "averageAbsoluteDifference": "SAD_AVG"}.get(cost, cost)
    grid = cgs.CudaGrid.from_ranges(start, end, count)
    n = grid.numElements()
    dc = torch.empty(n, dtype=torch.float32, device=cuda)
    r = cgs.search(name, cgs.CudaImage(torch.from_numpy(mov).to(cuda)), cgs.CudaImage(torch.from_numpy(fix).to(cuda)),
                   grid, costs=dc)
    want = dc.cpu().numpy()
    assert costs.shape == tuple(count) and costs.dtype == np.float32
    np.testing.assert_array_equal(costs.reshape(-1, order="F"), want)  # axis 0 fastest, as MATLAB
    assert int(idx.item()) == r.index + 1
    assert np.float32(best.item()) == np.float32(r.cost)
    np.testing.assert_array_equal(params.reshape(-1).astype(np.float32), np.asarray(r.params[:8], np.float32))


@pytest.mark.gpu
def test_mex_translation_grid_and_flat_volume(cuda, lib):
    fix, mov = _imgs(np.float64, (6, 6))
    idx, best, params, costs = mex(4, fix, mov, np.array([-3.0, -3.0]), np.array([3.0, 3.0]),
                                   np.array([103.0, 111.0]), "sumOfAbsoluteDifferences")
    assert costs.shape == (103, 111)
    flat = costs.reshape(-1, order="F")
    assert int(idx.item()) == int(np.argmin(flat)) + 1 and np.float32(best.item()) == flat.min()
    # fractional counts (allowed by the reference): 7.5 x 9 still decodes as a 7 x 9 box, but
    # 7.5 x 9.5 has (int)(7 * 9.5) = 66 points, not a box: a flat 66 x 1 column
    _, _, _, box = mex(4, fix, mov, np.array([-2.5, -1.75]), np.array([4.25, 3.5]), np.array([7.5, 9.0]), "SAD_SUM_T")
    assert box.shape == (7, 9)
    _, _, _, col = mex(4, fix, mov, np.array([-2.5, -1.75]), np.array([4.25, 3.5]), np.array([7.5, 9.5]), "SAD_SUM_T")
    assert col.shape == (66, 1)
