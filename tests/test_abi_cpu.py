"""CPU tests of the C ABI: the library loads, exports every declared symbol, and its
host-side grid arithmetic matches the reference's (via the oracle); argument checks fail
with status codes before any device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cugridsearch_b200.h")


def _declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w \*]*?\b(cgs_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_binding_list():
    import cugridsearch_b200._abi as abi
    assert _declared_functions() == sorted(abi.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in _declared_functions():
        assert hasattr(lib, name), f"libcgs_b200.so does not export {name}"
    assert lib.cgs_version() >= 100


def test_status_strings(lib):
    for s in range(8):
        assert lib.cgs_status_string(s)


GRIDS = [
    ([0.0, 0.9, 0.9, -0.05, -6, -6, -1e-4, -1e-4], [0.17, 1.1, 1.1, 0.05, 6, 6, 1e-4, 1e-4], [4] * 8),
    ([-0.2, 1.0, 1.0, 0.0, -24, -24, 0.0, 0.0], [0.2, 1.0, 1.2, 0.0, 24, 24, 1e-4, 0.0], [6, 3, 6, 1, 6, 6, 2, 5]),
    # main_mi-style fractional counts (cudaGridSearch_main_mi.cu:300-308)
    ([0.0, 1.5, 1.5, -0.4, -64, -48, 0, 0], [3.14159, 5, 5, 0.2, 192, 144, 0, 0], [8, 8, 8, 5, 25.7, 19.3, 1, 1]),
    ([-3.0, -3.0], [3.0, 3.0], [1000, 1000]),
]


@pytest.mark.parametrize("start,end,count", GRIDS)
def test_grid_arithmetic_matches_reference(lib, start, end, count):
    import cugridsearch_b200 as cgs
    g = cgs.CudaGrid.from_ranges(start, end, count)
    og = O.make_grid(start, end, count)
    np.testing.assert_array_equal(g.resolution(), np.array(list(og.resolution)[: len(start)], np.float32))
    np.testing.assert_array_equal(g.getAxisSampleCounts(), np.array(list(og.count)[: len(start)], np.float32))
    n = g.numElements()
    assert n == O.grid_num(og)
    rng = np.random.default_rng(1)
    for idx in [0, 1, n - 1] + list(rng.integers(0, n, 50)):
        np.testing.assert_array_equal(g.getGridPoint(int(idx)), O.grid_point(og, int(idx))[: len(start)])


def test_from_ranges_equals_the_setter_sequence(lib):
    """from_ranges sets the three rows and updates once; the reference's setter sequence (start,
    end, counts, each followed by an update) leaves the same grid, collapsed axes included."""
    import cugridsearch_b200 as cgs
    rng = np.random.default_rng(3)
    for _ in range(2000):
        s = rng.uniform(-50, 50, 8)
        e = s + np.where(rng.random(8) < 0.25, rng.choice([0.0, 1e-9, 1e-6, 1e-4], 8), rng.uniform(-10, 30, 8))
        c = rng.integers(1, 9, 8).astype(float)
        a = cgs.CudaGrid.from_ranges(list(s), list(e), list(c))
        b = cgs.CudaGrid(8)
        b.setStartPoint(list(s))
        b.setEndPoint(list(e))
        b.setNumSamples(list(c))
        assert bytes(a.g) == bytes(b.g)


def test_collapsed_axis(lib):
    import cugridsearch_b200 as cgs
    g = cgs.CudaGrid.from_ranges([0.0, 1.0], [0.0, 2.0], [10, 3])  # start == end collapses to 1 sample
    assert list(g.getAxisSampleCounts()) == [1.0, 3.0]
    assert g.numElements() == 3


def test_invalid_arguments_fail_before_device_work(lib):
    import cugridsearch_b200._abi as abi
    L = lib
    img = abi.CgsImage(0, 8, 8, 1, 0)
    g = abi.CgsGrid()
    g.dims = 8
    for a in range(8):
        g.count[a] = 2.0
        g.end[a] = 1.0
    L.cgs_grid_update(C.byref(g), -1)
    o = abi.CgsOptions(abi.COSTS["ZNCC"], 0, 0.0, 0, 0, 0)
    s = L.cgs_search(C.byref(img), C.byref(img), C.byref(g), C.byref(o), None, None, None)
    assert s == 1 and b"null" in L.cgs_last_error()
    img2 = abi.CgsImage(16, 0, 8, 1, 0)  # empty size
    assert L.cgs_search(C.byref(img2), C.byref(img2), C.byref(g), C.byref(o), None, 16, None) == 1
    img3 = abi.CgsImage(16, 8, 8, 5, 0)  # 5 channels
    assert L.cgs_search(C.byref(img3), C.byref(img3), C.byref(g), C.byref(o), None, 16, None) == 1
    bad = abi.CgsOptions(99, 0, 0.0, 0, 0, 0)
    ok = abi.CgsImage(16, 8, 8, 1, 0)
    assert L.cgs_search(C.byref(ok), C.byref(ok), C.byref(g), C.byref(bad), None, 16, None) == 1
    mi = abi.CgsOptions(abi.COSTS["MI"], 48, 0.0, 0, 0, 0)  # not a power of two
    assert L.cgs_search(C.byref(ok), C.byref(ok), C.byref(g), C.byref(mi), None, 16, None) == 1
    g2 = abi.CgsGrid()
    g2.dims = 2
    g2.count[0] = g2.count[1] = 2.0
    assert L.cgs_search(C.byref(ok), C.byref(ok), C.byref(g2), C.byref(o), None, 16, None) == 1  # needs 8 axes
    g2.dims = 9
    assert L.cgs_grid_update(C.byref(g2), -1) == 1


def test_python_mirror_rejects_host_memory():
    import numpy as np
    import torch
    import cugridsearch_b200 as cgs
    with pytest.raises(TypeError):
        cgs.CudaImage(torch.from_numpy(np.zeros((4, 4), np.float32)))


def test_batch_arguments_fail_before_device_work(lib):
    """cgs_batch_create validates every pair (naming it) before touching the device."""
    import cugridsearch_b200._abi as abi
    L = lib
    h = C.c_void_p(None)
    assert L.cgs_batch_create(None, 0, None, C.byref(h)) == 1 and not h.value
    g = abi.CgsGrid()
    g.dims = 8
    for a in range(8):
        g.count[a] = 2.0
        g.end[a] = 1.0
    L.cgs_grid_update(C.byref(g), -1)
    img = abi.CgsImage(16, 8, 8, 1, 0)
    ok = abi.CgsOptions(abi.COSTS["ZNCC"], 0, 0.0, 0, 0, 0)

    def pairs(*ps):
        return (abi.CgsPair * len(ps))(*ps)

    good = abi.CgsPair(img, img, g, ok, None, 64)
    assert L.cgs_batch_create(pairs(good, abi.CgsPair(img, img, g, ok, None, None)), 2, None, C.byref(h)) == 1
    assert b"pair 1" in L.cgs_last_error() and b"result" in L.cgs_last_error()
    unsupported = abi.CgsOptions(abi.COSTS["SAD_AVG_H"], 0, 0.0, 0, 0, 0)
    assert L.cgs_batch_create(pairs(abi.CgsPair(img, img, g, unsupported, None, 64)), 1, None, C.byref(h)) == 2
    rgb = abi.CgsImage(16, 8, 8, 3, 0)
    assert L.cgs_batch_create(pairs(abi.CgsPair(rgb, rgb, g, ok, None, 64)), 1, None, C.byref(h)) == 2
    bad_bins = abi.CgsOptions(abi.COSTS["MI"], 48, 0.0, 0, 0, 0)
    assert L.cgs_batch_create(pairs(abi.CgsPair(img, img, g, bad_bins, None, 64)), 1, None, C.byref(h)) == 1
    assert not h.value
    # the handle's queries refuse a null handle or output
    k = C.c_int32(-1)
    assert L.cgs_batch_kernel_launches(None, C.byref(k)) == 1 and k.value == -1
    t = (C.c_uint64 * 1)()
    assert L.cgs_batch_pair_times(None, t, t) == 1


def test_batch_struct_layout():
    """The ctypes mirrors of cgs_pair / cgs_batch_plan / cgs_tune_entry / cgs_argmin have the C
    sizes and offsets."""
    import subprocess
    import tempfile
    import cugridsearch_b200._abi as abi
    src = ('#include <stdio.h>\n#include <stddef.h>\n#include "cugridsearch_b200.h"\n'
           'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(cgs_pair), offsetof(cgs_pair, costs),'
           ' offsetof(cgs_pair, result), sizeof(cgs_batch_plan), sizeof(cgs_tune_entry), sizeof(cgs_argmin),'
           ' offsetof(cgs_argmin, verified), offsetof(cgs_argmin, index_fp64), offsetof(cgs_argmin, max_err_fp64));'
           ' return 0;}\n')
    with tempfile.TemporaryDirectory() as d:
        c_file, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
        open(c_file, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c_file, "-o", exe], check=True)
        got = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [C.sizeof(abi.CgsPair), abi.CgsPair.costs.offset, abi.CgsPair.result.offset,
                   C.sizeof(abi.CgsBatchPlan), C.sizeof(abi.CgsTuneEntry), C.sizeof(abi.CgsArgmin),
                   abi.CgsArgmin.verified.offset, abi.CgsArgmin.index_fp64.offset, abi.CgsArgmin.max_err_fp64.offset]


def test_homography_matches_reference_host_build(lib):
    """cgs_homography against the reference's parametersToHomography built for the host."""
    import cugridsearch_b200 as cgs
    if not O.have_ref():
        pytest.skip("reference harness not built")
    R = O.ref()
    R.cgsref_params_to_h.restype = None
    R.cgsref_params_to_h.argtypes = [C.POINTER(C.c_float), C.c_float, C.c_float, C.POINTER(C.c_float)]
    rng = np.random.default_rng(9)
    for _ in range(200):
        p = np.array([rng.uniform(-0.5, 0.5), rng.uniform(0.8, 1.2), rng.uniform(0.8, 1.2), rng.uniform(-0.1, 0.1),
                      rng.uniform(-30, 30), rng.uniform(-30, 30), rng.uniform(-1e-3, 1e-3), rng.uniform(-1e-3, 1e-3)],
                     np.float32)
        cx, cy = float(rng.integers(8, 300)) / 2, float(rng.integers(8, 300)) / 2
        ref = (C.c_float * 8)()
        R.cgsref_params_to_h((C.c_float * 8)(*p), cx, cy, ref)
        np.testing.assert_array_equal(cgs.homography(p, cx, cy), np.array(list(ref), np.float32))
