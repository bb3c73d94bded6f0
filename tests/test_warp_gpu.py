"""The image steps around a search against the reference's own kernels run on the same GPU from
the reference harness (oracle/_ref): the warp and the aligned overlay (cgs_transform_image,
cgs_fuse_aligned vs transformImage / fuseAlignedImages, src/gpu/cudaImageFunctions.cuh:40-112)
and the filter (cgs_filter_image vs CudaImage::filter, include/cudaTensorKernels.cuh:353-394).
Integer outputs match element for element, and so do the warp's float outputs; float outputs of
the overlay and the filter match to the last bits (nvcc fuses some of the reference's
multiply-adds differently in those two kernels).  The reference's bilinear taps reach one row
past an image, so its inputs are given a zero row (and one pixel) of padding, the value the
library defines there.  The intensity quantisation (transformPixel, which lives in a driver
that does not build here) is checked against a numpy restatement."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _ref():
    if not O.have_ref():
        pytest.skip("reference harness not built")
    L = O.ref()
    L.cgsref_transform_image.restype = C.c_int
    L.cgsref_transform_image.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_void_p,
                                         C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
    L.cgsref_fuse_aligned.restype = C.c_int
    L.cgsref_fuse_aligned.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p,
                                      C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                      C.c_int]
    return L


def _padded(cuda, img):
    """Device copy of an (H, W, C) image followed by a zero row and one zero pixel."""
    import torch
    h, w, c = img.shape
    buf = torch.zeros((h + 1) * w * c + c, dtype=torch.from_numpy(img).dtype, device=cuda)
    buf[: h * w * c] = torch.from_numpy(np.ascontiguousarray(img)).reshape(-1).to(cuda)
    return buf


def _image(buf, h, w, c):
    import cugridsearch_b200 as cgs
    return cgs.CudaImage(buf[: h * w * c].view(h, w, c))


def _params(rng):
    return np.array([rng.uniform(-0.3, 0.3), rng.uniform(0.85, 1.15), rng.uniform(0.85, 1.15), rng.uniform(-0.1, 0.1),
                     rng.uniform(-6, 6), rng.uniform(-6, 6), rng.uniform(-2e-3, 2e-3), rng.uniform(-2e-3, 2e-3)],
                    np.float32)


@pytest.mark.parametrize("dtype,channels", [(np.uint8, 1), (np.uint8, 3), (np.float32, 1), (np.float32, 3)])
def test_transform_image_matches_reference_kernel(cuda, lib, dtype, channels):
    import torch
    import cugridsearch_b200 as cgs
    L = _ref()
    rng = np.random.default_rng(17 + channels)
    ih, iw, oh, ow = 37, 45, 33, 41
    src = rng.uniform(0, 255, (ih, iw, channels))
    src = np.round(src).astype(np.uint8) if dtype == np.uint8 else src.astype(np.float32)
    buf = _padded(cuda, src)
    pix = 1 if dtype == np.uint8 else 0
    for trial in range(4):
        H = cgs.homography(_params(rng), iw / 2, ih / 2)
        fill = 7 if dtype == np.uint8 else -3.5
        ours = torch.full((oh, ow, channels), fill, dtype=buf.dtype, device=cuda)
        theirs = torch.full((oh, ow, channels), fill, dtype=buf.dtype, device=cuda)
        rows, cols = oh - trial, ow - 2 * trial
        cgs.transform_image(H, _image(buf, ih, iw, channels), cgs.CudaImage(ours), rows, cols)
        h8 = (C.c_float * 8)(*H)
        assert L.cgsref_transform_image(pix, channels, h8, rows, cols, buf.data_ptr(), ih, iw, theirs.data_ptr(),
                                        oh, ow) == 0
        torch.cuda.synchronize()
        a, b = ours.cpu().numpy(), theirs.cpu().numpy()
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (trial, np.argwhere(a != b)[:5])
        assert (a != fill).any() and (a == fill).any()  # some pixels map inside, some outside


@pytest.mark.parametrize("dtype,channels", [(np.uint8, 1), (np.uint8, 3), (np.float32, 1)])
def test_fuse_aligned_matches_reference_kernel(cuda, lib, dtype, channels):
    import torch
    import cugridsearch_b200 as cgs
    L = _ref()
    rng = np.random.default_rng(5 + channels)
    rh, rw, mh, mw = 30, 34, 31, 29
    gen = lambda h, w: rng.uniform(0, 255, (h, w, channels))
    ref_img, mov_img = gen(rh, rw), gen(mh, mw)
    if dtype == np.uint8:
        ref_img, mov_img = np.round(ref_img).astype(np.uint8), np.round(mov_img).astype(np.uint8)
    else:
        ref_img, mov_img = ref_img.astype(np.float32), mov_img.astype(np.float32)
    rbuf, mbuf = _padded(cuda, ref_img), _padded(cuda, mov_img)
    pix = 1 if dtype == np.uint8 else 0
    He = cgs.homography(_params(rng), mw / 2, mh / 2)
    Ht = cgs.homography(_params(rng), mw / 2, mh / 2)
    ch = channels - 1
    ours = torch.zeros((rh, rw, 3), dtype=rbuf.dtype, device=cuda)
    theirs = torch.zeros((rh, rw, 3), dtype=rbuf.dtype, device=cuda)
    cgs.fuse_aligned(He, Ht, _image(rbuf, rh, rw, channels), _image(mbuf, mh, mw, channels), cgs.CudaImage(ours), ch)
    he8, ht8 = (C.c_float * 8)(*He), (C.c_float * 8)(*Ht)
    assert L.cgsref_fuse_aligned(pix, channels, he8, ht8, rbuf.data_ptr(), rh, rw, mbuf.data_ptr(), mh, mw,
                                 theirs.data_ptr(), rh, rw, ch) == 0
    torch.cuda.synchronize()
    a, b = ours.cpu().numpy(), theirs.cpu().numpy()
    if dtype == np.uint8:
        assert np.array_equal(a, b), np.argwhere(a != b)[:5]
    else:
        # the reference's overlay kernel hoists its per-channel homography products out of its
        # pixel loops, and the compiler fuses some of them differently than in transformImage:
        # float outputs agree to the last bits, not bit for bit
        np.testing.assert_allclose(a, b, rtol=5e-5, atol=1e-3)


@pytest.mark.parametrize("dtype,channels,actions", [(np.uint8, 1, [1]), (np.uint8, 3, [1, 0, 1]),
                                                    (np.float32, 1, [1])])
@pytest.mark.parametrize("fsize", [(3, 3), (5, 5), (2, 4)])
def test_filter_matches_reference_kernel(cuda, lib, dtype, channels, actions, fsize):
    """cgs_filter_image against CudaImage::filter (filterProcess) on the same GPU: equal element
    for element, including the running sum carried across FILTER channels and the conversion of
    out-of-range sums to uint8."""
    import torch
    import cugridsearch_b200 as cgs
    L = _ref()
    L.cgsref_filter.restype = C.c_int
    L.cgsref_filter.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                C.c_void_p, C.POINTER(C.c_int)]
    rng = np.random.default_rng(fsize[0] * 10 + channels)
    h, w = 23, 31
    src = rng.uniform(0, 255, (h, w, channels))
    src = np.round(src).astype(np.uint8) if dtype == np.uint8 else src.astype(np.float32)
    filt = rng.normal(0, 0.6, fsize).astype(np.float32)
    filt[(fsize[0] - 1) // 2, (fsize[1] - 1) // 2] += 1.0  # sharpening-like: sums leave [0, 255]
    src_d = torch.from_numpy(src).to(cuda)
    filt_d = torch.from_numpy(filt).to(cuda)
    ours = torch.zeros_like(src_d)
    theirs = torch.zeros_like(src_d)
    cgs.filter_image(cgs.CudaImage(filt_d), cgs.CudaImage(src_d), cgs.CudaImage(ours), actions)
    acts = (C.c_int * channels)(*actions)
    assert L.cgsref_filter(1 if dtype == np.uint8 else 0, channels, filt_d.data_ptr(), fsize[0], fsize[1],
                           src_d.data_ptr(), h, w, theirs.data_ptr(), acts) == 0
    torch.cuda.synchronize()
    a, b = ours.cpu().numpy(), theirs.cpu().numpy()
    if dtype == np.uint8:
        assert np.array_equal(a, b), np.argwhere(a != b)[:5]
    else:
        # float sums: the compiler fuses the reference's multiply-adds a little differently
        np.testing.assert_allclose(a, b, rtol=5e-6, atol=2e-4)


def test_quantize_matches_restatement(cuda, lib):
    """cgs_quantize_image against transformPixel restated in numpy (signed-char read, float
    division and product truncated to int, stored modulo 256)."""
    import torch
    import cugridsearch_b200 as cgs
    rng = np.random.default_rng(4)
    img = rng.integers(0, 256, (19, 27, 3), dtype=np.uint8)
    for mod in (2.0, 7.5, 16.0, 0.75):
        d = torch.from_numpy(img.copy()).to(cuda)
        cgs.quantize_image(cgs.CudaImage(d), mod)
        v = img.view(np.int8).astype(np.float32)
        t = np.trunc(v / np.float32(mod)).astype(np.float32)
        want = (np.trunc(t * np.float32(mod)).astype(np.int64) & 0xFF).astype(np.uint8)
        np.testing.assert_array_equal(d.cpu().numpy(), want)
