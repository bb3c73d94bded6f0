// cgs_image.cu -- the image steps around a search in the reference's drivers.  Before it:
// filtering (CudaImage::filter -> filterProcess, include/cudaTensor.cuh:578-597 and
// include/cudaTensorKernels.cuh:353-394) and intensity quantisation (transformPixel,
// src/cpu/multispectral_ImageMatcher.cu:411-428).  After it: warping an image by the found
// homography (transformImage) and the three-colour overlay of the aligned pair
// (fuseAlignedImages), src/gpu/cudaImageFunctions.cuh:40-112.  The reference runs the warp and
// the overlay as single-thread kernels; here every output pixel has its own thread.
//
// Rounding.  The reference runs these on the device, built with nvcc's default multiply-add
// contraction, and this file is built the same way (it is the one translation unit compiled
// without -fmad=false): the per-pixel expressions keep the reference's form and operand order,
// so the compiler forms the same fused operations and the outputs match the reference's
// device results.
#include <cmath>
#include <string>

#include "cgs_internal.h"

namespace cgs {

// Pixel value of a CudaImage<T, C> at flat index c + C (x + W y) as float; indices at or past
// the end of the image (the bilinear tap of row H) read 0, the reference reading past its
// buffer (include/cudaTensor.cuh:561-566) defined.
template <typename T>
__device__ __forceinline__ float flat_tap(const T *d, uint32_t idx, uint32_t total) {
    return idx < total ? (float)d[idx] : 0.0f;
}

// CudaImage::inImage and valueAt_bilinear (include/cudaTensor.cuh:548-575), on a flat buffer.
__device__ __forceinline__ bool in_img(float y, float x, int W, int H) {
    return x >= 0 && y >= 0 && x < W && y < H;
}

template <typename T>
__device__ __forceinline__ float bilinear_flat(const T *d, int W, int H, int C, float y, float x, int c) {
    const uint32_t total = (uint32_t)C * (uint32_t)W * (uint32_t)H;
    const float fy = floorf(y), fx = floorf(x), cy = ceilf(y), cx = ceilf(x);
    auto at = [&](float yy, float xx) {
        return flat_tap(d, (uint32_t)c + (uint32_t)C * ((uint32_t)xx + (uint32_t)W * (uint32_t)yy), total);
    };
    const float tlc = at(fy, fx), trc = at(fy, cx), blc = at(cy, fx), brc = at(cy, cx);
    const float alpha_x = x - fx;
    const float alpha_y = y - fy;
    const float value_top = (1.0f - alpha_x) * tlc + alpha_x * trc;
    const float value_bottom = (1.0f - alpha_x) * blc + alpha_x * brc;
    return (1.0f - alpha_y) * value_top + alpha_y * value_bottom;
}

struct WarpH {
    float h[8];
};

// The inverse map of transformImage: output pixel (x, y) -> input coordinates.
__device__ __forceinline__ void warp_coord(const WarpH &H, int x, int y, float &new_x, float &new_y) {
    const float h11 = H.h[0], h12 = H.h[1], h13 = H.h[2], h21 = H.h[3], h22 = H.h[4], h23 = H.h[5], h31 = H.h[6],
                h32 = H.h[7];
    const float new_w = ((h21 * h32 - h22 * h31) * x + (h12 * h31 - h11 * h32) * y + h11 * h22 - h12 * h21);
    new_x = ((h22 - h23 * h32) * x + (h13 * h32 - h12) * y + h12 * h23 - h13 * h22) / new_w;
    new_y = ((h23 * h31 - h21) * x + (h11 - h13 * h31) * y + h13 * h21 - h11 * h23) / new_w;
}

// One output pixel of transformImage: dst channels dst_c0 .. dst_c0 + nch - 1 of pixel (x, y)
// receive source channels src_c0 .. where the inverse map of H lands inside the source.  The
// overlay runs it once per output channel, so every warp takes this same code.
template <typename T>
__global__ void warp_kernel(const WarpH H, int rows, int cols, const T *__restrict__ src, int sh, int sw, int sC,
                            int src_c0, int nch, T *__restrict__ dst, int dw, int dC, int dst_c0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const int y = i / cols, x = i - y * cols;
    float nx, ny;
    warp_coord(H, x, y, nx, ny);
    if (!in_img(ny, nx, sw, sh)) return;
    for (int c = 0; c < nch; c++)
        dst[(size_t)dst_c0 + c + (size_t)dC * ((size_t)x + (size_t)dw * y)] =
            (T)bilinear_flat(src, sw, sh, sC, ny, nx, src_c0 + c);
}

template <typename T>
static cudaError_t launch_warp(const WarpH &H, int rows, int cols, const void *src, int sh, int sw, int sC, int src_c0,
                               int nch, const void *dst, int dw, int dC, int dst_c0, cudaStream_t st) {
    const int n = rows * cols;
    warp_kernel<T><<<(n + 255) / 256, 256, 0, st>>>(H, rows, cols, (const T *)src, sh, sw, sC, src_c0, nch,
                                                    (T *)const_cast<void *>(dst), dw, dC, dst_c0);
    return cudaGetLastError();
}

static cudaError_t warp_any(int pix, const WarpH &H, int rows, int cols, const void *src, int sh, int sw, int sC,
                            int src_c0, int nch, const void *dst, int dw, int dC, int dst_c0, cudaStream_t st) {
    switch (pix) {
        case CGS_PIXEL_U8: return launch_warp<uint8_t>(H, rows, cols, src, sh, sw, sC, src_c0, nch, dst, dw, dC, dst_c0, st);
        case CGS_PIXEL_F64: return launch_warp<double>(H, rows, cols, src, sh, sw, sC, src_c0, nch, dst, dw, dC, dst_c0, st);
        case CGS_PIXEL_U16:
            return launch_warp<uint16_t>(H, rows, cols, src, sh, sw, sC, src_c0, nch, dst, dw, dC, dst_c0, st);
        default: return launch_warp<float>(H, rows, cols, src, sh, sw, sC, src_c0, nch, dst, dw, dC, dst_c0, st);
    }
}

// filterProcess: a (fh x fw) correlation of channel c of `in` at (row, col), taps outside the
// image taking the centre pixel's value, for channels whose action is FILTER; COPY channels are
// copied.  As in the reference, one running sum serves every FILTER channel of a pixel (it is
// not reset between channels) and the sum is converted to the pixel type.
template <typename T>
__global__ void filter_kernel(const float *__restrict__ filt, int fh, int fw, const T *__restrict__ in, int H, int W,
                              int C, uint32_t filter_mask, T *__restrict__ out) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= W || row >= H) return;
    float pixVal = 0;
    for (int c = 0; c < C; ++c) {
        const size_t o = (size_t)c + (size_t)C * ((size_t)col + (size_t)W * row);
        if (!((filter_mask >> c) & 1u)) {
            out[o] = in[o];
            continue;
        }
        const int r0 = row - (fh - 1) / 2, c0 = col - (fw - 1) / 2;
        for (int fr = 0; fr < fh; ++fr) {
            for (int fc = 0; fc < fw; ++fc) {
                const int r = r0 + fr, cc = c0 + fc;
                const bool inside = in_img((float)r, (float)cc, W, H);
                const size_t src = inside ? (size_t)c + (size_t)C * ((size_t)cc + (size_t)W * r) : o;
                pixVal += filt[fc + fw * fr] * in[src];
            }
        }
        out[o] = (T)pixVal;
    }
}

// transformPixel: each sample read as a signed char, v = (int)(v / mod), v = (int)(v * mod),
// stored back as the pixel type (uint8 images: modulo 256).
__global__ void quantize_kernel(uint8_t *__restrict__ img, int H, int W, int C, float mod) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    for (int c = 0; c < C; c++) {
        const size_t o = (size_t)c + (size_t)C * ((size_t)x + (size_t)W * y);
        const signed char pixel = (signed char)img[o];
        int temp = (int)pixel;
        temp /= mod;
        temp *= mod;
        img[o] = (uint8_t)temp;
    }
}

static cgs_status check_warp_image(const cgs_image *im, const char *name) {
    if (!im || !im->data) return fail(CGS_ERROR_INVALID_VALUE, std::string(name) + " is null");
    if (im->height < 1 || im->width < 1 || im->channels < 1 || im->channels > 4)
        return fail(CGS_ERROR_INVALID_VALUE, std::string(name) + " has an invalid size or channel count");
    if ((int64_t)im->height * im->width * im->channels >= ((int64_t)1 << 31))
        return fail(CGS_ERROR_UNSUPPORTED, std::string(name) + " is too large");
    return CGS_SUCCESS;
}

}  // namespace cgs

extern "C" {

cgs_status cgs_transform_image(const float H[8], int32_t rows, int32_t cols, const cgs_image *in, cgs_image *out,
                               cgs_stream_t stream) {
    using namespace cgs;
    cgs_status s;
    if (!H) return fail(CGS_ERROR_INVALID_VALUE, "H is null");
    if ((s = check_warp_image(in, "in")) != CGS_SUCCESS || (s = check_warp_image(out, "out")) != CGS_SUCCESS) return s;
    if (in->pixel != out->pixel || in->channels != out->channels)
        return fail(CGS_ERROR_INVALID_VALUE, "in and out must have the same pixel type and channels");
    if (rows < 0 || cols < 0 || rows > out->height || cols > out->width)
        return fail(CGS_ERROR_INVALID_VALUE, "rows x cols must lie inside the output image");
    if (rows == 0 || cols == 0) return CGS_SUCCESS;
    WarpH w;
    for (int k = 0; k < 8; k++) w.h[k] = H[k];
    CGS_CUDA(warp_any(in->pixel, w, rows, cols, in->data, in->height, in->width, in->channels, 0, in->channels,
                      out->data, out->width, out->channels, 0, (cudaStream_t)stream),
             "warp_kernel");
    return CGS_SUCCESS;
}

cgs_status cgs_fuse_aligned(const float estimated_H[8], const float true_H[8], const cgs_image *reference,
                            const cgs_image *moving, cgs_image *fused, int32_t channel, cgs_stream_t stream) {
    using namespace cgs;
    cgs_status s;
    if (!estimated_H || !true_H) return fail(CGS_ERROR_INVALID_VALUE, "a homography is null");
    if ((s = check_warp_image(reference, "reference")) != CGS_SUCCESS ||
        (s = check_warp_image(moving, "moving")) != CGS_SUCCESS || (s = check_warp_image(fused, "fused")) != CGS_SUCCESS)
        return s;
    if (reference->pixel != moving->pixel || fused->pixel != moving->pixel || reference->channels != moving->channels)
        return fail(CGS_ERROR_INVALID_VALUE, "the images must share the pixel type; reference and moving the channels");
    if (fused->channels != 3) return fail(CGS_ERROR_INVALID_VALUE, "the fused image has 3 channels");
    if (channel < 0 || channel >= moving->channels) return fail(CGS_ERROR_INVALID_VALUE, "channel out of range");
    // channel 0: moving under the estimate; 1: reference under the identity; 2: moving under
    // the true homography (fuseAlignedImages' three passes)
    WarpH hs[3];
    for (int k = 0; k < 8; k++) {
        hs[0].h[k] = estimated_H[k];
        hs[2].h[k] = true_H[k];
        hs[1].h[k] = (k == 0 || k == 4) ? 1.0f : 0.0f;
    }
    for (int c = 0; c < 3; c++) {
        const cgs_image *src = c == 1 ? reference : moving;
        CGS_CUDA(warp_any(src->pixel, hs[c], fused->height, fused->width, src->data, src->height, src->width,
                          src->channels, channel, 1, fused->data, fused->width, 3, c, (cudaStream_t)stream),
                 "warp_kernel");
    }
    return CGS_SUCCESS;
}

}  // extern "C"

extern "C" cgs_status cgs_filter_image(const cgs_image *filter, const cgs_image *in, cgs_image *out,
                                       const int32_t actions[], cgs_stream_t stream) {
    using namespace cgs;
    cgs_status s;
    if ((s = check_warp_image(filter, "filter")) != CGS_SUCCESS || (s = check_warp_image(in, "in")) != CGS_SUCCESS ||
        (s = check_warp_image(out, "out")) != CGS_SUCCESS)
        return s;
    if (!actions) return fail(CGS_ERROR_INVALID_VALUE, "actions is null");
    if (filter->pixel != CGS_PIXEL_F32 || filter->channels != 1)
        return fail(CGS_ERROR_INVALID_VALUE, "the filter is a single-channel float image");
    if (in->pixel != out->pixel || in->channels != out->channels || in->height != out->height ||
        in->width != out->width)
        return fail(CGS_ERROR_INVALID_VALUE, "in and out must have the same shape and pixel type");
    uint32_t mask = 0;
    for (int c = 0; c < in->channels; c++) {
        if (actions[c] != 0 && actions[c] != 1) return fail(CGS_ERROR_INVALID_VALUE, "actions are 0 (COPY) or 1 (FILTER)");
        mask |= (uint32_t)actions[c] << c;
    }
    const dim3 block(16, 16), grid((in->width + 15) / 16, (in->height + 15) / 16);
    cudaStream_t st = (cudaStream_t)stream;
    const float *f = static_cast<const float *>(filter->data);
    void *o = const_cast<void *>(out->data);
#define CGS_FILTER(T)                                                                                              \
    filter_kernel<T><<<grid, block, 0, st>>>(f, filter->height, filter->width, (const T *)in->data, in->height,   \
                                             in->width, in->channels, mask, (T *)o)
    switch (in->pixel) {
        case CGS_PIXEL_U8: CGS_FILTER(uint8_t); break;
        case CGS_PIXEL_F64: CGS_FILTER(double); break;
        case CGS_PIXEL_U16: CGS_FILTER(uint16_t); break;
        default: CGS_FILTER(float);
    }
#undef CGS_FILTER
    CGS_CUDA(cudaGetLastError(), "filter_kernel");
    return CGS_SUCCESS;
}

extern "C" cgs_status cgs_quantize_image(cgs_image *img, float mod, cgs_stream_t stream) {
    using namespace cgs;
    cgs_status s;
    if ((s = check_warp_image(img, "img")) != CGS_SUCCESS) return s;
    if (img->pixel != CGS_PIXEL_U8) return fail(CGS_ERROR_UNSUPPORTED, "intensity quantisation takes uint8 images");
    if (!(mod > 0.0f) || !std::isfinite(mod)) return fail(CGS_ERROR_INVALID_VALUE, "mod must be positive");
    const dim3 block(32, 32), grid((img->width + 31) / 32, (img->height + 31) / 32);
    quantize_kernel<<<grid, block, 0, (cudaStream_t)stream>>>((uint8_t *)const_cast<void *>(img->data), img->height,
                                                             img->width, img->channels, mod);
    CGS_CUDA(cudaGetLastError(), "quantize_kernel");
    return CGS_SUCCESS;
}

extern "C" cgs_status cgs_homography(const float params[8], float cx, float cy, int32_t centred, float H[8]) {
    using namespace cgs;
    if (!params || !H) return fail(CGS_ERROR_INVALID_VALUE, "params or H is null");
    // cos/sin with the host libm, as the reference's CPU path and the search kernels' tables
    const float c = std::cos(params[0]), s = std::sin(params[0]);
    const Homog h = centred ? h_centred(params, c, s, cx, cy) : h_uncentred(params, c, s);
    const float v[8] = {h.h11, h.h12, h.h13, h.h21, h.h22, h.h23, h.h31, h.h32};
    for (int k = 0; k < 8; k++) H[k] = v[k];
    return CGS_SUCCESS;
}
