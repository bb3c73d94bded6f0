/*
 * ref_harness.cu -- runs the REFERENCE's own cost functors on the host (TEST
 * INFRASTRUCTURE: parity oracle and timed CPU baseline; never part of the product).
 *
 * This file contains no reference code.  It #includes the unmodified reference headers
 * from the reference checkout at build time (oracle/Makefile, REF=...), instantiates the
 * __host__ __device__ functors (cudaErrorFunctions.cuh, cudaErrorFunction_mi.cuh) and
 * calls them with CudaImage objects whose _data are host pointers, exactly as the
 * reference itself does for its "Min Value check" (src/gpu/cudaGridSearch_main_mi.cu:388)
 * and its Levenberg-Marquardt functor (src/cpu/multispectral_ImageMatcher.cu:283-298).
 * The output, oracle/_ref/libcgs_ref.so, is not committed.
 *
 * The reference only decodes grid points on the device (CudaGrid::indexToGridPoint,
 * cudaGridSearch.cuh:160-187); the harness decodes with the same integer arithmetic and
 * takes the grid-value rounding mode (fused or not) as an argument.
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <omp.h>

#define CUDAFUNCTION __host__ __device__
#include "helper_cuda.h"
#include <cudaTensor.cuh>
#include "cudaGridSearch.cuh"
#include "cudaErrorFunctions.cuh"
#include "cudaErrorFunction_mi.cuh"

namespace {

enum { SAD_AVG = 0, SAD_AVG_H = 1, SAD_SUM_T = 2, SAD_SUM_T_REF = 3, SQD_REF = 4, NCC_REF = 5,
       SQD_ALT = 6, NCC_ALT = 7, MI_ALT = 8 };

// Images are passed padded: the caller allocates (H + 1) * W * C + C elements with zeros
// after the image so the reference's reads at ceil(y) == H stay inside the buffer.
template <typename P, uint32_t C>
float eval_c(int cost, const float *params, const void *mov, int mh, int mw, const void *fix, int fh, int fw) {
    CudaImage<P, C> M(mh, mw), F(fh, fw);
    M.data() = (P *)mov;
    F.data() = (P *)fix;
    nv_ext::Vec<float, 8> v(params);
    switch (cost) {
        case SAD_AVG: return averageAbsoluteDifference<float, float, 8, C, P>(v, M, F);
        case SQD_REF: return calcSQD<float, float, 8, C, P>(v, M, F);
        case NCC_REF: return calcNCC<float, float, 8, C, P>(v, M, F);
        case SQD_ALT: return calcSQDAlt<float, float, 8, C, P>(v, M, F);
        case NCC_ALT: return calcNCCAlt<float, float, 8, C, P>(v, M, F);
        case MI_ALT: return calcMIAlt<float, float, 8, C, P>(v, M, F);
        default: break;
    }
    if (C == 1) {
        CudaImage<P> M1(mh, mw), F1(fh, fw);
        M1.data() = (P *)mov;
        F1.data() = (P *)fix;
        switch (cost) {
            case SAD_AVG_H: return averageAbsoluteDifferenceH<float, float, 8, 1, P>(v, M1, F1);
            case SAD_SUM_T: return sumOfAbsoluteDifferences<float, float, 8, 1, P>(v, M1, F1);
            case SAD_SUM_T_REF: return sumOfAbsoluteDifferences<float, float, 8, 1, P>(v, &M1, &F1);
            default: break;
        }
    }
    return NAN;
}

template <typename P>
float eval_p(int cost, const float *params, const void *mov, int mh, int mw, const void *fix, int fh, int fw, int c) {
    switch (c) {
        case 1: return eval_c<P, 1>(cost, params, mov, mh, mw, fix, fh, fw);
        case 3: return eval_c<P, 3>(cost, params, mov, mh, mw, fix, fh, fw);
        default: return NAN;
    }
}

}  // namespace

/* The reference's own grid on the DEVICE: CudaGrid<float, D> with caller-allocated data,
 * setStartPoint / setEndPoint / setNumSamples (each runs updateProcess<<<1,1>>>), then
 * getGridPoint (gridPointProcess<<<1,1>>>) for each index.  Compiled by nvcc with its
 * default flags, as the reference's drivers are, so the device rounding of the decode
 * (start + i * res, contracted or not) is the reference's.  No axis may end up with one
 * sample (count < 2, or |end - start| < 1e-7 count, which updateProcess collapses): for
 * such an axis updateProcess reads start_point()[-1] (cudaGridSearch.cuh:266), before
 * the allocation.  matrix (4 x D floats) receives the grid after the updates.  Returns 0 on
 * success, 1 on a CUDA error, 2 on a bad argument. */
template <unsigned int D>
static int device_grid_points(const float *start, const float *end, const float *count, const int64_t *idx, int n,
                              float *out, float *matrix) {
    for (unsigned int a = 0; a < D; a++)  // no axis may collapse to one sample
        if (!(count[a] >= 2.0f) || !((double)std::fabs(end[a] - start[a]) >= 1.0e-7 * (double)count[a])) return 2;
    CudaGrid<float, D> g;
    if (cudaMalloc(&g.data(), g.bytesSize()) != cudaSuccess) return 1;
    // zeroed first: each setter runs updateProcess over all rows, and with uninitialised
    // counts or ends an axis could look collapsed before its own setter has run
    if (cudaMemset(g.data(), 0, g.bytesSize()) != cudaSuccess) return 1;
    g.setStartPoint(std::vector<float>(start, start + D));
    g.setEndPoint(std::vector<float>(end, end + D));
    g.setNumSamples(std::vector<float>(count, count + D));
    int rc = 0;
    if (cudaMemcpy(matrix, g.data(), g.bytesSize(), cudaMemcpyDeviceToHost) != cudaSuccess) rc = 1;
    for (int k = 0; k < n && rc == 0; k++) {
        float pt[D];
        g.getGridPoint(pt, (int)idx[k]);
        for (unsigned int a = 0; a < D; a++) out[(size_t)k * D + a] = pt[a];
    }
    if (cudaDeviceSynchronize() != cudaSuccess) rc = 1;
    cudaFree(g.data());
    return rc;
}

/* The reference's transformImage and fuseAlignedImages (cudaImageFunctions.cuh:40-112) on the
 * DEVICE, launched <<<1,1>>> as its drivers launch them and compiled with nvcc's default flags.
 * pix: 0 = float, 1 = uint8_t; channels 1 or 3.  Every pointer is a device pointer; the
 * input buffers must hold (H + 1) * W * C + C elements (zeros after the image), the reach of
 * the reference's bilinear taps.  Returns 0, 1 on a CUDA error, 2 on unsupported arguments. */
template <typename P, uint8_t C>
static int transform_t(const float *H, int rows, int cols, const void *in, int ih, int iw, void *out, int oh, int ow) {
    nv_ext::Vec<float, 8> h(H);
    CudaImage<P, C> I(ih, iw), O(oh, ow);
    I.data() = (P *)in;
    O.data() = (P *)out;
    transformImage<P, 8, C><<<1, 1>>>(h, rows, cols, I, O);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

template <typename P, uint8_t C>
static int fuse_t(const float *He, const float *Ht, const void *ref, int rh, int rw, const void *mov, int mh, int mw,
                  void *fused, int fh, int fw, int ch) {
    nv_ext::Vec<float, 8> he(He), ht(Ht);
    CudaImage<P, C> R(rh, rw), M(mh, mw);
    CudaImage<P, 3> F(fh, fw);
    R.data() = (P *)ref;
    M.data() = (P *)mov;
    F.data() = (P *)fused;
    fuseAlignedImages<P, 8, C><<<1, 1>>>(he, ht, R, M, F, ch);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

/* The reference's CudaImage::filter (filterProcess on the DEVICE, include/cudaTensor.cuh:578-597).
 * Device pointers; actions one per channel (0 COPY, 1 FILTER). */
template <typename P, uint32_t C>
static int filter_t(const float *filt, int fh, int fw, const void *in, int h, int w, void *out, const int *actions) {
    CudaImage<float, 1> F(fh, fw);
    F.data() = (float *)filt;
    CudaImage<P, C> I(h, w), O(h, w);
    I.data() = (P *)in;
    O.data() = (P *)out;
    CHANNEL_ACTION acts[C];
    for (uint32_t c = 0; c < C; c++) acts[c] = actions[c] ? FILTER : COPY;
    I.filter(F, O, acts);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

/* The reference's own GPU search (CudaGridSearcher::search_by_value -> evaluationKernel_by_value,
 * src/gpu/cudaGridSearch.cuh:287-314, 736-765) of calcNCC or calcMIAlt, compiled unchanged for
 * sm_100a, timed with CUDA events around the call.  The kernel also writes result[n] (bound
 * check '>'), so the result buffer holds n + 1 floats; its bilinear taps reach one row past an
 * image, so the image buffers hold (H + 1) W + 1 elements, zero after the image. */
typedef func_byvalue_t<float, float, 8, CudaImage<float, 1>, CudaImage<float, 1>> ref_fn_f32;
typedef func_byvalue_t<float, float, 8, CudaImage<uint8_t, 1>, CudaImage<uint8_t, 1>> ref_fn_u8;
__device__ ref_fn_f32 ref_dev_ncc_f32 = calcNCC<float, float, 8, 1, float>;
__device__ ref_fn_u8 ref_dev_mialt_u8 = calcMIAlt<float, float, 8, 1, uint8_t>;

template <typename P, typename Fn>
static int gpu_search_t(const Fn &dev_fn, const float *start, const float *end, const float *count, const void *mov,
                        int mh, int mw, const void *fix, int fh, int fw, float *result, float *ms) {
    CudaGrid<float, 8> g;
    if (cudaMalloc(&g.data(), g.bytesSize()) != cudaSuccess) return 1;
    if (cudaMemset(g.data(), 0, g.bytesSize()) != cudaSuccess) return 1;
    g.setStartPoint(std::vector<float>(start, start + 8));
    g.setEndPoint(std::vector<float>(end, end + 8));
    g.setNumSamples(std::vector<float>(count, count + 8));
    float counts[8];
    g.getAxisSampleCounts(counts);
    CudaTensor<float, 8> values(counts);
    values.data() = result;
    CudaImage<P, 1> M(mh, mw), F(fh, fw);
    M.data() = (P *)mov;
    F.data() = (P *)fix;
    Fn h;
    if (cudaMemcpyFromSymbol(&h, dev_fn, sizeof(Fn)) != cudaSuccess) return 1;
    CudaGridSearcher<float, float, 8> searcher(g, values);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    searcher.search_by_value(h, M, F);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(g.data());
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

extern "C" {

/* One reference functor evaluation. pix: 0 = float, 1 = uint8_t, 2 = double, 3 = uint16_t. */
float cgsref_eval(int cost, const float *params, int pix, const void *mov, int mh, int mw, const void *fix, int fh,
                  int fw, int channels) {
    switch (pix) {
        case 1: return eval_p<uint8_t>(cost, params, mov, mh, mw, fix, fh, fw, channels);
        case 2: return eval_p<double>(cost, params, mov, mh, mw, fix, fh, fw, channels);
        case 3: return eval_p<uint16_t>(cost, params, mov, mh, mw, fix, fh, fw, channels);
        default: return eval_p<float>(cost, params, mov, mh, mw, fix, fh, fw, channels);
    }
}

/* The reference's homography helpers, for bit-exact tests of the oracle restatement. */
void cgsref_params_to_h(const float *params, float cx, float cy, float *h) {
    nv_ext::Vec<float, 8> v(params);
    parametersToHomography<float, 8>(v, cx, cy, h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7]);
}

void cgsref_params_to_h_norm(const float *params, int mw, int mh, int fw, int fh, float *h) {
    nv_ext::Vec<float, 8> v(params);
    parametersToHomographyNorm<float, 8>(v, mw, mh, fw, fh, h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7]);
}

void cgsref_new_coord(const float *h_in, int x, int y, float *nx, float *ny) {
    float h[8];
    memcpy(h, h_in, sizeof(h));
    calcNewCoordH(h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], x, y, *nx, *ny);
}

float cgsref_bilinear(int pix, const void *data, int height, int width, float y, float x) {
    if (pix == 1) {
        CudaImage<uint8_t, 1> im(height, width);
        im.data() = (uint8_t *)data;
        return im.valueAt_bilinear(y, x, 0);
    }
    CudaImage<float, 1> im(height, width);
    im.data() = (float *)data;
    return im.valueAt_bilinear(y, x, 0);
}

/* Grid decode with the reference's integer arithmetic (cudaGridSearch.cuh:160-187).
 * counts/start/res as stored in the CudaGrid matrix after update(). */
static void decode(int dims, const float *start, const float *res, const float *count, int64_t index, int use_fma,
                   float *out) {
    int32_t inc[8], idx[8];
    inc[0] = 1;
    for (int a = 1; a < dims; a++) inc[a] = (int32_t)(count[a - 1] * (float)inc[a - 1]);
    int32_t rem = (int32_t)index;
    for (int a = dims - 1; a >= 0; a--) {
        idx[a] = rem / inc[a];
        rem -= idx[a] * inc[a];
    }
    for (int a = 0; a < 8; a++) out[a] = 0.0f;
    for (int a = 0; a < dims; a++)
        out[a] = use_fma ? fmaf((float)idx[a], res[a], start[a]) : start[a] + (float)idx[a] * res[a];
}

/* Reference functor over a strided sample of grid indices, OpenMP over all requested
 * threads (the timed CPU baseline).  costs[k] = cost at index first + k * stride. */
int cgsref_search(int cost, int dims, const float *start, const float *res, const float *count, int use_fma, int pix,
                  const void *mov, int mh, int mw, const void *fix, int fh, int fw, int channels, int64_t first,
                  int64_t n, int64_t stride, float *costs, int threads) {
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
    for (int64_t k = 0; k < n; k++) {
        float pt[8];
        decode(dims, start, res, count, first + k * stride, use_fma, pt);
        costs[k] = cgsref_eval(cost, pt, pix, mov, mh, mw, fix, fh, fw, channels);
    }
    return 0;
}

int cgsref_max_threads(void) { return omp_get_max_threads(); }

int cgsref_transform_image(int pix, int channels, const float *H, int rows, int cols, const void *in, int ih, int iw,
                           void *out, int oh, int ow) {
    if (pix == 0 && channels == 1) return transform_t<float, 1>(H, rows, cols, in, ih, iw, out, oh, ow);
    if (pix == 0 && channels == 3) return transform_t<float, 3>(H, rows, cols, in, ih, iw, out, oh, ow);
    if (pix == 1 && channels == 1) return transform_t<uint8_t, 1>(H, rows, cols, in, ih, iw, out, oh, ow);
    if (pix == 1 && channels == 3) return transform_t<uint8_t, 3>(H, rows, cols, in, ih, iw, out, oh, ow);
    return 2;
}

/* cost: NCC_REF on float images or MI_ALT on uint8 images (single channel, 8 axes). */
int cgsref_gpu_search(int cost, const float *start, const float *end, const float *count, const void *mov, int mh,
                      int mw, const void *fix, int fh, int fw, float *result, float *ms) {
    if (cost == NCC_REF)
        return gpu_search_t<float>(ref_dev_ncc_f32, start, end, count, mov, mh, mw, fix, fh, fw, result, ms);
    if (cost == MI_ALT)
        return gpu_search_t<uint8_t>(ref_dev_mialt_u8, start, end, count, mov, mh, mw, fix, fh, fw, result, ms);
    return 2;
}

int cgsref_filter(int pix, int channels, const float *filt, int fh, int fw, const void *in, int h, int w, void *out,
                  const int *actions) {
    if (pix == 0 && channels == 1) return filter_t<float, 1>(filt, fh, fw, in, h, w, out, actions);
    if (pix == 1 && channels == 1) return filter_t<uint8_t, 1>(filt, fh, fw, in, h, w, out, actions);
    if (pix == 1 && channels == 3) return filter_t<uint8_t, 3>(filt, fh, fw, in, h, w, out, actions);
    return 2;
}

int cgsref_fuse_aligned(int pix, int channels, const float *He, const float *Ht, const void *ref, int rh, int rw,
                        const void *mov, int mh, int mw, void *fused, int fh, int fw, int ch) {
    if (pix == 0 && channels == 1) return fuse_t<float, 1>(He, Ht, ref, rh, rw, mov, mh, mw, fused, fh, fw, ch);
    if (pix == 1 && channels == 1) return fuse_t<uint8_t, 1>(He, Ht, ref, rh, rw, mov, mh, mw, fused, fh, fw, ch);
    if (pix == 1 && channels == 3) return fuse_t<uint8_t, 3>(He, Ht, ref, rh, rw, mov, mh, mw, fused, fh, fw, ch);
    return 2;
}

int cgsref_device_grid_points(int dims, const float *start, const float *end, const float *count, const int64_t *idx,
                              int n, float *out, float *matrix) {
    switch (dims) {
        case 2: return device_grid_points<2>(start, end, count, idx, n, out, matrix);
        case 8: return device_grid_points<8>(start, end, count, idx, n, out, matrix);
        default: return 2;
    }
}

}  // extern "C"
