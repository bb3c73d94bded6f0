/*
 * cudaErrorFunctions.cuh -- the grid search's image-similarity functors (reference:
 * src/gpu/cudaErrorFunctions.cuh:31-507), as __host__ __device__ templates with the
 * reference's names and signatures, plus calcZNCC (no reference counterpart).
 *
 * How they run.  Passed to CudaGridSearcher as a device function pointer, a functor
 * listed in cudaGridSearch.cuh's dispatch table never executes this body: the searcher
 * recognises the pointer and runs the fused sm_100a search kernel of the library with
 * the matching cost (bit-identical results for the reference functors, within 1e-5
 * relative for calcZNCC).  The bodies below run when a functor is called directly (on the
 * host, as the reference's "Min Value check" does) and for instantiations the library has
 * no kernel for, through the searcher's generic one-thread-per-grid-point kernel.
 *
 * Each body evaluates the reference's expressions in the reference's order, so a host
 * build reproduces the reference's FP32 results bit for bit; the only deliberate
 * differences are at the reference's undefined behaviour: taps past the end of the image
 * read 0 (CudaImage::valueAt_bilinear) and the per-index device printf of
 * averageAbsoluteDifference (:82-85) is not issued.
 */
#ifndef CUGRIDSEARCH_CUDAERRORFUNCTIONS_CUH
#define CUGRIDSEARCH_CUDAERRORFUNCTIONS_CUH

#ifndef CUDAFUNCTION
#define CUDAFUNCTION __host__ __device__
#endif

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "cudaImageFunctions.cuh"
#include "cudaTensor.cuh"
#include "nvVectorNd.h"

namespace cgs_detail {

// One scanline sweep of calcSQDAlt / calcNCCAlt (cudaErrorFunctions.cuh:226-376): lambda
// starts at the row's entry point and steps by 1 (float) while below the exit point and
// the image width.  lambda_start is never negative (parametricAssignValues only assigns
// crossings in [0, f_width)), so a row takes at most colsf + 1 steps.
template <bool NCC, typename O, unsigned int D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION O scan_sqd_ncc(nv_ext::Vec<float, D> &parameters, const CudaImage<pixType, CHANNELS> &img_moved,
                                const CudaImage<pixType, CHANNELS> &img_fixed, bool stream_sums) {
    int colsf = img_fixed.width(), rowsf = img_fixed.height();
    int colsm = img_moved.width(), rowsm = img_moved.height();
    float h11 = 0, h12 = 0, h13 = 0, h21 = 0, h22 = 0, h23 = 0, h31 = 0, h32 = 0;
    float cx = (float)colsm / 2, cy = (float)rowsm / 2;
    parametersToHomography<float, D>(parameters, cx, cy, h11, h12, h13, h21, h22, h23, h31, h32);
    // running sums (the result sum in the functor's return type, as the reference's
    // func_precision output); with stream_sums each row is summed separately and the rows are then
    // added in order (calcNCCstreamAlt, cudaErrorFunctionsStreams.cuh:165-281)
    O out = 0;
    float i1 = 0, i2 = 0, mov_area = 0, fix_area = 0;
    for (int row = 0; row < rowsf; row++) {
        float ls = 0, le = (float)colsf, vx = 0, vy = 0, p0x = 0, p0y = 0;
        bool in = false;
        parametricAssignValues(h11, h12, h13, h21, h22, h23, h31, h32, colsm, rowsm, colsf, rowsf, row, ls, le, vx, vy,
                               p0x, p0y, in);
        const float mag = sqrt((vx * vx) + (vy * vy));
        if (!in) continue;  // the reference walks lambda here without effect
        O r_out = 0;
        float r_i1 = 0, r_i2 = 0, r_mov = 0, r_fix = 0;
        O &o = stream_sums ? r_out : out;
        float &a = stream_sums ? r_i1 : i1, &b = stream_sums ? r_i2 : i2;
        float &ma = stream_sums ? r_mov : mov_area, &fa = stream_sums ? r_fix : fix_area;
        int guard = colsf + 2;
        for (float lam = ls; lam < le && lam < colsf && guard > 0; lam += 1, guard--) {
            const float nx = (lam * vx) + p0x;
            const float ny = (lam * vy) + p0y;
            for (int c = 0; c < (int)CHANNELS; c++) {
                float vm = img_moved.valueAt_bilinear(ny, nx, c);
                float vf = img_fixed.valueAt_bilinear(row, lam, c);
                vm /= 255.0f;
                vf /= 255.0f;
                if (NCC) o += vm * vf;
                else o += (vm - vf) * (vm - vf);
                a += vm * vm;
                b += vf * vf;
            }
            ma += mag;
            fa += 1;
        }
        if (stream_sums) {
            out += r_out;
            i1 += r_i1;
            i2 += r_i2;
            mov_area += r_mov;
            fix_area += r_fix;
        }
    }
    const bool gate = mov_area / ((colsm * rowsm) * parameters[2]) > 0.25 && fix_area / (colsf * rowsf) > 0.35;
    if (!gate) return stream_sums ? (O)0 : (O)123123.0f;
    if (NCC) return (-1 * out) / sqrt(i1 * i2);
    return out / sqrt(i1 * i2);
}

// calcSQD / calcNCC pixel loop (cudaErrorFunctions.cuh:378-507): x outer, y inner, channel
// innermost; centred homography; samples where the mapped point is inside the moving image.
// With stream_sums each row is summed separately (calcSQDstream / calcNCCstream,
// cudaErrorFunctionsStreams.cuh:85-163, 283-351: row y, x loop, then rows added in order).
template <bool NCC, typename O, unsigned int D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION O pixel_sqd_ncc(nv_ext::Vec<float, D> &parameters, const CudaImage<pixType, CHANNELS> &img_moved,
                                 const CudaImage<pixType, CHANNELS> &img_fixed, bool stream_sums) {
    int colsf = img_fixed.width(), rowsf = img_fixed.height();
    int colsm = img_moved.width(), rowsm = img_moved.height();
    float h11 = 0, h12 = 0, h13 = 0, h21 = 0, h22 = 0, h23 = 0, h31 = 0, h32 = 0;
    float cx = (float)colsm / 2, cy = (float)rowsm / 2;
    parametersToHomography<float, D>(parameters, cx, cy, h11, h12, h13, h21, h22, h23, h31, h32);
    // the SQD sum has the functor's return type (func_precision output), the NCC sums are float
    typedef typename std::conditional<NCC, float, O>::type Acc;
    Acc out = 0;
    float i1 = 0, i2 = 0, n = 0;
    auto sample = [&](int x, int y, Acc &o, float &a, float &b, float &cnt) {
        float nx = 0, ny = 0;
        calcNewCoordH(h11, h12, h13, h21, h22, h23, h31, h32, x, y, nx, ny);
        for (int c = 0; c < (int)CHANNELS; c++) {
            if (!img_moved.inImage(ny, nx)) continue;
            const float temp = img_moved.valueAt_bilinear(ny, nx, c) / 255.0f;
            const float f = img_fixed.valueAt(y, x, c);
            if (NCC) {
                a += ((float)f / 255.0f) * (float)f / 255.0f;  // i1: fixed energy
                b += temp * temp;
                o += ((float)f / 255.0f) * temp;
            } else {
                o += (temp - f / 255.0f) * (temp - f / 255.0f);
                a += temp * temp;  // i1: moving energy
                b += (f / 255.0f) * f / 255.0f;
            }
            cnt += 1;
        }
    };
    if (!stream_sums) {
        for (int x = 0; x < colsf; x++)
            for (int y = 0; y < rowsf; y++) sample(x, y, out, i1, i2, n);
        if (NCC) return n > 0 ? (O)((-1 * out) / sqrt(i1 * i2)) : (O)0;
        return n > 0 ? (O)(out / sqrt(i1 * i2)) : (O)123123.0f;
    }
    for (int y = 0; y < rowsf; y++) {
        Acc r_o = 0;
        float r_a = 0, r_b = 0, r_n = 0;
        for (int x = 0; x < colsf; x++) sample(x, y, r_o, r_a, r_b, r_n);
        out += r_o;
        i1 += r_a;
        i2 += r_b;
        n += r_n;
    }
    if (NCC) return (i1 > 0 && i2 > 0) ? (O)((-1 * out) / sqrt(i1 * i2)) : (O)0;
    return (O)(out / sqrt(i1 * i2));
}

// Zero-mean NCC over the calcNCC samples, in double:
//   -sum((f - mf)(m - mm)) / sqrt(sum((f - mf)^2) sum((m - mm)^2)),
// +inf when nothing overlaps or either image is constant over the overlap.
template <unsigned int D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION float zncc(nv_ext::Vec<float, D> &parameters, const CudaImage<pixType, CHANNELS> &img_moved,
                        const CudaImage<pixType, CHANNELS> &img_fixed) {
    int colsf = img_fixed.width(), rowsf = img_fixed.height();
    float h11 = 0, h12 = 0, h13 = 0, h21 = 0, h22 = 0, h23 = 0, h31 = 0, h32 = 0;
    float cx = (float)img_moved.width() / 2, cy = (float)img_moved.height() / 2;
    parametersToHomography<float, D>(parameters, cx, cy, h11, h12, h13, h21, h22, h23, h31, h32);
    double sf = 0, sm = 0, sff = 0, smm = 0, sfm = 0, n = 0;
    for (int x = 0; x < colsf; x++)
        for (int y = 0; y < rowsf; y++) {
            float nx = 0, ny = 0;
            calcNewCoordH(h11, h12, h13, h21, h22, h23, h31, h32, x, y, nx, ny);
            if (!img_moved.inImage(ny, nx)) continue;
            for (int c = 0; c < (int)CHANNELS; c++) {
                const double m = (double)img_moved.valueAt_bilinear(ny, nx, c) - 127.5;
                const double f = (double)img_fixed.valueAt(y, x, c) - 127.5;
                sf += f;
                sm += m;
                sff += f * f;
                smm += m * m;
                sfm += f * m;
                n += 1;
            }
        }
    const float inf = INFINITY;
    if (n == 0) return inf;
    const double cov = sfm - sf * sm / n, vf = sff - sf * sf / n, vm = smm - sm * sm / n;
    if (!(vf > 0) || !(vm > 0)) return inf;
    return (float)(-cov / sqrt(vf * vm));
}

}  // namespace cgs_detail

// Mean |m - f| over the overlap, homography WITHOUT centring (h13 = sx*tx, h23 = sy*ty),
// loops c, x, y (cudaErrorFunctions.cuh:31-87).  No overlap gives 0/0 = NaN, as in the
// reference.
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision averageAbsoluteDifference(nv_ext::Vec<grid_precision, D> &parameters,
                                                      CudaImage<pixType, CHANNELS> img_moved,
                                                      CudaImage<pixType, CHANNELS> img_fixed) {
    int num_errors = 0;
    const float th = parameters[0], sx = parameters[1], sy = parameters[2], sh = parameters[3];
    const float tx = parameters[4], ty = parameters[5];
    const float h11 = sx * cos(th);
    const float h12 = ((sy * sh) * cos(th)) - (sy * sin(th));
    const float h13 = sx * tx;
    const float h21 = sx * sin(th);
    const float h22 = ((sy * sh) * sin(th)) + (sy * cos(th));
    const float h23 = sy * ty;
    const float h31 = parameters[6];
    const float h32 = parameters[7];
    float sum = 0;
    for (int c = 0; c < (int)CHANNELS; c++) {
        for (int x = 0; x < img_fixed.width(); x++) {
            for (int y = 0; y < img_fixed.height(); y++) {
                const float w = ((((h21 * h32) - (h22 * h31)) * x + ((h12 * h31) - (h11 * h32)) * y) + (h11 * h22)) -
                                (h12 * h21);
                const float nx = (((((h22 - (h23 * h32)) * x) + ((h13 * h32) - h12) * y) + (h12 * h23)) - (h13 * h22)) / w;
                const float ny = (((((h23 * h31) - h21) * x + (h11 - (h13 * h31)) * y) + (h13 * h21)) - (h11 * h23)) / w;
                if (img_moved.inImage(ny, nx)) {
                    sum += fabsf(img_moved.valueAt(ny, nx, c) - img_fixed.valueAt(y, x, c));
                    num_errors++;
                }
            }
        }
    }
    return (func_precision)sum / num_errors;
}

// Sum of |m - f| under the translation (t[0], t[1]), samples inside the moving image only
// (cudaErrorFunctions.cuh:89-114).
template <typename func_precision, typename grid_precision, unsigned int D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision sumOfAbsoluteDifferences(nv_ext::Vec<grid_precision, D> &t, CudaImage<pixType> img_moved,
                                                     CudaImage<pixType> img_fixed) {
    float sum = 0;
    for (int c = 0; c < (int)CHANNELS; c++)
        for (int x = 0; x < img_fixed.width(); x++)
            for (int y = 0; y < img_fixed.height(); y++)
                if (img_moved.inImage(y + t[1], x + t[0]))
                    sum += fabsf(img_moved.valueAt(y + t[1], x + t[0], c) - img_fixed.valueAt(y, x, c));
    return (func_precision)sum;
}

// The by-reference form (cudaErrorFunctions.cuh:171-192): every fixed pixel, samples outside
// the moving image read as 0.
template <typename func_precision, typename grid_precision, unsigned int D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision sumOfAbsoluteDifferences(nv_ext::Vec<grid_precision, D> &t, CudaImage<pixType> *img_moved,
                                                     CudaImage<pixType> *img_fixed) {
    float sum = 0;
    for (int c = 0; c < (int)CHANNELS; c++)
        for (int x = 0; x < img_fixed->width(); x++)
            for (int y = 0; y < img_fixed->height(); y++)
                sum += fabsf(img_moved->valueAt(y + t[1], x + t[0], c) - img_fixed->valueAt(y, x, c));
    return (func_precision)sum;
}

// Mean |m - f| with the 8 grid values used as the raw homography H = [h11 h12 h13; h21 h22
// h23; h31 h32 1] mapping fixed -> moving directly (cudaErrorFunctions.cuh:194-224).
template <typename func_precision, typename grid_precision, unsigned int D = 8, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision averageAbsoluteDifferenceH(nv_ext::Vec<grid_precision, D> &H, CudaImage<pixType> img_moved,
                                                       CudaImage<pixType> img_fixed) {
    int num_errors = 0;
    float sum = 0;
    for (int c = 0; c < (int)CHANNELS; c++) {
        for (int x = 0; x < img_fixed.width(); x++) {
            for (int y = 0; y < img_fixed.height(); y++) {
                // H[6]*x + H[7]*y + 1.0: the float sum plus a double 1.0, rounded once to float
                const float z = (float)((double)((H[6] * x) + (H[7] * y)) + 1.0);
                const float yp = (((H[3] * x) + (H[4] * y)) + H[5]) / z;
                const float xp = (((H[0] * x) + (H[1] * y)) + H[2]) / z;
                if (img_moved.inImage(yp, xp)) {
                    sum += fabsf(img_moved.valueAt(yp, xp, c) - img_fixed.valueAt(y, x, c));
                    num_errors++;
                }
            }
        }
    }
    return (func_precision)sum / num_errors;
}

// Scanline SQD (cudaErrorFunctions.cuh:226-300): sum (m-f)^2 / sqrt(sum m^2 sum f^2) on
// values / 255; 123123 unless the overlap passes the 0.25 (moving) / 0.35 (fixed) gates.
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcSQDAlt(nv_ext::Vec<grid_precision, D> &parameters,
                                       CudaImage<pixType, CHANNELS> img_moved, CudaImage<pixType, CHANNELS> img_fixed) {
    return (func_precision)cgs_detail::scan_sqd_ncc<false, func_precision>(parameters, img_moved, img_fixed, false);
}

// Scanline NCC (cudaErrorFunctions.cuh:302-376): -sum m f / sqrt(sum m^2 sum f^2).
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcNCCAlt(nv_ext::Vec<grid_precision, D> &parameters,
                                       CudaImage<pixType, CHANNELS> img_moved, CudaImage<pixType, CHANNELS> img_fixed) {
    return (func_precision)cgs_detail::scan_sqd_ncc<true, func_precision>(parameters, img_moved, img_fixed, false);
}

// Pixel-loop SQD (cudaErrorFunctions.cuh:378-446); 123123 when nothing overlaps.
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcSQD(nv_ext::Vec<grid_precision, D> &parameters, CudaImage<pixType, CHANNELS> img_moved,
                                    CudaImage<pixType, CHANNELS> img_fixed) {
    return (func_precision)cgs_detail::pixel_sqd_ncc<false, func_precision>(parameters, img_moved, img_fixed, false);
}

// Pixel-loop NCC (cudaErrorFunctions.cuh:448-507); 0 when nothing overlaps.
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcNCC(nv_ext::Vec<grid_precision, D> &parameters, CudaImage<pixType, CHANNELS> img_moved,
                                    CudaImage<pixType, CHANNELS> img_fixed) {
    return (func_precision)cgs_detail::pixel_sqd_ncc<true, func_precision>(parameters, img_moved, img_fixed, false);
}

// Zero-mean NCC over the calcNCC samples (no reference counterpart; the library's
// CGS_COST_ZNCC with no overlap gate).
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcZNCC(nv_ext::Vec<grid_precision, D> &parameters,
                                     CudaImage<pixType, CHANNELS> img_moved, CudaImage<pixType, CHANNELS> img_fixed) {
    return (func_precision)cgs_detail::zncc(parameters, img_moved, img_fixed);
}

#endif  // CUGRIDSEARCH_CUDAERRORFUNCTIONS_CUH
