/*
 * cudaErrorFunction_mi.cuh -- mutual-information functors (reference:
 * src/gpu/cudaErrorFunction_mi.cuh:8-255).
 *
 *   calcMIAlt  -- the reference's scanline MI: normalised coordinates, 64 bins of
 *                 floor(64 v / 256), float counts, result -MI x fix_area (:117-255).
 *   calcMI     -- the reference's calcMI does not compile (:27); here it is the library's
 *                 exact MI cost (CGS_COST_MI) with 32 bins: integer joint counts of
 *                 floor(32 v / 256) over the calcNCC samples, -MI x overlap / (W_f H_f C),
 *                 +inf when nothing overlaps.
 *   calcMIBins -- the same with BINS bins (a power of two from 2 to 64).
 *
 * Like the functors of cudaErrorFunctions.cuh, these bodies run only when called directly
 * or through the generic kernel; the searcher runs recognised pointers on the fused kernel.
 */
#ifndef CUGRIDSEARCH_CUDAERRORFUNCTION_MI_CUH
#define CUGRIDSEARCH_CUDAERRORFUNCTION_MI_CUH

#ifndef CUDAFUNCTION
#define CUDAFUNCTION __host__ __device__
#endif

#include <cmath>
#include <cstdint>

#include "cudaImageFunctions.cuh"
#include "cudaTensor.cuh"
#include "nvVectorNd.h"

namespace cgs_detail {

// floor(bins * (v / 256)) as an index; values outside [0, 256) (undefined behaviour in the
// reference, which indexes its arrays with the result) are clamped to the end bins.
CUDAFUNCTION inline int mi_bin(float v, int bins) {
    const float b = floor(bins * (v / 256.0f));
    if (!(b >= 0.0f)) return 0;
    return b > (float)(bins - 1) ? bins - 1 : (int)b;
}

// Exact-count MI over the calcNCC samples (centred homography, calcNewCoordH, inImage).
template <int BINS, unsigned int D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION float mi_exact(nv_ext::Vec<float, D> &parameters, const CudaImage<pixType, CHANNELS> &img_moved,
                            const CudaImage<pixType, CHANNELS> &img_fixed) {
    static_assert(BINS >= 2 && BINS <= 64 && (BINS & (BINS - 1)) == 0, "BINS must be a power of two in [2, 64]");
    int colsf = img_fixed.width(), rowsf = img_fixed.height();
    float h11 = 0, h12 = 0, h13 = 0, h21 = 0, h22 = 0, h23 = 0, h31 = 0, h32 = 0;
    float cx = (float)img_moved.width() / 2, cy = (float)img_moved.height() / 2;
    parametersToHomography<float, D>(parameters, cx, cy, h11, h12, h13, h21, h22, h23, h31, h32);
    uint32_t cnt[BINS * BINS];
    for (int i = 0; i < BINS * BINS; i++) cnt[i] = 0;
    uint32_t n = 0;
    for (int x = 0; x < colsf; x++)
        for (int y = 0; y < rowsf; y++) {
            float nx = 0, ny = 0;
            calcNewCoordH(h11, h12, h13, h21, h22, h23, h31, h32, x, y, nx, ny);
            if (!img_moved.inImage(ny, nx)) continue;
            for (int c = 0; c < (int)CHANNELS; c++) {
                const int bf = mi_bin(img_fixed.valueAt(y, x, c), BINS);
                const int bm = mi_bin(img_moved.valueAt_bilinear(ny, nx, c), BINS);
                cnt[bf * BINS + bm] += 1;
                n++;
            }
        }
    if (n == 0) return INFINITY;
    double hf[BINS], hm[BINS];
    for (int i = 0; i < BINS; i++) hf[i] = hm[i] = 0;
    for (int i = 0; i < BINS; i++)
        for (int j = 0; j < BINS; j++) {
            hf[i] += cnt[i * BINS + j];
            hm[j] += cnt[i * BINS + j];
        }
    double acc = 0;
    const double dn = (double)n;
    for (int i = 0; i < BINS; i++)
        for (int j = 0; j < BINS; j++) {
            const double v = cnt[i * BINS + j];
            if (v > 0) acc += v * log2(v * dn / (hf[i] * hm[j]));
        }
    const double total = (double)colsf * rowsf * CHANNELS;
    return (float)(-(acc / dn) * (dn / total));
}

}  // namespace cgs_detail

// Scanline MI in normalised coordinates (cudaErrorFunction_mi.cuh:117-255).  As in the
// reference, parameters[1] and parameters[2] are rescaled in place by
// parametersToHomographyNorm.  Fixed samples are taken at (row, lambda) mapped back to
// pixels; the float row and lambda recurrences and the double fix_area steps are the
// reference's.
template <typename func_precision, typename grid_precision, uint8_t D = 8, uint8_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcMIAlt(nv_ext::Vec<grid_precision, D> &parameters,
                                      CudaImage<pixType, CHANNELS> img_moved, CudaImage<pixType, CHANNELS> img_fixed) {
    int colsf = img_fixed.width(), rowsf = img_fixed.height();
    int colsm = img_moved.width(), rowsm = img_moved.height();
    const int binN = 64;
    func_precision output = 0;
    float h11 = 0, h12 = 0, h13 = 0, h21 = 0, h22 = 0, h23 = 0, h31 = 0, h32 = 0;
    float pxy[64][64];
    float px[64], py[64];
    for (int i = 0; i < 64; i++) {
        px[i] = py[i] = 0;
        for (int j = 0; j < 64; j++) pxy[i][j] = 0;
    }
    int count = 0;
    float fix_area = 0;
    parametersToHomographyNorm<float, 8>(parameters, colsm, rowsm, colsf, rowsf, h11, h12, h13, h21, h22, h23, h31,
                                         h32);
    int row_guard = rowsf + 2;
    for (float row = -0.5; row < 0.5 && row_guard > 0; row += 1 / ((float)(rowsf - 1)), row_guard--) {
        float ls = 0, le = 1, vx = 0, vy = 0, p0x = 0, p0y = 0;
        bool in = false;
        parametricAssignValuesNorm(h11, h12, h13, h21, h22, h23, h31, h32, colsm, rowsm, colsf, rowsf, row, ls, le, vx,
                                   vy, p0x, p0y, in);
        if (!in) continue;
        int guard = colsf + 2;
        for (float lam = ls; lam < le && lam < 1 && guard > 0; lam += 1 / ((float)(colsf - 1)), guard--) {
            float nx = (lam * vx) + p0x;
            float ny = (lam * vy) + p0y;
            nx = (nx + 0.5) * (colsm);
            ny = (ny + 0.5) * (rowsm);
            const float rowIdx = ((row + 0.5) * (rowsf - 1));
            const float lamIdx = (lam * (colsf - 1));
            for (int c = 0; c < (int)CHANNELS; c++) {
                const int bx = cgs_detail::mi_bin(img_fixed.valueAt(rowIdx, lamIdx, c), binN);
                const int by = cgs_detail::mi_bin(img_moved.valueAt(ny, nx, c), binN);
                pxy[bx][by] += (1.0f);
                px[bx] += (1.0f);
                py[by] += (1.0f);
                count += 1;
            }
            fix_area += 1.0 / (colsf * rowsf);
        }
    }
    for (int i = 0; i < binN * binN; i++) {
        if (i < binN) {
            px[i] /= count;
            py[i] /= count;
        }
        pxy[i / binN][i % binN] /= count;
    }
    for (int x = 0; x < binN; x++)
        for (int y = 0; y < binN; y++) {
            const float P = pxy[x][y], Px = px[x], Py = py[y];
            if (P > 0 && Px > 0 && Py > 0) output += P * (log2(P) - (log2(Px) + log2(Py)));
        }
    return -1 * output * fix_area;
}

template <typename func_precision, typename grid_precision, uint8_t D = 8, uint8_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcMI(nv_ext::Vec<grid_precision, D> &parameters, CudaImage<pixType, CHANNELS> img_moved,
                                   CudaImage<pixType, CHANNELS> img_fixed) {
    return (func_precision)cgs_detail::mi_exact<32>(parameters, img_moved, img_fixed);
}

template <typename func_precision, typename grid_precision, uint8_t D, uint8_t CHANNELS, typename pixType, int BINS>
CUDAFUNCTION func_precision calcMIBins(nv_ext::Vec<grid_precision, D> &parameters,
                                       CudaImage<pixType, CHANNELS> img_moved, CudaImage<pixType, CHANNELS> img_fixed) {
    return (func_precision)cgs_detail::mi_exact<BINS>(parameters, img_moved, img_fixed);
}

#endif  // CUGRIDSEARCH_CUDAERRORFUNCTION_MI_CUH
