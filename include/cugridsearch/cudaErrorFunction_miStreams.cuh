/*
 * cudaErrorFunction_miStreams.cuh -- the block-cooperative normalised-MI functors of the
 * reference (src/gpu/cudaErrorFunction_miStreams.cuh:9-368), defined with the reference's
 * names and signatures.
 *
 * Both build a 64 x 64 joint histogram of floor(64 v / 256) and return
 * -2 MI / (H_fixed + H_moving).  In the reference the histogram is shared by a block and
 * filled with float atomics, per-row sums go to __shared__ arrays, and calcMIstreamAlt's
 * area accumulators are never zeroed.  Here each functor is one thread computing the same
 * quantities with the area sums starting at zero; counts are whole numbers, so the order
 * of the increments does not change them.  The searcher runs these through its generic
 * kernel (one thread per grid point).
 */
#ifndef CUGRIDSEARCH_CUDAERRORFUNCTION_MISTREAMS_CUH
#define CUGRIDSEARCH_CUDAERRORFUNCTION_MISTREAMS_CUH

#include "cudaErrorFunction_mi.cuh"
#include "cudaErrorFunctionsStreams.cuh"

namespace cgs_detail {

struct NmiHist {
    float pxy[64][64];
    float px[64], py[64];
    int total;

    CUDAFUNCTION void clear() {
        for (int i = 0; i < 64; i++) {
            px[i] = py[i] = 0;
            for (int j = 0; j < 64; j++) pxy[i][j] = 0;
        }
        total = 0;
    }

    CUDAFUNCTION void add(float fixed_value, float moving_value) {
        const int bm = mi_bin(moving_value, 64);
        const int bf = mi_bin(fixed_value, 64);
        pxy[bf][bm] += 1.0f;
        py[bm] += 1.0f;
        px[bf] += 1.0f;
        total += 1;
    }

    // -2 MI / (Hx + Hy): per fixed bin the MI terms in moving-bin order, then the bins and
    // the entropies in bin order (cudaErrorFunction_miStreams.cuh:150-205).
    template <typename F>
    CUDAFUNCTION F normalised_mi() const {
        F output = 0;
        float Hx = 0, Hy = 0;
        for (int i = 0; i < 64; i++) {
            float row = 0;
            for (int x = 0; x < 64; x++) {
                const float P = pxy[i][x] / total, Py = py[x] / total, Px = px[i] / total;
                if (P > 0 && Px > 0 && Py > 0) row += P * (log2(P) - (log2(Px) + log2(Py)));
            }
            output += row;
            const float Px = px[i] / total, Py = py[i] / total;
            if (Px > 0) Hx -= Px * log2(Px);
            if (Py > 0) Hy -= Py * log2(Py);
        }
        return -1 * 2 * output / (Hx + Hy);
    }
};

}  // namespace cgs_detail

// Scanline samples (parametricAssignValues, lambda += 1, fixed image at (row, lambda)),
// gated by the 0.25 / 0.35 overlap fractions; 123123 when a gate fails
// (cudaErrorFunction_miStreams.cuh:9-210).  Uses 16 KB of thread-local memory.
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcMIstreamAlt(nv_ext::Vec<grid_precision, D> &H, CudaImage<pixType, CHANNELS> img_moved,
                                          CudaImage<pixType, CHANNELS> img_fixed) {
    int colsf = img_fixed.width(), rowsf = img_fixed.height();
    int colsm = img_moved.width(), rowsm = img_moved.height();
    cgs_detail::NmiHist h;
    h.clear();
    float h11 = 0, h12 = 0, h13 = 0, h21 = 0, h22 = 0, h23 = 0, h31 = 0, h32 = 0;
    float cx = (float)colsm / 2, cy = (float)rowsm / 2;
    parametersToHomography<grid_precision, D>(H, cx, cy, h11, h12, h13, h21, h22, h23, h31, h32);
    float mov_area = 0, fix_area = 0;
    for (int y = 0; y < rowsf; y++) {
        float ls = 0, le = (float)colsf, vx = 0, vy = 0, p0x = 0, p0y = 0;
        bool in = false;
        parametricAssignValues(h11, h12, h13, h21, h22, h23, h31, h32, colsm, rowsm, colsf, rowsf, y, ls, le, vx, vy,
                               p0x, p0y, in);
        const float mag = sqrt((vx * vx) + (vy * vy));
        if (!in) continue;
        float row_mov = 0, row_fix = 0;
        int guard = colsf + 2;
        for (float lam = ls; lam < le && lam < colsf && guard > 0; lam += 1, guard--) {
            const float nx = (lam * vx) + p0x;
            const float ny = (lam * vy) + p0y;
            for (int c = 0; c < (int)CHANNELS; c++) {
                h.add(img_fixed.valueAt(y, lam, c), img_moved.valueAt(ny, nx, c));
                row_mov += mag;
                row_fix += 1;
            }
        }
        mov_area += row_mov;
        fix_area += row_fix;
    }
    if (mov_area / ((colsm * rowsm) * H[2]) > 0.25 && fix_area / (colsf * rowsf) > 0.35)
        return h.template normalised_mi<func_precision>();
    return (func_precision)123123.0f;
}

// Pixel-loop samples (calcNewCoordH, inImage), row by row (cudaErrorFunction_miStreams.cuh:212-368).
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcMIstream(nv_ext::Vec<grid_precision, D> &H, CudaImage<pixType, CHANNELS> img_moved,
                                       CudaImage<pixType, CHANNELS> img_fixed) {
    int colsf = img_fixed.width(), rowsf = img_fixed.height();
    cgs_detail::NmiHist h;
    h.clear();
    float h11 = 0, h12 = 0, h13 = 0, h21 = 0, h22 = 0, h23 = 0, h31 = 0, h32 = 0;
    float cx = (float)img_moved.width() / 2, cy = (float)img_moved.height() / 2;
    parametersToHomography<grid_precision, D>(H, cx, cy, h11, h12, h13, h21, h22, h23, h31, h32);
    for (int y = 0; y < rowsf; y++)
        for (int x = 0; x < colsf; x++) {
            float nx = 0, ny = 0;
            calcNewCoordH(h11, h12, h13, h21, h22, h23, h31, h32, x, y, nx, ny);
            for (int c = 0; c < (int)CHANNELS; c++)
                if (img_moved.inImage(ny, nx)) h.add(img_fixed.valueAt(y, x, c), img_moved.valueAt(ny, nx, c));
        }
    return h.template normalised_mi<func_precision>();
}

#endif  // CUGRIDSEARCH_CUDAERRORFUNCTION_MISTREAMS_CUH
