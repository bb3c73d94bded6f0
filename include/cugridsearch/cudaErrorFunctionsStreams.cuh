/*
 * cudaErrorFunctionsStreams.cuh -- the block-cooperative functors of the reference
 * (src/gpu/cudaErrorFunctionsStreams.cuh:31-351), defined with the reference's names and
 * signatures so code that takes their addresses compiles unchanged.
 *
 * In the reference each thread of a block sums one fixed-image row into a __shared__ array
 * indexed by the global row and thread 0 adds the rows up and returns the result; other
 * threads return 0 (or nothing, for rows past the image: undefined behaviour), and every
 * thread writes its return value to the same result element.  Here each functor is a
 * single-thread function computing what thread 0 computes -- per-row partial sums added in
 * row order, with each variant's own gates and no-overlap values -- so every caller gets
 * the same, deterministic value.  The searcher runs these through its generic kernel (one
 * thread per grid point); THREADS_PER_BLOCK is kept for source compatibility only.
 */
#ifndef CUGRIDSEARCH_CUDAERRORFUNCTIONSSTREAMS_CUH
#define CUGRIDSEARCH_CUDAERRORFUNCTIONSSTREAMS_CUH

#include "cudaErrorFunctions.cuh"

#ifndef THREADS_PER_BLOCK
#define THREADS_PER_BLOCK 1024
#endif

// Mean |m - f| under the translation (t[0], t[1]) (cudaErrorFunctionsStreams.cuh:31-83):
// row partials over (channel, x), then rows in order; no overlap gives 0 (count 0 -> 1).
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision averageAbsoluteDifference_stream(nv_ext::Vec<grid_precision, D> &t,
                                                           CudaImage<pixType, CHANNELS> img_moved,
                                                           CudaImage<pixType, CHANNELS> img_fixed) {
    float total = 0;
    int count = 0;
    for (int y = 0; y < img_fixed.height(); y++) {
        float row_sum = 0;
        int row_n = 0;
        for (int c = 0; c < (int)CHANNELS; c++)
            for (int x = 0; x < img_fixed.width(); x++)
                if (img_moved.inImage(y + t[1], x + t[0])) {
                    row_sum += fabsf(img_moved.valueAt(y + t[1], x + t[0], c) - img_fixed.valueAt(y, x, c));
                    row_n++;
                }
        total += row_sum;
        count += row_n;
    }
    if (count == 0) count = 1;
    return (func_precision)total / count;
}

// calcNCC with row partials (cudaErrorFunctionsStreams.cuh:85-163); 0 unless both energies
// are positive.
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcNCCstream(nv_ext::Vec<grid_precision, D> &H, CudaImage<pixType, CHANNELS> img_moved,
                                        CudaImage<pixType, CHANNELS> img_fixed) {
    return cgs_detail::pixel_sqd_ncc<true, func_precision>(H, img_moved, img_fixed, true);
}

// calcNCCAlt with row partials (cudaErrorFunctionsStreams.cuh:165-281); 0 (not 123123)
// when the overlap gates fail.
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcNCCstreamAlt(nv_ext::Vec<grid_precision, D> &H, CudaImage<pixType, CHANNELS> img_moved,
                                           CudaImage<pixType, CHANNELS> img_fixed) {
    return cgs_detail::scan_sqd_ncc<true, func_precision>(H, img_moved, img_fixed, true);
}

// calcSQD with row partials (cudaErrorFunctionsStreams.cuh:283-351); no overlap gives
// 0 / 0 = NaN (no 123123 sentinel).
template <typename func_precision, typename grid_precision, uint32_t D, uint32_t CHANNELS, typename pixType>
CUDAFUNCTION func_precision calcSQDstream(nv_ext::Vec<grid_precision, D> &H, CudaImage<pixType, CHANNELS> img_moved,
                                        CudaImage<pixType, CHANNELS> img_fixed) {
    return cgs_detail::pixel_sqd_ncc<false, func_precision>(H, img_moved, img_fixed, true);
}

#endif  // CUGRIDSEARCH_CUDAERRORFUNCTIONSSTREAMS_CUH
