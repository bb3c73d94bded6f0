/*
 * cugridsearch_b200.h -- C ABI of the B200 (sm_100a) homography grid search.
 *
 * The hot path of uncc-visionlab/cuGridSearch is an exhaustive search over an
 * 8-parameter homography grid for the argmin of an image-similarity cost.  This header
 * is the drop-in boundary for that path: plain C types, caller-owned device pointers,
 * status codes instead of exit(), and an explicit CUDA stream on every call.  Each
 * entry point names the reference interface it replaces (file:line in the reference).
 *
 * Threading: every call is safe to issue from several host threads; device scratch is
 * stream-ordered (taken from a library memory pool on the given stream), so calls on
 * different streams do not share scratch.  Asynchronous calls return before the GPU
 * work finishes; results become valid when the stream reaches them.
 */
#ifndef CUGRIDSEARCH_B200_H
#define CUGRIDSEARCH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same type as the CUDA runtime's cudaStream_t; 0 is the legacy default stream. */
typedef struct CUstream_st *cgs_stream_t;

typedef enum cgs_status {
    CGS_SUCCESS = 0,
    CGS_ERROR_INVALID_VALUE = 1,   /* bad descriptor, size or option                        */
    CGS_ERROR_UNSUPPORTED = 2,     /* valid request this build does not implement           */
    CGS_ERROR_GRID_TOO_LARGE = 3,  /* more than 2^31 - 1 grid points (reference int32 index) */
    CGS_ERROR_OUT_OF_MEMORY = 4,   /* device scratch could not be allocated                 */
    CGS_ERROR_CUDA = 5,            /* a CUDA runtime call failed; see cgs_last_error()       */
    CGS_ERROR_NO_DEVICE = 6,       /* no sm_100 device, or the kernels cannot load          */
    CGS_ERROR_DEVICE_TIMEOUT = 7   /* a bounded device-side wait gave up                    */
} cgs_status;

/* Cost functions.  0-8 reproduce the reference functors; 9-10 are the benchmark costs. */
typedef enum cgs_cost {
    CGS_COST_SAD_AVG = 0,       /* averageAbsoluteDifference   src/gpu/cudaErrorFunctions.cuh:31-87    */
    CGS_COST_SAD_AVG_H = 1,     /* averageAbsoluteDifferenceH  src/gpu/cudaErrorFunctions.cuh:194-224  */
    CGS_COST_SAD_SUM_T = 2,     /* sumOfAbsoluteDifferences, by value      cudaErrorFunctions.cuh:89-114  */
    CGS_COST_SAD_SUM_T_REF = 3, /* sumOfAbsoluteDifferences, by reference  cudaErrorFunctions.cuh:171-192 */
    CGS_COST_SQD_REF = 4,       /* calcSQD      src/gpu/cudaErrorFunctions.cuh:378-446 */
    CGS_COST_NCC_REF = 5,       /* calcNCC      src/gpu/cudaErrorFunctions.cuh:448-507 */
    CGS_COST_SQD_ALT = 6,       /* calcSQDAlt   src/gpu/cudaErrorFunctions.cuh:226-300 */
    CGS_COST_NCC_ALT = 7,       /* calcNCCAlt   src/gpu/cudaErrorFunctions.cuh:302-376 */
    CGS_COST_MI_ALT = 8,        /* calcMIAlt    src/gpu/cudaErrorFunction_mi.cuh:117-255 (64 bins) */
    CGS_COST_ZNCC = 9,          /* zero-mean NCC over the calcNCC sampling                 */
    CGS_COST_MI = 10,           /* -MI x overlap fraction from exact B x B integer counts   */
    CGS_COST_COUNT = 11
} cgs_cost;

/* Pixel types of CudaImage<T, C>.  Every tap is converted to float as the reference's
 * valueAt_bilinear does (float tlc = _data[...], include/cudaTensor.cuh:563). */
typedef enum cgs_pixel { CGS_PIXEL_F32 = 0, CGS_PIXEL_U8 = 1, CGS_PIXEL_F64 = 2, CGS_PIXEL_U16 = 3 } cgs_pixel;

/* CudaImage<T, C> (include/cudaTensor.cuh:507-596): dims {C, W, H}, HWC row-major,
 * element (y, x, c) at c + C * (x + W * y).  data is a caller-owned DEVICE pointer. */
typedef struct cgs_image {
    const void *data;
    int32_t height, width, channels; /* channels 1..4 */
    int32_t pixel;                   /* cgs_pixel */
} cgs_image;

/* CudaGrid<float, D> (src/gpu/cudaGridSearch.cuh:74-79): the 4 x D matrix of rows
 * {start, end, resolution, count}.  Counts are floats, as in the reference.  Fill
 * start/end/count and call cgs_grid_update() before searching (the reference's setters
 * each call update(), cudaGridSearch.cuh:198-215). */
typedef struct cgs_grid {
    int32_t dims; /* 1..8 */
    float start[8];
    float end[8];
    float resolution[8];
    float count[8];
} cgs_grid;

typedef struct cgs_options {
    int32_t cost;            /* cgs_cost */
    int32_t mi_bins;         /* CGS_COST_MI: power of two in [2, 64]; 0 means 32 */
    float overlap_gate;      /* CGS_COST_ZNCC / CGS_COST_MI: minimum overlap fraction of the
                                fixed image (pixels x channels), else the cost is +inf */
    int32_t points_per_warp; /* 0 = tuned; else 1, 2 or 4 */
    int32_t warps_per_block; /* 0 = tuned; else 4, 8 or 16 */
    int32_t flags;           /* CGS_FLAG_* */
} cgs_options;

/* Evaluate grid points in the reference's index order (axis 0 fastest) instead of the
 * locality order the library picks.  Results are identical; only speed differs. */
#define CGS_FLAG_NATURAL_ORDER 1
/* Sampling modes.  Every mode makes the reference's discrete decisions exactly (which
 * samples fall inside the moving image; MI bins).  EXACT additionally forms every sample
 * with the reference's operation sequence, so sample values are bit-identical to the
 * reference's host path; FAST forms them with fused arithmetic (FP32-accurate, about 1e-6
 * relative) and is about twice as fast.  Default: EXACT for the reference functors (costs
 * 0-8), FAST for CGS_COST_ZNCC and CGS_COST_MI.  The scanline functors (6-8) are always exact. */
#define CGS_FLAG_EXACT_SAMPLES 2
#define CGS_FLAG_FAST_SAMPLES 4
/* Where the 2x2 bilinear taps come from.  QUAD: a staged copy of the moving image that holds
 * each pixel's footprint as one 16-byte element (4x the moving image in scratch); TEXTURE:
 * texture gathers (scalar loads for MI).  Default: quads for the fast sampling path of every
 * cost but MI, texture otherwise (the faster choice measured on B200).  Results are identical;
 * only speed and scratch size differ. */
#define CGS_FLAG_QUAD_TAPS 8
#define CGS_FLAG_TEXTURE_TAPS 16
/* Zero-mean NCC and MI on the fast path run span kernels by default (single channel; MI with
 * at most 32 bins and neither taps flag): in/out decisions per image row; ZNCC reads its taps
 * from per-block moving-image windows in shared memory, MI keeps its histograms there.  This
 * flag selects the per-sample decision kernel instead.  Both make the same decisions and form
 * the same bins: ZNCC costs agree within FP32 summation order, MI costs are bit-identical. */
#define CGS_FLAG_PER_SAMPLE_DECISIONS 32
/* Skip the FP64 verification pass (see cgs_argmin).  Without the pass the verification fields
 * read verified = 0, index_fp64 = -1, cost_fp64 = NaN. */
#define CGS_FLAG_NO_VERIFY 64

/* Argmin of a search: the lowest cost, ties broken by the lowest grid index.  NaN and
 * +inf costs never win (the reference compares with '<', cudaTensor.cuh:256 and
 * cudaTensorKernels.cuh:45-49); if no cost is finite, valid = 0 and index = -1.
 *
 * FP64 verification (cgs_search, unless CGS_FLAG_NO_VERIFY): the search sums in FP32; afterwards
 * every grid point whose FP32 cost lies within 2e-5 x max(1, |cost|) of the minimum (at most
 * CGS_VERIFY_MAX of them) is re-scored on the device with the reference's exact sampling and FP64
 * sums -- the arithmetic of an FP64 CPU oracle -- and the fields below report the result.  The
 * band is twice the per-point FP32 tolerance, so index_fp64 is the FP64 argmin of the whole grid
 * whenever the FP32 costs are within that tolerance. */
#define CGS_VERIFY_MAX 64
typedef struct cgs_argmin {
    float cost;
    int32_t valid;
    int64_t index;
    float params[8];      /* grid point of index, decoded as CudaGrid::getGridPoint does */
    int32_t status;       /* cgs_status of the device work (CGS_ERROR_DEVICE_TIMEOUT if a wait gave up) */
    int32_t verified;     /* grid points re-scored in FP64 (0: no verification pass ran) */
    int32_t candidates;   /* grid points in the band (> verified: the first CGS_VERIFY_MAX found were re-scored) */
    int32_t reserved;
    int64_t index_fp64;   /* lowest FP64 cost among the re-scored points, lowest index on ties (-1: none) */
    double cost_fp64;     /* FP64 cost of `index` (NaN if not verified) */
    double err_fp64;      /* |cost - cost_fp64| */
    double max_err_fp64;  /* largest |FP32 cost - FP64 cost| over the re-scored points */
} cgs_argmin;

/* CudaGrid::update(changed_axis) -- updateProcess<<<1,1>>> (src/gpu/cudaGridSearch.cuh:100-105,
 * 235-272), computed on the host with the same FP32 arithmetic. */
cgs_status cgs_grid_update(cgs_grid *grid, int32_t changed_axis);

/* CudaGrid::numElements (src/gpu/cudaGridSearch.cuh:89-98). */
cgs_status cgs_grid_num_elements(const cgs_grid *grid, uint64_t *num);

/* CudaGrid::getGridPoint (src/gpu/cudaGridSearch.cuh:189-196) -> gridPointProcess /
 * indexToGridPoint (:160-187, :274-279): host decode with the device's FP32 result. */
cgs_status cgs_grid_point(const cgs_grid *grid, int64_t index, float out[8]);

/* CudaGridSearcher::search / search_by_value / search_by_value_block / search_by_value_stream
 * / search_by_reference[_stream] (src/gpu/cudaGridSearch.cuh:553-556, 562-649, 653-732,
 * 736-765, 796-827, 831-853) followed by CudaTensor::find_extrema (include/cudaTensor.cuh:215-265)
 * and CudaGrid::getGridPoint: one fused sm_100a launch evaluates every grid point and
 * reduces the argmin.
 *   moving, fixed : device images (moving is sampled, fixed is iterated), as the reference's
 *                   functor arguments (img_moved, img_fixed).
 *   costs         : nullable DEVICE array of num_elements floats, costs[i] = cost of grid
 *                   index i (the reference's result tensor, axis 0 fastest).  The reference
 *                   kernel also writes costs[num_elements] (bound check '>' at
 *                   cudaGridSearch.cuh:295); this one does not.
 *   result        : DEVICE pointer to one cgs_argmin, written when the stream reaches it. */
cgs_status cgs_search(const cgs_image *moving, const cgs_image *fixed, const cgs_grid *grid,
                      const cgs_options *options, float *costs, cgs_argmin *result, cgs_stream_t stream);

/* CudaTensor<float, D>::find_extrema (include/cudaTensor.cuh:215-265 -> findExtremaProcess /
 * reduceMin6, include/cudaTensorKernels.cuh:133-220, 247-330): argmin of n device floats
 * with lowest-index ties.  result is a DEVICE pointer; params are left zero. */
cgs_status cgs_argmin_f32(const float *values, uint64_t n, cgs_argmin *result, cgs_stream_t stream);

/* cgs_search without any device allocation.  This entry point has no counterpart in the
 * reference; it exists for callers that cannot allocate device memory while they run: a
 * real-time or streaming loop that reserves its memory budget up front, where an allocation
 * may block on an implicit synchronisation or fail once a caching allocator (PyTorch's, for
 * one) holds nearly all free memory, or a host that owns device memory through its own pool.
 * Same arguments, results and status codes as cgs_search; the caller still provides the
 * images, the costs array and the result.  Differences:
 *   - scratch is a fixed 16 MiB array in the library's device image, held by every GPU that
 *     loads the library until the process exits.  Images whose staged copies do not fit
 *     (about 2 x 4 bytes x channels x width x height) are rejected with
 *     CGS_ERROR_INVALID_VALUE and a message giving both sizes;
 *   - the first call on a device looks up that array's device address (cudaGetSymbolAddress,
 *     with the device current); make that first call before any stream capture;
 *   - all calls on a device share the array, so calls that overlap on the GPU (on different
 *     streams, or from different host threads) race: serialise them;
 *   - points_per_warp / warps_per_block are ignored (4 points per warp, 16 warps; MI keeps its
 *     own shape);
 *   - it runs the pixel-loop costs (SAD_AVG, SAD_AVG_H, SAD_SUM_T, SAD_SUM_T_REF, SQD_REF,
 *     NCC_REF, ZNCC, MI) on 1- and 3-channel images; the scanline functors (SQD_ALT, NCC_ALT,
 *     MI_ALT) and other channel counts return CGS_ERROR_UNSUPPORTED;
 *   - the array's device address is kept from the first call on a device, so the entry point
 *     must not be used across a device reset (cudaDeviceReset). */
cgs_status cgs_search_noalloc(const cgs_image *moving, const cgs_image *fixed, const cgs_grid *grid,
                              const cgs_options *options, float *costs, cgs_argmin *result, cgs_stream_t stream);

/* CudaGridSearcher::covariance_by_value -> calculateCovariance_by_value
 * (src/gpu/cudaGridSearch.cuh:316-419, 768-794): curvature of the cost surface around the
 * grid minimum.  With f_min the lowest cost below zero (lowest index on ties; 0 at index 0
 * when no cost is negative) at grid point x_min, every other grid point x with cost f
 * (0 read as -1e-9) contributes g g^T, g = (x - x_min) s / |x - x_min|,
 * s = (log|f_min| - log|f|) / |x - x_min|, unless s < 0.
 *   costs : DEVICE array of the first n costs of the grid (n <= element count), as the
 *           cost tensor of cgs_search.
 *   covar : DEVICE array of dims x dims doubles, row-major, overwritten with the sum (the
 *           reference adds into a caller-initialised float matrix; the caller adds).
 * The terms are summed in double in a fixed order (deterministic). */
cgs_status cgs_covariance(const cgs_grid *grid, const float *costs, uint64_t n, double *covar, cgs_stream_t stream);

/* Joint histogram of the MI cost (CGS_COST_MI sampling: centred homography of params, the
 * calcNCC pixel loop) at one parameter vector: hist[bf * bins + bm] counts the (pixel, channel)
 * samples whose fixed value falls in bin bf and moving value in bin bm, bin = floor(v * bins / 256)
 * clamped.  hist is a DEVICE array of bins * bins uint32 (zeroed by the call).  The counts are
 * those the search kernel forms at that grid point; the reference forms its 64-bin counts the
 * same way in calcMIAlt (src/gpu/cudaErrorFunction_mi.cuh:189-195). */
cgs_status cgs_mi_histogram(const cgs_image *moving, const cgs_image *fixed, const float params[8], int32_t bins,
                            uint32_t *hist, cgs_stream_t stream);

/* Coarse-to-fine search, the loop of the reference's driver (src/gpu/cudaGridSearch_main_mi.cu:
 * 312-363): `depth` searches, each followed by re-centring every axis on the argmin's value p
 * with the reference's float arithmetic -- start' = p - (end - start) / 4, then
 * end' = p + (end - start') / 4 using the updated start -- the counts set again and the grid
 * updated as its setters do.  levels (host, nullable, depth entries) receives each level's
 * argmin; final_grid (host, nullable) the last level's grid.  A level without a finite cost
 * ends the loop (its argmin, valid = 0, fills the remaining entries).  Synchronous: every level
 * waits for the previous argmin. */
cgs_status cgs_search_refine(const cgs_image *moving, const cgs_image *fixed, const cgs_grid *grid,
                             const cgs_options *options, int32_t depth, cgs_argmin *levels, cgs_grid *final_grid,
                             cgs_stream_t stream);

/* ---------------------------------------------------------------- after the search
 *
 * parametersToHomography (src/gpu/cudaImageFunctions.cuh:216-252; centred = 1, centre (cx, cy),
 * normalised by h33) or the uncentred form inlined in averageAbsoluteDifference
 * (src/gpu/cudaErrorFunctions.cuh:42-57; centred = 0): H = {h11, h12, h13, h21, h22, h23, h31,
 * h32} of parameters [theta, sx, sy, shear, tx, ty, kx, ky], in the reference's float
 * operation order (host). */
cgs_status cgs_homography(const float params[8], float cx, float cy, int32_t centred, float H[8]);

/* transformImage (src/gpu/cudaImageFunctions.cuh:40-60), one thread per output pixel: for
 * every (x, y) in [0, cols) x [0, rows) the inverse map of H gives a point of `in`; where it
 * lies inside `in`, out(y, x, c) = in.valueAt_bilinear(point, c) converted to the pixel type,
 * elsewhere `out` keeps its value.  in and out are DEVICE images of one pixel type and channel
 * count; out is written (its data pointer is treated as writable).  The arithmetic is the
 * reference's device build (fused multiply-adds where nvcc forms them). */
cgs_status cgs_transform_image(const float H[8], int32_t rows, int32_t cols, const cgs_image *in, cgs_image *out,
                               cgs_stream_t stream);

/* fuseAlignedImages (src/gpu/cudaImageFunctions.cuh:62-112): the 3-channel overlay, channel 0
 * the moving image under estimated_H, 1 the reference image as it is, 2 the moving image under
 * true_H, each sampled at `channel` of its source; pixels that map outside keep their value.
 * fused is a DEVICE 3-channel image of the sources' pixel type (written). */
cgs_status cgs_fuse_aligned(const float estimated_H[8], const float true_H[8], const cgs_image *reference,
                            const cgs_image *moving, cgs_image *fused, int32_t channel, cgs_stream_t stream);

/* ---------------------------------------------------------------- before the search
 *
 * CudaImage::filter (include/cudaTensor.cuh:578-597 -> filterProcess, include/cudaTensorKernels.cuh:
 * 353-394): per pixel, channels whose action is 1 (FILTER) receive the correlation with `filter`
 * (a DEVICE single-channel float image, centred at ((h - 1) / 2, (w - 1) / 2)), taps outside
 * the image taking the centre pixel's value; channels whose action is 0 (COPY) are copied.  As
 * in the reference one running sum serves all FILTER channels of a pixel (it is not reset per
 * channel) and is converted to the pixel type.  actions: host array, one entry per channel.
 * in and out: DEVICE images of one shape and type (out is written). */
cgs_status cgs_filter_image(const cgs_image *filter, const cgs_image *in, cgs_image *out, const int32_t actions[],
                            cgs_stream_t stream);

/* Intensity quantisation of a uint8 image in place (transformPixel,
 * src/cpu/multispectral_ImageMatcher.cu:411-428): each sample read as a signed char v,
 * v = (int)(v / mod), v = (int)(v * mod), stored back modulo 256.  The reference's threads at
 * x == width or y == height (bound check '>') also rewrite the next row's first pixel or write
 * past the image; here every pixel is quantised exactly once. */
cgs_status cgs_quantize_image(cgs_image *img, float mod, cgs_stream_t stream);

/* ---------------------------------------------------------------- batched search
 *
 * Many image pairs of uneven sizes, each with its own grid and cost, evaluated by one recorded
 * launch sequence (a persistent kernel over the per-sample pairs, one multi-pair span kernel over
 * the ZNCC pairs).  The reference searches one pair per call and its callers loop
 * over pairs and refinement levels (src/gpu/cudaGridSearch_main_mi.cu:312-363, one
 * search_by_value + find_extrema per pass); a batch replaces that loop.  Each pair's costs and
 * argmin equal those of cgs_search on the same pair: bit for bit with block_split = 0, within
 * FP32 summation order with block_split = 1 (the argmin may then differ only between points
 * whose costs tie within that rounding). */
typedef struct cgs_pair {
    cgs_image moving;      /* DEVICE images, single channel                                  */
    cgs_image fixed;
    cgs_grid grid;
    cgs_options options;   /* cost: CGS_COST_SAD_AVG, _SQD_REF, _NCC_REF, _ZNCC or _MI; mi_bins,
                              overlap_gate and flags as for cgs_search.  points_per_warp and
                              warps_per_block are ignored: the batch plan applies.  Taps:
                              ZNCC pairs follow cgs_search's choice (quads on the fast
                              sampling path unless CGS_FLAG_TEXTURE_TAPS); the other costs
                              read texture gathers (MI: scalar loads), whatever the flags   */
    float *costs;          /* nullable DEVICE dump of this pair's grid (as cgs_search)       */
    cgs_argmin *result;    /* DEVICE result of this pair                                     */
} cgs_pair;

/* Launch plan of the batch kernel (one for the whole launch). */
typedef struct cgs_batch_plan {
    int32_t points_per_warp; /* 1, 2, 4 or 8 grid points evaluated together by a warp; MI pairs
                                take at most 2 (their per-warp histograms fill shared memory) */
    int32_t warps_per_block; /* 4, 8 or 16: blocks of 128, 256 or 512 threads                 */
    int32_t block_split;     /* 0: each warp owns its points and sweeps every pixel for them; MI
                                histograms are private per warp.  1: a block's warps share its
                                points and split the pixels; MI histograms are per block      */
    int32_t reserved;
} cgs_batch_plan;

/* One autotuner measurement: the plan, the kernel time on the tuning sample (+inf when the
 * plan does not fit), and the status of the attempt. */
typedef struct cgs_tune_entry {
    cgs_batch_plan plan;
    float ms;
    int32_t status;
} cgs_tune_entry;

typedef struct cgs_batch cgs_batch; /* opaque handle */

/* Creates a batch: validates every pair, lays out device scratch for all of them (one block
 * from the library's pool, held until cgs_batch_destroy), orders the pairs by estimated work
 * (cheapest first) and records one CUDA graph: clear scratch, stage every pair; the ZNCC pairs
 * that cgs_search runs on its span kernel (fast sampling, no per-sample flag) in one multi-pair
 * span launch, with cgs_search's costs and argmins bit for bit; the other pairs in the
 * persistent batch kernel, for the plan (NULL: 4 points per warp, 16 warps, warp-private
 * histograms; 2 points per warp, then block-shared histograms, where those do not fit); then,
 * pair after pair, cgs_search's own launches for MI pairs that it runs on its MI span kernel and
 * whose grids have at least 4 span tasks per SM (their results are cgs_search's, FP64
 * verification included).  The images, dumps and results are bound to the handle: update image
 * CONTENTS in place between launches.  Errors name the failing pair. */
cgs_status cgs_batch_create(const cgs_pair *pairs, int32_t n, const cgs_batch_plan *plan, cgs_batch **batch);

/* Replays the batch graph on `stream` (asynchronous).  Launches of one batch are serialised. */
cgs_status cgs_batch_launch(cgs_batch *batch, cgs_stream_t stream);

/* Sets the launch plan (re-records the graph) / reads it. */
cgs_status cgs_batch_set_plan(cgs_batch *batch, const cgs_batch_plan *plan);
cgs_status cgs_batch_get_plan(const cgs_batch *batch, cgs_batch_plan *plan);

/* Autotuner: times every plan (points_per_warp x warps_per_block x block_split, 24 candidates)
 * on a sample of the batch -- the first sample_points points of every pair's grid (<= 0: 4096),
 * the kernel alone, best of two runs after a warm-up -- and applies the fastest.  entries (up to
 * max_entries, nullable) receive every measurement. */
cgs_status cgs_batch_autotune(cgs_batch *batch, int32_t sample_points, cgs_tune_entry *entries, int32_t max_entries,
                              int32_t *n_entries, cgs_batch_plan *best);

/* Device time stamps (%globaltimer, ns) of the last launch, per pair in the caller's order: the
 * start of the pair's first task and the end of its last (pairs searched by span kernels: the
 * start and end of their own launches).  Waits for the launch. */
cgs_status cgs_batch_pair_times(cgs_batch *batch, uint64_t *start_ns, uint64_t *end_ns);

/* Kernel launches of one cgs_batch_launch (the kernel nodes of the recorded graph).  No
 * counterpart in the reference. */
cgs_status cgs_batch_kernel_launches(const cgs_batch *batch, int32_t *n);

/* Releases the handle's graph, textures and device memory (waits for its last launch). */
cgs_status cgs_batch_destroy(cgs_batch *batch);

/* One-shot batch: create, launch on `stream`, wait, destroy.  Synchronous. */
cgs_status cgs_search_batched(const cgs_pair *pairs, int32_t n, const cgs_batch_plan *plan, cgs_stream_t stream);

/* Autotunes a temporary batch of these pairs and returns the best plan. */
cgs_status cgs_autotune(const cgs_pair *pairs, int32_t n, int32_t sample_points, cgs_batch_plan *best);

/* ---------------------------------------------------------------- learned proposal network
 *
 * No counterpart in the reference.  A small CNN looks at an image pair and predicts where the
 * grid search's argmin lies: for each of the 8 parameters a centre c (grid-range units: -1 at
 * the grid's start, +1 at its end) and a log-radius s (the same units).  It is trained on pairs
 * whose labels are this library's own grid-search argmins, by this library's kernels (BF16
 * tensor-core implicit-GEMM convolutions with FP32 accumulation, FP32 MLP, Adam); the proposal
 * then narrows the grid (cgs_proposal_window, cgs_grid_window) and the full grid stays the fallback.
 *
 * Architecture: the pair box-averaged to 128 x 128 (fixed, moving as 2 channels), five 3x3
 * stride-2 convolutions with ReLU (32-64-128-128-256 channels), global average pool, dense
 * 256 -> 128 (ReLU) -> 16 (c[0..7], s[0..7]).  Loss: mean over samples and parameters of the
 * Laplace negative log-likelihood |c - y| e^-s + s, s clamped to [-6, 4]. */
typedef struct cgs_net cgs_net; /* opaque: parameters, Adam state, activations of one batch */

/* Number of FP32 parameters (the flat layout of get/set_params). */
int64_t cgs_net_param_count(void);

/* Allocates a network for batches of up to max_batch pairs, He-initialised from seed. */
cgs_status cgs_net_create(int32_t max_batch, uint64_t seed, cgs_net **net);
cgs_status cgs_net_destroy(cgs_net *net);

/* Copies of the flat FP32 parameters / the gradients of the last backward (host buffers of
 * cgs_net_param_count() floats).  Synchronising. */
cgs_status cgs_net_get_params(const cgs_net *net, float *host_params);
cgs_status cgs_net_set_params(cgs_net *net, const float *host_params);
cgs_status cgs_net_get_grads(const cgs_net *net, float *host_grads);

/* Forward pass on n pairs: fixed and moving are DEVICE stacks of n single-channel float images
 * of side x side pixels (side a multiple of 128; box-averaged to 128).  out (nullable) is a
 * DEVICE array of n x 16 floats.  Asynchronous on stream. */
cgs_status cgs_net_forward(cgs_net *net, const float *fixed, const float *moving, int32_t n, int32_t side, float *out,
                           cgs_stream_t stream);

/* Backward pass of the last forward: labels is a DEVICE array of n x 8 targets (grid-range
 * units); gradients land in the network; loss (nullable DEVICE float) receives the mean loss. */
cgs_status cgs_net_backward(cgs_net *net, const float *labels, float *loss, cgs_stream_t stream);

/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected) with learning rate lr. */
cgs_status cgs_net_adam_step(cgs_net *net, float lr, cgs_stream_t stream);

/* A window of a grid by index: on axis a the count[a] consecutive values from index first[a].
 * Its values are the grid's own (decoded as CudaGrid::indexToGridPoint does), so a search of
 * the window evaluates points of the grid.  `grid` needs integral counts. */
cgs_status cgs_grid_window(const cgs_grid *grid, const int32_t first[8], const int32_t count[8], cgs_grid *window);

/* The window a proposal implies on `full` (integral counts): per axis the values centred on the
 * value nearest the proposed centre c that hold every value within the radius e^s of c
 * (half-width floor(radius / resolution + 1/2)), widened to min_values or narrowed to
 * max_values (both odd) and shifted to stay inside the grid.  out is the network's 16 outputs
 * of the pair (host); first/count receive the window (axes past dims: 0 / 1). */
cgs_status cgs_proposal_window(const cgs_grid *full, const float out[16], int32_t min_values, int32_t max_values,
                               int32_t first[8], int32_t count[8]);

/* Synchronous convenience: cgs_search on `stream`, then copies the argmin to *host_result. */
cgs_status cgs_search_sync(const cgs_image *moving, const cgs_image *fixed, const cgs_grid *grid,
                           const cgs_options *options, float *costs, cgs_argmin *host_result,
                           cgs_stream_t stream);

/* Human-readable status, and the last error message recorded on the calling thread. */
const char *cgs_status_string(cgs_status status);
const char *cgs_last_error(void);

/* Library version (major * 10000 + minor * 100 + patch). */
int32_t cgs_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CUGRIDSEARCH_B200_H */
