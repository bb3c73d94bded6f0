/*
 * cgs_oracle.h -- CPU oracle for the homography grid search (TEST INFRASTRUCTURE).
 *
 * This library is the checker, never the product: only tests/, the smoke()
 * entry point and the CPU-baseline leg of bench.py load it.  It restates the
 * reference cost functors of uncc-visionlab/cuGridSearch in plain C with the
 * reference's FP32 operation order (compiled with -ffp-contract=off so no
 * multiply-add is fused), and adds FP64-accumulation variants that sample the
 * images exactly as the FP32 code does but sum in double.  Every function cites
 * the reference file:line it restates.  Parity of the restatement is pinned by
 * bit-exact comparison against the reference's own functor source compiled for
 * the host (oracle/ref_harness.cu -> oracle/_ref/libcgs_ref.so).
 */
#ifndef CGS_ORACLE_H
#define CGS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Cost identifiers; the product C-ABI uses the same numbering. */
enum {
    OG_SAD_AVG = 0,      /* averageAbsoluteDifference   src/gpu/cudaErrorFunctions.cuh:31-87   */
    OG_SAD_AVG_H = 1,    /* averageAbsoluteDifferenceH  src/gpu/cudaErrorFunctions.cuh:194-224 */
    OG_SAD_SUM_T = 2,    /* sumOfAbsoluteDifferences (by value)      cudaErrorFunctions.cuh:89-114  */
    OG_SAD_SUM_T_REF = 3,/* sumOfAbsoluteDifferences (by reference)  cudaErrorFunctions.cuh:171-192 */
    OG_SQD_REF = 4,      /* calcSQD     cudaErrorFunctions.cuh:378-446 */
    OG_NCC_REF = 5,      /* calcNCC     cudaErrorFunctions.cuh:448-507 */
    OG_SQD_ALT = 6,      /* calcSQDAlt  cudaErrorFunctions.cuh:226-300 */
    OG_NCC_ALT = 7,      /* calcNCCAlt  cudaErrorFunctions.cuh:302-376 */
    OG_MI_ALT = 8,       /* calcMIAlt   cudaErrorFunction_mi.cuh:117-255 (64 bins) */
    OG_ZNCC = 9,         /* zero-mean NCC over the calcNCC sampling (no reference counterpart) */
    OG_MI = 10,          /* MI from exact integer B x B counts over the calcNCC sampling */
    OG_NUM_COSTS = 11
};

enum { OG_PIX_F32 = 0, OG_PIX_U8 = 1, OG_PIX_F64 = 2, OG_PIX_U16 = 3 };

typedef struct {
    const void *data;   /* host pointer, HWC row-major (CudaImage layout, cudaTensor.cuh:512-534) */
    int32_t height, width, channels;
    int32_t pix;        /* OG_PIX_* */
} og_image;

/* Options for the costs that have no reference counterpart. */
typedef struct {
    int32_t mi_bins;        /* MI: power of two in [2, 256] */
    float overlap_gate;     /* ZNCC/MI: minimum overlap fraction of the fixed image, else +inf */
} og_opts;

/* Grid descriptor: the 4 x D matrix of CudaGrid (cudaGridSearch.cuh:74-79). */
typedef struct {
    int32_t dims;
    float start[8], end[8], resolution[8], count[8];
} og_grid;

/* Reference CudaGrid::update() semantics (cudaGridSearch.cuh:235-272), on host. */
void og_grid_update(og_grid *g, int changed_axis);
/* Dimensional increments / element count exactly as indexToGridPoint and numElements
 * compute them (float products truncated to int32; cudaGridSearch.cuh:89-98,168-172). */
void og_grid_increments(const og_grid *g, int32_t inc[8]);
int64_t og_grid_num_elements(const og_grid *g);
/* indexToGridPoint (cudaGridSearch.cuh:160-187). use_fma selects fmaf(i,res,start)
 * (nvcc's contraction of start + i*res) or a separate multiply and add. */
void og_grid_point(const og_grid *g, int64_t index, int use_fma, float out[8]);

/* One cost at one parameter vector.  The FP32 variant mirrors the reference's
 * arithmetic; the FP64 variant samples identically and accumulates in double.
 * n_out (nullable) receives the number of contributing (pixel, channel) terms. */
float og_cost_f32(int cost, const float *params, const og_image *mov, const og_image *fix,
                  const og_opts *opts, int64_t *n_out);
double og_cost_f64(int cost, const float *params, const og_image *mov, const og_image *fix,
                   const og_opts *opts, int64_t *n_out);

/* Joint histogram (bins x bins, row = fixed bin, column = moving bin) of MI or MI_ALT
 * at one parameter vector; returns the number of counted terms. */
int64_t og_histogram(int cost, const float *params, const og_image *mov, const og_image *fix,
                     const og_opts *opts, uint32_t *hist);

/* Homography helpers (exposed for bit-exact tests of the restatement). */
void og_params_to_h(const float *params, float cx, float cy, float h[8]);       /* cudaImageFunctions.cuh:216-252 */
void og_params_to_h_uncentred(const float *params, float h[8]);                 /* cudaErrorFunctions.cuh:42-57 */
void og_params_to_h_norm(const float *params, int mw, int mh, int fw, int fh, float h[8]); /* :181-214 */
void og_new_coord(const float h[8], int x, int y, float *nx, float *ny);        /* :277-285 */
void og_bilinear_probe(const og_image *img, float y, float x, int c, float *out); /* cudaTensor.cuh:561-575 */

/* Grid search on the CPU: every grid index in [first, first + count) with the given
 * stride.  costs32/costs64 are nullable.  Returns 0 on success.  threads <= 0 means
 * all OpenMP threads. */
int og_search(int cost, const og_grid *g, int use_fma, const og_image *mov, const og_image *fix,
              const og_opts *opts, int64_t first, int64_t count, int64_t stride,
              float *costs32, double *costs64, int threads);

/* calculateCovariance_by_value (src/gpu/cudaGridSearch.cuh:316-419) over the first n costs
 * of grid g: f_min = lowest cost below zero (strict '<' from 0 at index 0), then for every
 * other index the term g g^T with the reference's per-term float operations as its device
 * build evaluates them (fused |x - x_min|^2).  out_f64 (nullable): terms summed in double;
 * out_ref (nullable): summed sequentially in float with fused multiply-adds, the
 * reference's own accumulation.  Both dims x dims row-major, overwritten. */
void og_covariance(const og_grid *g, const float *costs, int64_t n, double *out_f64, float *out_ref);

#ifdef __cplusplus
}
#endif
#endif
