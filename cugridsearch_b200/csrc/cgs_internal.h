// cgs_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "cgs_kernels.cuh"

namespace cgs {

// Host helpers of cgs_search.cu shared with the other C-ABI translation units.
cgs_status fail(cgs_status s, const std::string &msg);   // sets cgs_last_error()
cgs_status cuda_fail(cudaError_t e, const char *what);   // CUDA error -> status + message
cgs_status get_pool(int dev, cudaMemPool_t *out);        // the device's scratch pool

struct DeviceInfo {
    int dev = -1;
    int sms = 0;
    int major = 0;
    int tex_align = 512;
    int tex_pitch_align = 32;
};
cgs_status device_info(DeviceInfo *d);  // current device; fails unless sm_100

// CudaGrid's increments and element count (float count x int increment, truncated).
void grid_increments(const cgs_grid &g, int32_t inc[8], int64_t *num);
cgs_status check_grid(const cgs_grid *g);

// Staging-kernel parameters of one pair (prep_kernel / batch_prep_kernel).
struct PrepParams {
    const void *mov_src;
    const void *fix_src;
    int32_t mov_pix, fix_pix;
    int32_t mh, mw, fh, fw, c;
    float *mov_dst;
    float *fix_dst;
    int64_t mplane, fplane;
    int32_t mpitch, fpitch;
    unsigned long long *key;
    unsigned int *done;
    unsigned int *status;
    float *vmax;  // zeroed before the launch
    float *shifts;       // {fixed, moving} subsample means (ZNCC shifts), written by block 0, or null
    int32_t fix_alias;   // stage the fixed image like the moving one (scanline functors)
    float *row_table;    // calcMIAlt row values, or null
    int32_t rowsf;
    float4 *quad_dst;    // moving-image tap quads (W x H per channel), or null
    int64_t qplane;
    int32_t quad_form;   // 0: {P00, P10, P01 - P00, P11 - P10}; 1 (span kernel): {P00, P01 - P00, P10 - P00,
                         // (P11 - P10) - (P01 - P00)}, P(dy, dx) the tap at (y + dy, x + dx)
};

// Staged layout of a moving/fixed image pair inside one scratch block.
struct Staging {
    int32_t mpitch = 0, fpitch = 0;
    int64_t mplane = 0, fplane = 0;
    size_t mov_off = 0, fix_off = 0, rows_off = 0, quad_off = 0, bytes = 0;
    int64_t qplane = 0;  // quads per channel (0: no quad planes)
};

Staging staging_layout(const cgs_image &mov, const cgs_image &fix, int tex_align, int tex_pitch_align,
                       bool fix_alias = false, bool row_table = false, bool quads = false);
char *staging_origin(void *scratch, int tex_align);  // first tex_align boundary of a block
bool exact_samples(int cost, int flags);             // sampling mode of a request

// Request validation and kernel parameters shared by every pixel-loop entry point.
cgs_status check_request(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid, const cgs_options *options,
                         int *mi_bins);
cgs_status fill_params(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid, const cgs_options &o,
                       int mi_bins, SearchParams *p, int64_t *n64);
int64_t set_chunks(SearchParams *p, const Staging &st, int C, int fix_h);
PrepParams make_prep(const cgs_image *mov, const cgs_image *fix, const Staging &st, char *sb, float *mstage,
                     float *fstage);
size_t acc_bytes(int cost, int G, int NW, bool block_split, int mi_bins);
const void *batch_prep_kernel_fn();  // batch_prep_kernel(const PrepParams *), grid (x, pairs)

#define CGS_CUDA(call, what)                                    \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cgs::cuda_fail(e_, what); \
    } while (0)

// Kernel of a pixel-loop cost for (channels, points per warp, warps per CTA, quad taps), or null.
using KernelGetter = const void *(*)(int C, int G, int NW, bool quad);
const void *kernel_sad_avg(int C, int G, int NW, bool quad);
const void *kernel_sad_avg_h(int C, int G, int NW, bool quad);
const void *kernel_sad_sum_t(int C, int G, int NW, bool quad);
const void *kernel_sad_sum_t_ref(int C, int G, int NW, bool quad);
const void *kernel_sqd_ref(int C, int G, int NW, bool quad);
const void *kernel_ncc_ref(int C, int G, int NW, bool quad);
const void *kernel_zncc(int C, int G, int NW, bool quad);
const void *kernel_mi(int C, int G, int NW, bool quad);

// Scanline functors (calcSQDAlt, calcNCCAlt, calcMIAlt) and their shared-memory size.
const void *kernel_scan(int cost, int C);
size_t scan_smem_bytes(int cost);

// Span kernel of zero-mean NCC (cgs_span.cuh): G points per warp, NW warps, tiles of 32 TX
// columns; `check` selects the self-checking build.  Its shared-memory size, the largest quad
// plane it takes, and the launch of its own staging step (the fixed rows' FP64 prefix sums, the
// moving shift folded into the quads) after prep_kernel.
const void *kernel_span_zncc(int G, int NW, int TX, bool check);
size_t span_kernel_smem(int G, int NW, int TH, int TX, int tiles, int cap);
int64_t span_max_quads();
cudaError_t launch_span_prep(const float *fix, int fpitch, int fw, int fh, double2 *prefix, float4 *quads,
                             int64_t nquads, const float *shifts, cudaStream_t stream);
constexpr unsigned int kStatusSpanBounds = 0x100u;  // result status bit of the self-checking span build
constexpr int kMinSpanCap = 1024;                   // smallest useful window stage (quads)
struct SpanPlan {
    int G = 4, NW = 16, TX = 2, TH = 16;
    int tiles_x = 0, tiles_y = 0, cap = 0, pitch_mod = 0;
    bool check = false;
    size_t smem = 0;
    const void *kfn = nullptr;
};
bool span_plan(const cgs_image &mov, const cgs_image &fix, const cgs_options &o, SpanPlan *sp);
// The multi-pair span kernel of batches for a plan (null where not instantiated), and the
// staging step of many pairs: per pair its arguments and block count, then one launch over all.
const void *kernel_span_zncc_batch(int G, int NW, int TX, bool check);
void span_prep_batch_args(const float *fix, int fpitch, int fw, int fh, double2 *prefix, float4 *quads,
                          int64_t nquads, const float *shifts, SpanPrepArgs *a, int *blocks);
cudaError_t launch_span_prep_batch(const SpanPrepArgs *args, int n, int blocks, cudaStream_t stream);
// Span kernel of MI (cgs_span_mi.cuh): 2 points per warp, NW warps, histograms of B <= 32 bins;
// its shared-memory size and its staging step (the fixed bins times B + 1, int32; the quads'
// largest slope bound into a header word).
const void *kernel_span_mi(int NW, bool check);
size_t span_mi_kernel_smem(int NW, int TH, int B);
cudaError_t launch_span_prep_mi(const float *fix, int fpitch, int fw, int fh, int B, int32_t *bins,
                                const float4 *quads, int64_t nquads, unsigned int *lmax, cudaStream_t stream);
bool span_mi_plan(const cgs_image &mov, const cgs_image &fix, const cgs_options &o, int mi_bins, SpanPlan *sp);

// FP64 verification pass (cgs_verify.cu): band collection and re-scoring after a search whose
// costs are in p.costs and result in p.result; hdr is zeroed device scratch.
constexpr int kVerifyMax = CGS_VERIFY_MAX;
size_t verify_scratch_bytes();
cgs_status launch_verify(const SearchParams &p, void *hdr, cudaStream_t stream, int sms);
bool verify_supported(int cost);

// A search in a caller's scratch block (cgs_search.cu): for requests that cgs_search runs on a
// span kernel (ZNCC or MI on the fast sampling path), the batch runs them with the same launches
// and results.  span_route_bytes: whether cgs_search runs this pair on a span kernel, the
// scratch it then needs (staging, span tables, verification header) and the kernel's grid
// points per task; span_route_enqueue: the search's launches on `stream` with that scratch
// (tex_align-aligned, `bytes` long).
struct ExtScratch {
    char *ptr = nullptr;
    size_t bytes = 0;
    bool query = false;
    uint32_t points_per_task = 0;  // query: the span kernel's grid points per task
};
bool span_route_bytes(const cgs_pair &q, size_t *bytes, uint32_t *points_per_task);
cgs_status span_route_enqueue(const cgs_pair &q, char *scratch, size_t bytes, cudaStream_t stream);

// Plain-load (no texture object) variants at 4 points per warp and 16 warps, for the
// allocation-free entry point.
const void *kernel_sad_avg_loads(int C);
const void *kernel_sad_avg_h_loads(int C);
const void *kernel_sad_sum_t_loads(int C);
const void *kernel_sad_sum_t_ref_loads(int C);
const void *kernel_sqd_ref_loads(int C);
const void *kernel_ncc_ref_loads(int C);
const void *kernel_zncc_loads(int C);

}  // namespace cgs

// Instantiates search_kernel<COST, C, G, NW, taps> for C in {1, 3}, G in {1, 2, 4}, NW in
// {8, 16}, with the cost's default taps or quad taps.
#define CGS_KERNEL_CASES(COST, C, NWV, TP)                                                    \
    if (G == 1) return (const void *)search_kernel<COST, C, 1, NWV, TP>;                      \
    if (G == 2) return (const void *)search_kernel<COST, C, 2, NWV, TP>;                      \
    if (G == 4) return (const void *)search_kernel<COST, C, 4, NWV, TP>;
#define CGS_KERNEL_SHAPES(COST, TP)                                                            \
    if (C == 1 && NW == 16) { CGS_KERNEL_CASES(COST, 1, 16, TP) }                             \
    if (C == 3 && NW == 16) { CGS_KERNEL_CASES(COST, 3, 16, TP) }                             \
    if (C == 1 && NW == 8) { CGS_KERNEL_CASES(COST, 1, 8, TP) }                               \
    if (C == 3 && NW == 8) { CGS_KERNEL_CASES(COST, 3, 8, TP) }
#define CGS_DEFINE_KERNEL_GETTER(NAME, COST)                                                   \
    namespace cgs {                                                                           \
    const void *NAME(int C, int G, int NW, bool quad) {                                       \
        if (quad) { CGS_KERNEL_SHAPES(COST, kTapsQuad) }                                      \
        else { CGS_KERNEL_SHAPES(COST, default_taps(COST)) }                                  \
        return nullptr;                                                                       \
    }                                                                                         \
    }

#define CGS_DEFINE_LOADS_GETTER(NAME, COST)                                                    \
    namespace cgs {                                                                           \
    const void *NAME(int C) {                                                                 \
        if (C == 1) return (const void *)search_kernel<COST, 1, 4, 16, kTapsLoads>;           \
        if (C == 3) return (const void *)search_kernel<COST, 3, 4, 16, kTapsLoads>;           \
        return nullptr;                                                                       \
    }                                                                                         \
    }
