// Span-kernel instantiations (zero-mean NCC, one channel), 16 warps per CTA: 4 points per warp
// with tiles of 64, 128 or 256 columns, 2 points per warp with 128 or 256; plain and self-checking;
// the multi-pair kernel of batches (4 points per warp, tiles of 256 columns); and the fixed rows'
// prefix sums.
#include <algorithm>

#include "cgs_internal.h"
#include "cgs_span.cuh"

namespace cgs {

template <int G, bool CHECK>
static const void *span16(int TX) {
    if constexpr (G == 4) {
        if (TX == 2) return (const void *)span_kernel<G, 16, 2, CHECK>;
        if (TX == 8) return (const void *)span_kernel<G, 16, 8, CHECK>;
    }
    if (TX == 4) return (const void *)span_kernel<G, 16, 4, CHECK>;
    if constexpr (G == 2) {
        if (TX == 8) return (const void *)span_kernel<G, 16, 8, CHECK>;
    }
    return nullptr;
}

const void *kernel_span_zncc(int G, int NW, int TX, bool check) {
    if (NW != 16) return nullptr;
    if (G == 4) return check ? span16<4, true>(TX) : span16<4, false>(TX);
    if (G == 2) return check ? span16<2, true>(TX) : span16<2, false>(TX);
    return nullptr;
}

size_t span_kernel_smem(int G, int NW, int TH, int TX, int tiles, int cap) {
    return span_smem_bytes(G, NW, TH, TX, tiles, cap);
}

int64_t span_max_quads() { return kSpanMaxQuads; }

static int span_prep_row_blocks(int fh) { return (int)(((int64_t)fh * 32 + 255) / 256); }
static int span_prep_quad_blocks(int64_t nquads) { return (int)std::min<int64_t>((nquads + 255) / 256, 1024); }

cudaError_t launch_span_prep(const float *fix, int fpitch, int fw, int fh, double2 *prefix, float4 *quads,
                             int64_t nquads, const float *shifts, cudaStream_t stream) {
    const SpanPrepArgs a{fix, fpitch, fw, fh, prefix, span_prep_row_blocks(fh), quads, nquads, shifts};
    span_prep_kernel<<<a.row_blocks + span_prep_quad_blocks(nquads), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

const void *kernel_span_zncc_batch(int G, int NW, int TX, bool check) {
    if (G == 4 && NW == 16 && TX == 8 && !check) return (const void *)span_batch_kernel<4, 16, 8, false>;
    return nullptr;
}

void span_prep_batch_args(const float *fix, int fpitch, int fw, int fh, double2 *prefix, float4 *quads,
                          int64_t nquads, const float *shifts, SpanPrepArgs *a, int *blocks) {
    *a = SpanPrepArgs{fix, fpitch, fw, fh, prefix, span_prep_row_blocks(fh), quads, nquads, shifts};
    *blocks = a->row_blocks + span_prep_quad_blocks(nquads);
}

cudaError_t launch_span_prep_batch(const SpanPrepArgs *args, int n, int blocks, cudaStream_t stream) {
    span_prep_batch_kernel<<<dim3(blocks, n), 256, 0, stream>>>(args);
    return cudaGetLastError();
}

}  // namespace cgs
