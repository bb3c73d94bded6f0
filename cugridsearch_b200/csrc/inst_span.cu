// Span-kernel instantiations (zero-mean NCC, one channel), 16 warps per CTA: 4 points per warp
// with tiles of 64, 128 or 256 columns, 2 points per warp with 128 or 256; plain and self-checking;
// and the fixed rows' prefix sums.
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

cudaError_t launch_span_prep(const float *fix, int fpitch, int fw, int fh, double2 *prefix, float4 *quads,
                             int64_t nquads, const float *shifts, cudaStream_t stream) {
    const int row_blocks = (int)(((int64_t)fh * 32 + 255) / 256);
    const int quad_blocks = (int)std::min<int64_t>((nquads + 255) / 256, 1024);
    span_prep_kernel<<<row_blocks + quad_blocks, 256, 0, stream>>>(fix, fpitch, fw, fh, prefix, row_blocks, quads,
                                                                   nquads, shifts);
    return cudaGetLastError();
}

}  // namespace cgs
