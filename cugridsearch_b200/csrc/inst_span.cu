// Span-kernel instantiations (zero-mean NCC, one channel), 16 warps per CTA: 4 points per warp
// with tiles of 32, 64 or 128 columns, 2 points per warp with 64 or 128; plain and self-checking.
#include "cgs_internal.h"
#include "cgs_span.cuh"

namespace cgs {

template <int G, bool CHECK>
static const void *span16(int TX) {
    if constexpr (G == 4) {
        if (TX == 1) return (const void *)span_kernel<G, 16, 1, CHECK>;
    }
    if (TX == 2) return (const void *)span_kernel<G, 16, 2, CHECK>;
    if (TX == 4) return (const void *)span_kernel<G, 16, 4, CHECK>;
    return nullptr;
}

const void *kernel_span_zncc(int G, int NW, int TX, bool check) {
    if (NW != 16) return nullptr;
    if (G == 4) return check ? span16<4, true>(TX) : span16<4, false>(TX);
    if (G == 2) return check ? span16<2, true>(TX) : span16<2, false>(TX);
    return nullptr;
}

size_t span_kernel_smem(int G, int NW, int TH, int tiles, int cap) { return span_smem_bytes(G, NW, TH, tiles, cap); }

}  // namespace cgs
