// MI span-kernel instantiations (one channel, 16 warps of 2 points, plain and self-checking) and
// its staging step.
#include <algorithm>

#include "cgs_internal.h"
#include "cgs_span_mi.cuh"

namespace cgs {

const void *kernel_span_mi(int NW, bool check) {
    if (NW != 16) return nullptr;
    return check ? (const void *)span_mi_kernel<16, true> : (const void *)span_mi_kernel<16, false>;
}

size_t span_mi_kernel_smem(int NW, int TH, int B) { return span_mi_smem_bytes(NW, TH, B); }

cudaError_t launch_span_prep_mi(const float *fix, int fpitch, int fw, int fh, int B, int32_t *bins,
                                const float4 *quads, int64_t nquads, unsigned int *lmax, cudaStream_t stream) {
    const int blocks = (int)std::min<int64_t>((std::max<int64_t>((int64_t)fh * fpitch, nquads) + 255) / 256, 1024);
    span_prep_mi_kernel<<<blocks, 256, 0, stream>>>(fix, fpitch, fw, fh, B, bins, quads, nquads, lmax);
    return cudaGetLastError();
}

}  // namespace cgs
