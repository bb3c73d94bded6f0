// cgs_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include "cgs_kernels.cuh"

namespace cgs {

// Kernel of a pixel-loop cost for (channels, points per warp, warps per CTA), or null.
using KernelGetter = const void *(*)(int C, int G, int NW);
const void *kernel_sad_avg(int C, int G, int NW);
const void *kernel_sad_avg_h(int C, int G, int NW);
const void *kernel_sad_sum_t(int C, int G, int NW);
const void *kernel_sad_sum_t_ref(int C, int G, int NW);
const void *kernel_sqd_ref(int C, int G, int NW);
const void *kernel_ncc_ref(int C, int G, int NW);
const void *kernel_zncc(int C, int G, int NW);
const void *kernel_mi(int C, int G, int NW);

}  // namespace cgs

// Instantiates search_kernel<COST, C, G, NW> for C in {1, 3}, G in {1, 2, 4}.
#define CGS_DEFINE_KERNEL_GETTER(NAME, COST, NWV)                                              \
    namespace cgs {                                                                           \
    const void *NAME(int C, int G, int NW) {                                                  \
        if (NW != NWV) return nullptr;                                                        \
        if (C == 1) {                                                                         \
            if (G == 1) return (const void *)search_kernel<COST, 1, 1, NWV>;                  \
            if (G == 2) return (const void *)search_kernel<COST, 1, 2, NWV>;                  \
            if (G == 4) return (const void *)search_kernel<COST, 1, 4, NWV>;                  \
        } else if (C == 3) {                                                                  \
            if (G == 1) return (const void *)search_kernel<COST, 3, 1, NWV>;                  \
            if (G == 2) return (const void *)search_kernel<COST, 3, 2, NWV>;                  \
            if (G == 4) return (const void *)search_kernel<COST, 3, 4, NWV>;                  \
        }                                                                                     \
        return nullptr;                                                                       \
    }                                                                                         \
    }
