// Kernel instantiations of the scanline functors calcSQDAlt, calcNCCAlt and calcMIAlt.
#include "cgs_internal.h"
#include "cgs_scan.cuh"

namespace cgs {

const void *kernel_scan(int cost, int C) {
    if (C == 1) {
        if (cost == CGS_COST_SQD_ALT) return (const void *)scan_kernel<CGS_COST_SQD_ALT, 1, kScanWarps>;
        if (cost == CGS_COST_NCC_ALT) return (const void *)scan_kernel<CGS_COST_NCC_ALT, 1, kScanWarps>;
        if (cost == CGS_COST_MI_ALT) return (const void *)scan_kernel<CGS_COST_MI_ALT, 1, kScanWarps>;
    } else if (C == 3) {
        if (cost == CGS_COST_SQD_ALT) return (const void *)scan_kernel<CGS_COST_SQD_ALT, 3, kScanWarps>;
        if (cost == CGS_COST_NCC_ALT) return (const void *)scan_kernel<CGS_COST_NCC_ALT, 3, kScanWarps>;
        if (cost == CGS_COST_MI_ALT) return (const void *)scan_kernel<CGS_COST_MI_ALT, 3, kScanWarps>;
    }
    return nullptr;
}

size_t scan_smem_bytes(int cost) {
    size_t b = 8 * kScanWarps + (size_t)kScanWarps * kScanRows * (sizeof(RowInfo) + kMaxSegs * sizeof(Seg));
    if (cost == CGS_COST_MI_ALT) b += (size_t)kScanWarps * 65 * 65 * 4;
    return b;
}

}  // namespace cgs
