// Batch-kernel instantiations with 4 grid point(s) per warp (one translation unit per
// points-per-warp value, compiled in parallel).
#include "cgs_batch.cuh"
CGS_DEFINE_BATCH_GETTER(batch_kernel_g4, 4)
