// Kernel instantiations for CGS_COST_SAD_AVG_H (one translation unit per cost, compiled in parallel).
#include "cgs_internal.h"
CGS_DEFINE_KERNEL_GETTER(kernel_sad_avg_h, CGS_COST_SAD_AVG_H)
CGS_DEFINE_LOADS_GETTER(kernel_sad_avg_h_loads, CGS_COST_SAD_AVG_H)
