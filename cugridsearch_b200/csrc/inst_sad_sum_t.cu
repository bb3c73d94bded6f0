// Kernel instantiations for CGS_COST_SAD_SUM_T (one translation unit per cost, compiled in parallel).
#include "cgs_internal.h"
CGS_DEFINE_KERNEL_GETTER(kernel_sad_sum_t, CGS_COST_SAD_SUM_T)
CGS_DEFINE_LOADS_GETTER(kernel_sad_sum_t_loads, CGS_COST_SAD_SUM_T)
