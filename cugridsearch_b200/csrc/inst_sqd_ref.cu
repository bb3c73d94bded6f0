// Kernel instantiations for CGS_COST_SQD_REF (one translation unit per cost, compiled in parallel).
#include "cgs_internal.h"
CGS_DEFINE_KERNEL_GETTER(kernel_sqd_ref, CGS_COST_SQD_REF)
CGS_DEFINE_LOADS_GETTER(kernel_sqd_ref_loads, CGS_COST_SQD_REF)
