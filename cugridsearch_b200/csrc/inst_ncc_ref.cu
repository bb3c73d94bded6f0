// Kernel instantiations for CGS_COST_NCC_REF (one translation unit per cost, compiled in parallel).
#include "cgs_internal.h"
CGS_DEFINE_KERNEL_GETTER(kernel_ncc_ref, CGS_COST_NCC_REF)
CGS_DEFINE_LOADS_GETTER(kernel_ncc_ref_loads, CGS_COST_NCC_REF)
