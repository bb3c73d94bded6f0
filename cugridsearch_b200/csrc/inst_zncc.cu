// Kernel instantiations for CGS_COST_ZNCC (one translation unit per cost, compiled in parallel).
#include "cgs_internal.h"
CGS_DEFINE_KERNEL_GETTER(kernel_zncc, CGS_COST_ZNCC)
CGS_DEFINE_LOADS_GETTER(kernel_zncc_loads, CGS_COST_ZNCC)
