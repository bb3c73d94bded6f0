// Kernel instantiations for CGS_COST_MI (one translation unit per cost, compiled in parallel).
#include "cgs_internal.h"
CGS_DEFINE_KERNEL_GETTER(kernel_mi, CGS_COST_MI)
