/*
 * cgsCompat.cuh -- error handling and small device helpers shared by the drop-in template
 * headers (cudaTensor.cuh, cudaGridSearch.cuh).
 *
 * The reference prints and calls exit() on any CUDA error (src/gpu/cudaGridSearch.cuh:51-56,
 * gpuAssert).  The drop-in headers throw cgs_compat::Error instead, carrying the library's
 * status code and message; define CGS_COMPAT_EXIT before including them to get the
 * reference's print-and-exit behaviour.  Define CGS_COMPAT_VERBOSE to get the reference's
 * progress lines ("CudaGrid has N search samples.", "Time Taken: ...", the find_extrema
 * summary) on stdout.
 */
#ifndef CUGRIDSEARCH_CGSCOMPAT_CUH
#define CUGRIDSEARCH_CGSCOMPAT_CUH

#ifndef CUDAFUNCTION
#define CUDAFUNCTION __host__ __device__
#endif

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "../cugridsearch_b200.h"

namespace cgs_compat {

struct Error : std::runtime_error {
    cgs_status status;
    Error(const std::string &what, cgs_status st) : std::runtime_error(what), status(st) {}
};

inline void fail(const std::string &what, cgs_status st) {
#ifdef CGS_COMPAT_EXIT
    fprintf(stderr, "GPUassert: %s\n", what.c_str());
    exit((int)st);
#else
    throw Error(what, st);
#endif
}

// A library call's status; the message is the library's own (cgs_last_error).
inline void check(cgs_status st, const char *where) {
    if (st != CGS_SUCCESS) fail(std::string(where) + ": " + cgs_last_error(), st);
}

inline void check_cuda(cudaError_t e, const char *where) {
    if (e != cudaSuccess) fail(std::string(where) + ": " + cudaGetErrorString(e), CGS_ERROR_CUDA);
}

// Launch status of the kernel just enqueued plus completion of the default stream: the
// template wrappers are blocking, as the reference's are (cudaDeviceSynchronize after each
// launch, cudaGridSearch.cuh:759-761).
inline void check_launch(const char *where) {
    check_cuda(cudaPeekAtLastError(), where);
    check_cuda(cudaDeviceSynchronize(), where);
}

// Grid-stride launch shape for element-wise helpers: a few waves over the SMs.
inline void launch_shape(uint64_t n, unsigned &blocks, unsigned &threads) {
    threads = 256;
    const uint64_t want = (n + threads - 1) / threads;
    blocks = (unsigned)(want < 148u * 8u ? (want > 0 ? want : 1) : 148u * 8u);
}

}  // namespace cgs_compat

#endif  // CUGRIDSEARCH_CGSCOMPAT_CUH
