/* Host definitions of the CUDA built-in index variables (TEST INFRASTRUCTURE).
 * averageAbsoluteDifference reads blockDim/blockIdx/threadIdx only to print a progress
 * line every 100000th grid index (src/gpu/cudaErrorFunctions.cuh:82-85); on the host
 * those symbols do not exist, so the harness defines them with a grid index of 1, which
 * never prints.  The functor's value does not depend on them. */
#include <vector_types.h>
extern const uint3 __device_builtin_variable_threadIdx;
const uint3 __device_builtin_variable_threadIdx = {1u, 0u, 0u};
extern const uint3 __device_builtin_variable_blockIdx;
const uint3 __device_builtin_variable_blockIdx = {0u, 0u, 0u};
extern const dim3 __device_builtin_variable_blockDim;
const dim3 __device_builtin_variable_blockDim(1u, 1u, 1u);
