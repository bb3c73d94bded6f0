// cgs_covariance.cu -- the curvature estimate around the grid minimum of a cost tensor
// (CudaGridSearcher::covariance_by_value -> calculateCovariance_by_value,
// src/gpu/cudaGridSearch.cuh:316-419 and 768-794), as two stream-ordered kernels.
//
// The reference runs it in ONE device thread: it scans the cost tensor for the lowest
// value below zero (its running minimum starts at 0, index 0), decodes that grid point
// x_min, and for every other grid point x with cost f (f = 0 read as -1e-9) forms
//   slope = (log|f_min| - log|f|) / |x - x_min|      (skipped when negative)
//   g     = (x - x_min) * slope / |x - x_min|
// and adds g g^T into a D x D matrix.  Here kernel 1 finds the minimum with the same
// strict '<' and lowest-index rule (orderable 64-bit keys), kernel 2 evaluates every term
// in parallel with the reference's per-term float operations -- including the multiply-add
// its device build fuses in |x - x_min|^2 -- and sums the exact double products g_r g_c in
// a fixed order (per-block partials, then the last block adds the blocks in order), so the
// result is deterministic and closer to the exact sum than the reference's sequential
// float accumulation.
#include <algorithm>
#include <cmath>

#include "cgs_internal.h"

namespace cgs {

namespace {

constexpr int kCovThreads = 256;

struct CovParams {
    int dims;
    float start[8], res[8];
    int32_t inc[8];
    const float *costs;
    uint32_t n;
    unsigned long long *key;  // minimum key (preset to all ones)
    unsigned int *ticket;     // last-block ticket (preset to all ones)
    double *partial;          // [blocks][D * D]
    double *out;              // D * D
};

// Grid point of index i: the reference's integer decode, start + i * res fused.
__device__ __forceinline__ void decode(const CovParams &p, uint32_t i, float *x) {
    int32_t rem = (int32_t)i;
#pragma unroll
    for (int a = 7; a >= 0; a--) {
        if (a < p.dims) {
            const int32_t k = rem / p.inc[a];
            rem -= k * p.inc[a];
            x[a] = __fmaf_rn((float)k, p.res[a], p.start[a]);
        } else {
            x[a] = 0.0f;
        }
    }
}

// Lowest cost strictly below zero, lowest index among equals.
__global__ void __launch_bounds__(kCovThreads) cov_min_kernel(const CovParams p) {
    __shared__ unsigned long long wk[kCovThreads / 32];
    unsigned long long best = ~0ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        const float v = __ldg(p.costs + i);
        if (v < 0.0f) {
            const unsigned long long k = make_key(v, i);
            best = k < best ? k : best;
        }
    }
    best = warp_min_u64(best);
    if ((threadIdx.x & 31) == 0) wk[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kCovThreads / 32; w++) best = wk[w] < best ? wk[w] : best;
        if (best != ~0ull) atomicMin(p.key, best);
    }
}

template <int D>
__global__ void __launch_bounds__(kCovThreads) cov_sum_kernel(const CovParams p) {
    constexpr int NT = D * (D + 1) / 2;  // upper triangle
    __shared__ double red[kCovThreads / 32][NT];
    __shared__ bool last;

    // the minimum: none below zero leaves the reference's start value (0 at index 0)
    const unsigned long long k = *p.key;
    const bool have = k != ~0ull;
    const uint32_t imin = have ? (uint32_t)(k & 0xffffffffu) : 0u;
    const float fmin = have ? key_cost(k) : 0.0f;
    float xm[8];
    decode(p, imin, xm);
    const float lmin = logf(fabsf(fmin));

    double acc[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) acc[t] = 0.0;

    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        if (i == imin) continue;
        float x[8];
        decode(p, i, x);
        float f = __ldg(p.costs + i);
        if (f == 0.0f) f = -1e-9f;
        float d[D];
        float len = 0.0f;
#pragma unroll
        for (int a = 0; a < D; a++) {
            d[a] = __fsub_rn(x[a], xm[a]);
            len = __fmaf_rn(d[a], d[a], len);
        }
        len = __fsqrt_rn(len);
        const float slope = __fmul_rn(__fsub_rn(lmin, logf(fabsf(f))), __fdiv_rn(1.0f, len));
        if (slope < 0.0f) continue;
        float g[D];
#pragma unroll
        for (int a = 0; a < D; a++) g[a] = __fdiv_rn(__fmul_rn(d[a], slope), len);
        int t = 0;
#pragma unroll
        for (int r = 0; r < D; r++)
#pragma unroll
            for (int c = r; c < D; c++) acc[t++] += (double)g[r] * (double)g[c];
    }

    // block sum in a fixed order: warps by shuffles, then warp 0 over the warps
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < NT; t++) {
        double v = acc[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][t] = v;
    }
    __syncthreads();
    if (threadIdx.x < NT) {
        double v = 0.0;
        for (int w = 0; w < kCovThreads / 32; w++) v += red[w][threadIdx.x];
        p.partial[(size_t)blockIdx.x * NT + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(p.ticket, 1u) + 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < NT) {
        double v = 0.0;
        for (uint32_t b = 0; b < gridDim.x; b++) v += __ldcg(p.partial + (size_t)b * NT + threadIdx.x);
        // upper-triangle slot t -> (r, c); write both halves of the symmetric matrix
        int t = threadIdx.x, r = 0;
        while (t >= D - r) {
            t -= D - r;
            r++;
        }
        const int c = r + t;
        p.out[r * D + c] = v;
        p.out[c * D + r] = v;
    }
}

template <int D>
void launch_sum(int blocks, cudaStream_t s, const CovParams &p) {
    cov_sum_kernel<D><<<blocks, kCovThreads, 0, s>>>(p);
}

}  // namespace

}  // namespace cgs

extern "C" {

cgs_status cgs_covariance(const cgs_grid *grid, const float *costs, uint64_t n, double *covar,
                          cgs_stream_t stream_) {
    using namespace cgs;
    cudaStream_t stream = (cudaStream_t)stream_;
    cgs_status s;
    if ((s = check_grid(grid)) != CGS_SUCCESS) return s;
    if (!covar) return fail(CGS_ERROR_INVALID_VALUE, "covar is null");
    int32_t inc[8];
    int64_t num;
    grid_increments(*grid, inc, &num);
    if (n > (uint64_t)(num < 0 ? 0 : num)) return fail(CGS_ERROR_INVALID_VALUE, "n exceeds the grid's element count");
    if (n > 0 && !costs) return fail(CGS_ERROR_INVALID_VALUE, "costs is null");
    DeviceInfo di;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;
    const int D = grid->dims;
    CGS_CUDA(cudaMemsetAsync(covar, 0, sizeof(double) * D * D, stream), "cudaMemsetAsync");
    if (n == 0) return CGS_SUCCESS;
    const int nt = D * (D + 1) / 2;
    const int blocks = (int)std::min<uint64_t>((n + kCovThreads - 1) / kCovThreads, (uint64_t)di.sms * 4);
    cudaMemPool_t pool;
    if ((s = get_pool(di.dev, &pool)) != CGS_SUCCESS) return s;
    const size_t bytes = 16 + sizeof(double) * (size_t)blocks * nt;
    void *scratch = nullptr;
    CGS_CUDA(cudaMallocFromPoolAsync(&scratch, bytes, pool, stream), "cudaMallocFromPoolAsync");
    CovParams p{};
    p.dims = D;
    for (int a = 0; a < 8; a++) {
        p.start[a] = a < D ? grid->start[a] : 0.0f;
        p.res[a] = a < D ? grid->resolution[a] : 0.0f;
        p.inc[a] = a < D ? inc[a] : 1;
    }
    p.costs = costs;
    p.n = (uint32_t)n;
    p.key = static_cast<unsigned long long *>(scratch);
    p.ticket = reinterpret_cast<unsigned int *>(static_cast<char *>(scratch) + 8);
    p.partial = reinterpret_cast<double *>(static_cast<char *>(scratch) + 16);
    p.out = covar;
    cudaError_t e = cudaMemsetAsync(scratch, 0xff, 16, stream);
    if (e == cudaSuccess) {
        cov_min_kernel<<<blocks, kCovThreads, 0, stream>>>(p);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        switch (D) {
            case 1: launch_sum<1>(blocks, stream, p); break;
            case 2: launch_sum<2>(blocks, stream, p); break;
            case 3: launch_sum<3>(blocks, stream, p); break;
            case 4: launch_sum<4>(blocks, stream, p); break;
            case 5: launch_sum<5>(blocks, stream, p); break;
            case 6: launch_sum<6>(blocks, stream, p); break;
            case 7: launch_sum<7>(blocks, stream, p); break;
            default: launch_sum<8>(blocks, stream, p); break;
        }
        e = cudaGetLastError();
    }
    cudaFreeAsync(scratch, stream);
    if (e != cudaSuccess) return cuda_fail(e, "covariance");
    return CGS_SUCCESS;
}

}  // extern "C"
