// cgs_verify.cu -- the FP64 verification pass of a search.
//
// A search sums in FP32 (partial sums per lane, folded in FP64 for ZNCC); its argmin is decided
// on those FP32 costs.  The verification pass re-scores, with FP64 sums, every grid point whose
// FP32 cost lies within a band of the FP32 minimum -- 2e-5 x max(1, |best|), twice the per-point
// FP32 tolerance, so that the FP64 argmin of the whole grid is among them whenever the FP32 costs
// are within tolerance -- and reports, in the search's cgs_argmin:
//   cost_fp64     the FP64 cost of the reported index,
//   err_fp64      |FP32 cost - FP64 cost| of the reported index,
//   index_fp64    the lowest FP64 cost among the re-scored points (lowest index on ties),
//   max_err_fp64  the largest |FP32 - FP64| among them,
//   verified / candidates  how many points were re-scored / lay in the band (at most kVerifyMax
//                 are re-scored; the first found when more lie in the band).
// Each re-scored point is one CTA: every fixed pixel sampled with the reference's exact operation
// sequence (calcNewCoordH + inImage + valueAt_bilinear, src/gpu/cudaImageFunctions.cuh:277-285,
// include/cudaTensor.cuh:548-575), the cost's moments summed in FP64 and the cost formed in FP64
// -- the same samples and arithmetic as the CPU oracle's FP64 functions, so cost_fp64 agrees with
// them to the FP64 summation order.
#include <algorithm>

#include "cgs_internal.h"

namespace cgs {

struct VerifyHdr {
    unsigned int count;   // points found in the band
    unsigned int ticket;  // CTAs done
    uint32_t cand[kVerifyMax];
    double c64[kVerifyMax];
};

size_t verify_scratch_bytes() { return sizeof(VerifyHdr); }

bool verify_supported(int cost) {
    return cost == CGS_COST_SAD_AVG || cost == CGS_COST_SAD_AVG_H || cost == CGS_COST_SAD_SUM_T ||
           cost == CGS_COST_SAD_SUM_T_REF || cost == CGS_COST_SQD_REF || cost == CGS_COST_NCC_REF ||
           cost == CGS_COST_ZNCC || cost == CGS_COST_MI;
}

// Band of the FP32 minimum: every point within it, up to kVerifyMax, into the header.
__global__ void verify_collect_kernel(const float *__restrict__ costs, uint32_t n, const cgs_argmin *res,
                                      VerifyHdr *h) {
    const cgs_argmin r = *res;
    if (!r.valid) return;
    const float best = r.cost;
    const float thr = best + 2e-5f * fmaxf(1.0f, fabsf(best));
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float c = __ldg(costs + i);
        if (c <= thr) {
            const unsigned int slot = atomicAdd(&h->count, 1u);
            if (slot < (unsigned int)kVerifyMax) h->cand[slot] = i;
        }
    }
}

__device__ __forceinline__ double block_sum(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];  // the same order in every thread
    return s;
}

// FP64 cost of grid index `idx` (the whole CTA; every thread returns it).
template <int COST>
__device__ double rescore(const SearchParams &p, uint32_t idx, double *red, uint32_t *hist) {
    int32_t ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int32_t rem = (int32_t)idx;
    for (int a = p.dims - 1; a >= 0; a--) {
        ax[a] = rem / p.inc[a];
        rem -= ax[a] * p.inc[a];
    }
    float q[8];
    grid_values(p, ax, q);
    const float2 cs = p.trig[min(ax[0], kMaxTrig - 1)];
    const MapCoef k = make_coef<COST>(q, cs, p);
    const int fw = p.fix.w, fh = p.fix.h, C = p.fix.c;
    const float mw = p.mov_wf, mh = p.mov_hf;
    constexpr bool kAll = COST == CGS_COST_SAD_SUM_T_REF;  // outside samples read as 0 and count
    const int B = p.mi_bins;
    const float sB = (float)B * (1.0f / 256.0f);
    if constexpr (COST == CGS_COST_MI) {
        for (int i = threadIdx.x; i < B * B; i += blockDim.x) hist[i] = 0u;
        __syncthreads();
    }
    const double fsh = COST == CGS_COST_ZNCC ? (double)p.shifts[0] : 0.0;
    const double msh = COST == CGS_COST_ZNCC ? (double)p.shifts[1] : 0.0;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, cnt = 0.0;
    const int64_t npix = (int64_t)fw * fh;
    for (int64_t i = threadIdx.x; i < npix; i += blockDim.x) {
        const int y = (int)(i / fw), x = (int)(i - (int64_t)y * fw);
        float ex, ey;
        exact_map(k, (float)x, (float)y, ex, ey);
        const bool inside = in_image(ey, ex, mw, mh);
        if (!inside && !kAll) continue;
        for (int c = 0; c < C; c++) {
            const float fv = p.fix.data[c * p.fix.plane + (int64_t)y * p.fix.pitch + x];
            const float mv = inside ? bilinear_in(p.mov.data + c * p.mov.plane, p.mov.pitch, ey, ex) : 0.0f;
            if constexpr (COST == CGS_COST_SAD_AVG || COST == CGS_COST_SAD_AVG_H || COST == CGS_COST_SAD_SUM_T ||
                          COST == CGS_COST_SAD_SUM_T_REF) {
                s0 += (double)fabsf(xs(mv, fv));
            } else if constexpr (COST == CGS_COST_NCC_REF || COST == CGS_COST_SQD_REF) {
                const float temp = xd(mv, 255.0f), fn = xd(fv, 255.0f), ff = xd(xm(fn, fv), 255.0f);
                if constexpr (COST == CGS_COST_NCC_REF) {
                    s0 += (double)ff;                          // i1
                    s1 += (double)temp * (double)temp;         // i2
                    s2 += (double)fn * (double)temp;           // ic
                } else {
                    const double d = (double)temp - (double)fn;
                    s0 += d * d;                               // out
                    s1 += (double)temp * (double)temp;         // i1
                    s2 += (double)ff;                          // i2
                }
            } else if constexpr (COST == CGS_COST_ZNCC) {
                const double f = (double)fv - fsh, m = (double)mv - msh;
                s0 += f;
                s1 += m;
                s2 += f * f;
                s3 += m * m;
                s4 += f * m;
            } else if constexpr (COST == CGS_COST_MI) {
                const int bf = min(max((int)floorf(fv * sB), 0), B - 1);
                const int bm = min(max((int)floorf(mv * sB), 0), B - 1);
                atomicAdd(&hist[bf * B + bm], 1u);
            }
            cnt += 1.0;
        }
    }
    const double n = block_sum(cnt, red);
    if constexpr (COST == CGS_COST_MI) {
        __syncthreads();  // every count is in
        double acc = 0.0;
        for (int i = threadIdx.x; i < B * B; i += blockDim.x) {
            const uint32_t v = hist[i];
            if (!v) continue;
            const int bf = i / B, bm = i - bf * B;
            uint32_t hf = 0, hm = 0;
            for (int j = 0; j < B; j++) {
                hf += hist[bf * B + j];
                hm += hist[j * B + bm];
            }
            acc += (double)v * log2(((double)v * n) / ((double)hf * (double)hm));
        }
        acc = block_sum(acc, red);
        if (n == 0.0 || (float)n < p.gate_n) return __longlong_as_double(0x7ff0000000000000ll);
        return -(acc / n) * (n / (double)p.total_terms);
    } else {
        s0 = block_sum(s0, red);
        s1 = block_sum(s1, red);
        s2 = block_sum(s2, red);
        if constexpr (COST == CGS_COST_SAD_AVG || COST == CGS_COST_SAD_AVG_H) {
            return s0 / n;  // 0 / 0 is NaN, as in the reference
        } else if constexpr (COST == CGS_COST_SAD_SUM_T || COST == CGS_COST_SAD_SUM_T_REF) {
            return s0;
        } else if constexpr (COST == CGS_COST_NCC_REF) {
            return n > 0.0 ? -s2 / sqrt(s0 * s1) : 0.0;
        } else if constexpr (COST == CGS_COST_SQD_REF) {
            return n > 0.0 ? s0 / sqrt(s1 * s2) : 123123.0;
        } else {
            s3 = block_sum(s3, red);
            s4 = block_sum(s4, red);
            const double a[5] = {s0, s1, s2, s3, s4};
            const double inf = __longlong_as_double(0x7ff0000000000000ll);
            if (n == 0.0 || (float)n < p.gate_n) return inf;
            const double cov = a[4] - a[0] * a[1] / n, vf = a[2] - a[0] * a[0] / n, vm = a[3] - a[1] * a[1] / n;
            if (!(vf > kZnccDegenerate * a[2]) || !(vm > kZnccDegenerate * a[3])) return inf;
            return -cov / sqrt(vf * vm);
        }
    }
}

// FP64 order of a cost: NaN and +inf never win (as the argmin keys).
__device__ __forceinline__ bool fp64_less(double a, uint32_t ia, double b, uint32_t ib) {
    const bool fa = a < __longlong_as_double(0x7ff0000000000000ll), fb = b < __longlong_as_double(0x7ff0000000000000ll);
    if (fa != fb) return fa;
    if (!fa) return ia < ib;
    return a < b || (a == b && ia < ib);
}

// One CTA per band point; the last CTA writes the verification fields of the result.
template <int COST>
__global__ void __launch_bounds__(256) verify_kernel(const __grid_constant__ SearchParams p, VerifyHdr *h) {
    extern __shared__ __align__(16) unsigned char vsm[];
    double *red = reinterpret_cast<double *>(vsm);
    uint32_t *hist = reinterpret_cast<uint32_t *>(vsm + 32 * sizeof(double));
    __shared__ unsigned int last;
    const cgs_argmin r0 = *p.result;
    const unsigned int found = r0.valid ? h->count : 0u;
    const unsigned int nc = min(found, (unsigned int)kVerifyMax);
    if (blockIdx.x < nc) {
        const double c = rescore<COST>(p, h->cand[blockIdx.x], red, hist);
        if (threadIdx.x == 0) h->c64[blockIdx.x] = c;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&h->ticket, 1u) + 1u == gridDim.x;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    cgs_argmin r = *p.result;
    r.verified = (int32_t)nc;
    r.candidates = (int32_t)found;
    r.cost_fp64 = __longlong_as_double(0x7ff8000000000000ll);
    r.err_fp64 = r.cost_fp64;
    r.max_err_fp64 = 0.0;
    r.index_fp64 = -1;
    uint32_t bi = 0;
    double bc = 0.0;
    bool have = false;
    for (unsigned int k = 0; k < nc; k++) {
        const uint32_t i = h->cand[k];
        const double c64 = h->c64[k], c32 = (double)p.costs[i];
        if (!have || fp64_less(c64, i, bc, bi)) {
            bi = i;
            bc = c64;
            have = true;
        }
        const double e = fabs(c32 - c64);
        if (e == e) r.max_err_fp64 = fmax(r.max_err_fp64, e);
        if ((int64_t)i == r.index) {
            r.cost_fp64 = c64;
            r.err_fp64 = fabs((double)r.cost - c64);
        }
    }
    if (have) r.index_fp64 = (int64_t)bi;
    *p.result = r;
}

// Band collection and re-scoring on `stream` after a search whose costs are in p.costs and whose
// result is p.result.  hdr: zeroed device scratch of verify_scratch_bytes().
cgs_status launch_verify(const SearchParams &p, void *hdr, cudaStream_t stream, int sms) {
    VerifyHdr *h = static_cast<VerifyHdr *>(hdr);
    const int blocks = (int)std::min<uint64_t>((p.n + 255) / 256, (uint64_t)sms * 4);
    verify_collect_kernel<<<blocks, 256, 0, stream>>>(p.costs, p.n, p.result, h);
    const void *kfn = nullptr;
    switch (p.cost) {
        case CGS_COST_SAD_AVG: kfn = (const void *)verify_kernel<CGS_COST_SAD_AVG>; break;
        case CGS_COST_SAD_AVG_H: kfn = (const void *)verify_kernel<CGS_COST_SAD_AVG_H>; break;
        case CGS_COST_SAD_SUM_T: kfn = (const void *)verify_kernel<CGS_COST_SAD_SUM_T>; break;
        case CGS_COST_SAD_SUM_T_REF: kfn = (const void *)verify_kernel<CGS_COST_SAD_SUM_T_REF>; break;
        case CGS_COST_SQD_REF: kfn = (const void *)verify_kernel<CGS_COST_SQD_REF>; break;
        case CGS_COST_NCC_REF: kfn = (const void *)verify_kernel<CGS_COST_NCC_REF>; break;
        case CGS_COST_ZNCC: kfn = (const void *)verify_kernel<CGS_COST_ZNCC>; break;
        case CGS_COST_MI: kfn = (const void *)verify_kernel<CGS_COST_MI>; break;
        default: return CGS_SUCCESS;  // not re-scored: verified = 0
    }
    const size_t smem = 32 * sizeof(double) + (p.cost == CGS_COST_MI ? (size_t)p.mi_bins * p.mi_bins * 4 : 0);
    SearchParams pv = p;
    void *args[] = {&pv, &h};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaLaunchKernel(kfn, dim3(kVerifyMax), dim3(256), args, smem, stream);
    if (e != cudaSuccess) return cuda_fail(e, "verification pass");
    return CGS_SUCCESS;
}

}  // namespace cgs
