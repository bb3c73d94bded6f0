// cgs_device.cuh -- device building blocks of the sm_100a grid search.
//
// Bit-exact sampling.  The reference evaluates its cost functors with plain FP32
// operators; built for the host (its CPU path) no multiply-add is fused.  Every value
// that feeds a DISCRETE decision -- the homography, the mapped coordinates (in/out of the
// moving image, floor/ceil taps), the bilinear weights and the interpolated value (MI bin
// index) -- is computed here with explicitly rounded intrinsics in the reference's
// operation order, so each sample equals the reference's host sample bit for bit.  Only
// the order of the cost SUMS differs (warp-parallel instead of sequential).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cugridsearch_b200.h"

namespace cgs {

// Explicitly rounded FP32 operations: never contracted into FMA by the compiler.  The host
// versions are plain IEEE operations (the host build has no fused multiply-add).
#ifdef __CUDA_ARCH__
#define CGS_RN(dev, op) return dev(a, b)
#else
#define CGS_RN(dev, op) return a op b
#endif
__host__ __device__ __forceinline__ float xm(float a, float b) { CGS_RN(__fmul_rn, *); }
__host__ __device__ __forceinline__ float xa(float a, float b) { CGS_RN(__fadd_rn, +); }
__host__ __device__ __forceinline__ float xs(float a, float b) { CGS_RN(__fsub_rn, -); }
__host__ __device__ __forceinline__ float xd(float a, float b) { CGS_RN(__fdiv_rn, /); }
#undef CGS_RN

// Homography h11..h32 (h33 = 1), row-major without h33.
struct Homog {
    float h11, h12, h13, h21, h22, h23, h31, h32;
};

// parametersToHomography (src/gpu/cudaImageFunctions.cuh:216-252): centred on (cx, cy),
// decomposition C*K*T*R*Sh*Sc*C, normalised by h33.  Parameters [theta, sx, sy, shear,
// tx, ty, kx, ky]; c, s = cos(theta), sin(theta) from the host (same libm as the
// reference's CPU path).  Parenthesisation follows C's parse of the reference lines.
__host__ __device__ __forceinline__ Homog h_centred(const float *q, float c, float s, float cx, float cy) {
    const float sx = q[1], sy = q[2], sh = q[3], tx = q[4], ty = q[5], kx = q[6], ky = q[7];
    const float a2 = xa(xm(cx, kx), 1.0f);
    const float a4 = xm(cx, ky);
    const float a6 = xa(xm(c, a2), xm(a4, s));
    const float t5 = xa(xs(xm(sh, a6), xm(s, a2)), xm(a4, c));
    const float u3 = xm(cx, sx), u6 = xm(cy, sy);
    const float b2 = xa(xm(cy, ky), 1.0f);
    const float b4 = xm(cy, kx);
    const float b6 = xa(xm(s, b2), xm(b4, c));
    const float v5 = xs(xa(xm(sh, b6), xm(c, b2)), xm(b4, s));
    const float d3 = xa(xm(kx, c), xm(ky, s));
    const float e5 = xs(xa(xm(sh, d3), xm(ky, c)), xm(kx, s));
    const float h11 = xm(sx, a6);
    const float h12 = xm(sy, t5);
    const float h13 = xa(xs(xs(xa(cx, xm(tx, a2)), xm(u3, a6)), xm(u6, t5)), xm(a4, ty));
    const float h21 = xm(sx, b6);
    const float h22 = xm(sy, v5);
    const float h23 = xa(xs(xs(xa(cy, xm(ty, b2)), xm(u3, b6)), xm(u6, v5)), xm(b4, tx));
    const float h31 = xm(sx, d3);
    const float h32 = xm(sy, e5);
    const float h33 = xa(xs(xs(xa(xm(kx, tx), xm(ky, ty)), xm(u6, e5)), xm(u3, d3)), 1.0f);
    Homog h;
    h.h11 = xd(h11, h33); h.h12 = xd(h12, h33); h.h13 = xd(h13, h33);
    h.h21 = xd(h21, h33); h.h22 = xd(h22, h33); h.h23 = xd(h23, h33);
    h.h31 = xd(h31, h33); h.h32 = xd(h32, h33);
    return h;
}

// Uncentred parametrisation of averageAbsoluteDifference (src/gpu/cudaErrorFunctions.cuh:42-57).
__host__ __device__ __forceinline__ Homog h_uncentred(const float *q, float c, float s) {
    const float sx = q[1], sy = q[2], sh = q[3], tx = q[4], ty = q[5];
    Homog h;
    h.h11 = xm(sx, c);
    h.h12 = xs(xm(xm(sy, sh), c), xm(sy, s));
    h.h13 = xm(sx, tx);
    h.h21 = xm(sx, s);
    h.h22 = xa(xm(xm(sy, sh), s), xm(sy, c));
    h.h23 = xm(sy, ty);
    h.h31 = q[6];
    h.h32 = q[7];
    return h;
}

// Inverse map of calcNewCoordH (src/gpu/cudaImageFunctions.cuh:277-285): fixed pixel
// (x, y) -> moving coordinates through the adjugate of H.  The coefficient products are
// per grid point; the per-pixel part keeps the reference's association
// (((A*x + B*y) + P) - Q) / w.
struct InvMap {
    float A, B, P, Q;      // w  = ((A*x + B*y) + P) - Q
    float C1, C2, R, S;    // X  = ((C1*x + C2*y) + R) - S
    float D1, D2, T, U;    // Y  = ((D1*x + D2*y) + T) - U

    __device__ __forceinline__ void set(const Homog &h) {
        A = xs(xm(h.h21, h.h32), xm(h.h22, h.h31));
        B = xs(xm(h.h12, h.h31), xm(h.h11, h.h32));
        P = xm(h.h11, h.h22);
        Q = xm(h.h12, h.h21);
        C1 = xs(h.h22, xm(h.h23, h.h32));
        C2 = xs(xm(h.h13, h.h32), h.h12);
        R = xm(h.h12, h.h23);
        S = xm(h.h13, h.h22);
        D1 = xs(xm(h.h23, h.h31), h.h21);
        D2 = xs(h.h11, xm(h.h13, h.h31));
        T = xm(h.h13, h.h21);
        U = xm(h.h11, h.h23);
    }
    __device__ __forceinline__ void map(float x, float y, float &mx, float &my) const {
        const float w = xs(xa(xa(xm(A, x), xm(B, y)), P), Q);
        const float X = xs(xa(xa(xm(C1, x), xm(C2, y)), R), S);
        const float Y = xs(xa(xa(xm(D1, x), xm(D2, y)), T), U);
        mx = xd(X, w);
        my = xd(Y, w);
    }
};

// Forward raw-H map of averageAbsoluteDifferenceH (src/gpu/cudaErrorFunctions.cuh:205-207):
// z = H[6]*x + H[7]*y + 1.0 (the double add of the float sum and 1.0 rounds once, like a
// float add), y' = (H[3]*x + H[4]*y + H[5]) / z, x' = (H[0]*x + H[1]*y + H[2]) / z.
struct RawMap {
    float H[8];
    __device__ __forceinline__ void map(float x, float y, float &mx, float &my) const {
        const float z = xa(xa(xm(H[6], x), xm(H[7], y)), 1.0f);
        my = xd(xa(xa(xm(H[3], x), xm(H[4], y)), H[5]), z);
        mx = xd(xa(xa(xm(H[0], x), xm(H[1], y)), H[2]), z);
    }
};

// Staged image: one FP32 plane per channel.  The reference addresses a CudaImage with a flat
// index, so a ceil(x) == W tap reads pixel 0 of the NEXT row and a tap in row H reads past
// the image (CudaImage::valueAt_bilinear, include/cudaTensor.cuh:561-566 with toIndex :531-534).
// The staged moving image makes that explicit in a pitched layout: column W of row y holds
// pixel (0, y + 1) (zero for the last row) and row H is zero, so 2x2 taps at (x, y) and
// (x + 1, y + 1) read exactly the reference's values for every in-image sample, through plain
// loads or texture gathers alike.  Planes are stacked: plane c starts at row c * (H + 1).
struct Plane {
    const float *data;
    int32_t h, w, c;
    int32_t pitch;   // row pitch in floats
    int64_t plane;   // plane stride in floats
};

// CudaImage::inImage (include/cudaTensor.cuh:548-550).
__device__ __forceinline__ bool in_image(float y, float x, float wf, float hf) {
    return x >= 0.0f && y >= 0.0f && x < wf && y < hf;
}

// CudaImage::valueAt_bilinear at an in-image point (include/cudaTensor.cuh:561-575), in the
// reference's operation order.  The right/bottom taps are read at floor + 1; where the
// reference's ceil equals floor (an integral coordinate) the weight of that tap is exactly 0,
// so the value is the same.  pl is a staged moving plane with row pitch `pitch`.
__device__ __forceinline__ float bilinear_in(const float *__restrict__ pl, int32_t pitch, float y, float x) {
    const float fy = floorf(y), fx = floorf(x);
    const int32_t i = (int32_t)fx + pitch * (int32_t)fy;
    const float tlc = __ldg(pl + i);
    const float trc = __ldg(pl + i + 1);
    const float blc = __ldg(pl + i + pitch);
    const float brc = __ldg(pl + i + pitch + 1);
    const float ax = xs(x, fx), ay = xs(y, fy);
    const float omx = xs(1.0f, ax), omy = xs(1.0f, ay);
    const float top = xa(xm(omx, tlc), xm(ax, trc));
    const float bot = xa(xm(omx, blc), xm(ax, brc));
    return xa(xm(omy, top), xm(ay, bot));
}

// Orderable 64-bit argmin key: (cost bits mapped to unsigned order) << 32 | index.
// Lowest key = lowest cost, then lowest index.  NaN and +inf never win (~0).
__device__ __forceinline__ unsigned long long make_key(float v, uint32_t index) {
    if (!(v < __int_as_float(0x7f800000))) return ~0ull;
    uint32_t b = __float_as_uint(v);
    if (v == 0.0f) b = 0u;  // -0 and +0 compare equal: same key
    b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return ((unsigned long long)b << 32) | (unsigned long long)index;
}

__host__ __device__ __forceinline__ float key_cost(unsigned long long k) {
    uint32_t b = (uint32_t)(k >> 32);
    b = (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}

// The FP64 verification fields of a result before (or without) a verification pass.
__host__ __device__ __forceinline__ void clear_verify_fields(cgs_argmin &r) {
    r.verified = 0;
    r.candidates = 0;
    r.reserved = 0;
    r.index_fp64 = -1;
    r.cost_fp64 = __builtin_nan("");
    r.err_fp64 = __builtin_nan("");
    r.max_err_fp64 = 0.0;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u < v ? u : v;
    }
    return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---- mbarrier + bulk-copy (TMA) helpers, sm_90+ PTX ----------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// One contiguous global -> shared bulk copy; dst, src and bytes multiples of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: gives up after `limit_ns` of wall time and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

}  // namespace cgs
