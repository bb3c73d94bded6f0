// cgs_net.cu -- the learned proposal network: a small CNN that looks at an image pair and
// predicts where the grid search's argmin lies (a centre per parameter) and how sure it is
// (a log-radius per parameter), trained and run with hand-written sm_100a kernels.
//
// Architecture.  Input: the pair box-averaged to 128 x 128, fixed and moving as 2 channels,
// (v - 127.5) / 64.  Five 3x3 stride-2 convolutions (pad 1, channels 32-64-128-128-256, ReLU):
// 128 -> 64 -> 32 -> 16 -> 8 -> 4; global average pool (256); fc 256 -> 128 + ReLU; fc
// 128 -> 16 (8 centres in [-1, 1] grid-range units, 8 log-radii).
//
// Numerics.  Activations are NHWC BF16, weights FP32 masters with BF16 copies; every
// convolution is an implicit GEMM on the BF16 tensor cores with FP32 accumulation: the forward
// and the data gradient on tcgen05 (UMMA, TMEM accumulators; conv_umma_kernel), the weight
// gradient on mma.sync m16n8k16; pooling, the MLP, the loss and Adam run in FP32.
//
// Loss.  Laplace negative log-likelihood of the label y per parameter: |c - y| e^-s + s with
// s clamped to [-6, 4] (no gradient outside), averaged over batch and parameters.
//
// Parameters are one flat FP32 vector: for each conv layer W [Cout][Kp] (Kp = 9 Cin rounded up
// to 32, the padding zero) then b [Cout]; fc1 W [128][256], b [128]; fc2 W [16][128], b [16].
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "cgs_internal.h"

typedef __nv_bfloat16 bf16;

namespace cgs {
namespace net {

constexpr int kLayers = 5;
constexpr int kCin[kLayers] = {2, 32, 64, 128, 128};
constexpr int kCout[kLayers] = {32, 64, 128, 128, 256};
constexpr int kSide = 128;  // input side; layer l output side = 64 >> l
constexpr int kFeat = 256, kHid = 128, kOut = 16, kParams8 = 8;

__host__ __device__ constexpr int side_in(int l) { return kSide >> l; }
__host__ __device__ constexpr int side_out(int l) { return kSide >> (l + 1); }
constexpr int kdim(int l) { return 9 * kCin[l]; }
constexpr int kpad(int l) { return (kdim(l) + 31) / 32 * 32; }

// Offsets of the flat parameter vector.
struct Layout {
    int64_t w[kLayers], b[kLayers];
    int64_t fc1w, fc1b, fc2w, fc2b, total;
    Layout() {
        int64_t o = 0;
        for (int l = 0; l < kLayers; l++) {
            w[l] = o;
            o += (int64_t)kCout[l] * kpad(l);
            b[l] = o;
            o += kCout[l];
        }
        fc1w = o;
        o += (int64_t)kHid * kFeat;
        fc1b = o;
        o += kHid;
        fc2w = o;
        o += (int64_t)kOut * kHid;
        fc2b = o;
        o += kOut;
        total = o;
    }
};

// ---------------------------------------------------------------- tensor-core tile

constexpr int BM = 64, BN = 64, BK = 32, PAD = 8, LDS = BK + PAD;  // smem row: 80 bytes
constexpr int kThreads = 128;                                        // 4 warps, 32 x 32 each

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A warp's 32 x 32 block of C += A[BM x BK] B[BK x BN] for one BK slice.  As is [BM][LDS] and
// Bs is [BN][LDS], both k-contiguous.  Fragments of m16n8k16 (g = lane / 4, t = lane % 4):
// A regs {row g, k 2t..}, {row g+8, k 2t..}, {row g, k 2t+8..}, {row g+8, k 2t+8..};
// B regs {k 2t.., col g}, {k 2t+8.., col g}; C {row g, col 2t, 2t+1}, {row g+8, col 2t, 2t+1}.
__device__ __forceinline__ void warp_mma(const bf16 *As, const bf16 *Bs, int wm, int wn, float (&acc)[2][4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
        uint32_t a[2][4], b[4][2];
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const bf16 *p = As + (wm + i * 16 + g) * LDS + kk + 2 * t;
            a[i][0] = *reinterpret_cast<const uint32_t *>(p);
            a[i][1] = *reinterpret_cast<const uint32_t *>(p + 8 * LDS);
            a[i][2] = *reinterpret_cast<const uint32_t *>(p + 8);
            a[i][3] = *reinterpret_cast<const uint32_t *>(p + 8 * LDS + 8);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bf16 *p = Bs + (wn + j * 8 + g) * LDS + kk + 2 * t;
            b[j][0] = *reinterpret_cast<const uint32_t *>(p);
            b[j][1] = *reinterpret_cast<const uint32_t *>(p + 8);
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], a[i], b[j]);
    }
}

// Output coordinates of accumulator element (i, j, r) of warp (wm, wn) in a tile at (m0, n0).
__device__ __forceinline__ void acc_coord(int m0, int n0, int wm, int wn, int i, int j, int r, int &m, int &n) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    m = m0 + wm + i * 16 + g + ((r & 2) ? 8 : 0);
    n = n0 + wn + j * 8 + 2 * t + (r & 1);
}

// ---------------------------------------------------------------- convolution problems

// Geometry of conv layer l on a batch of n: input [n][H][H][Cin], output [n][Ho][Ho][Cout].
struct ConvGeom {
    int n, H, Ho, Cin, Cout, K, Kp;
};

// 8 consecutive k = (tap, ci) of the im2col row of output pixel (b, ho, wo), as bf16 (zeros
// outside the image and past K).
__device__ __forceinline__ uint4 im2col8(const bf16 *__restrict__ x, const ConvGeom &g, int b, int ho, int wo,
                                         int k8) {
    uint4 v = make_uint4(0, 0, 0, 0);
    if (k8 >= g.K) return v;
    if ((g.Cin & 7) == 0) {
        const int tap = k8 / g.Cin, ci = k8 - tap * g.Cin;
        const int hi = 2 * ho + tap / 3 - 1, wi = 2 * wo + tap % 3 - 1;
        if (hi >= 0 && hi < g.H && wi >= 0 && wi < g.H)
            v = *reinterpret_cast<const uint4 *>(x + (((int64_t)b * g.H + hi) * g.H + wi) * g.Cin + ci);
        return v;
    }
    bf16 e[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int k = k8 + j;
        e[j] = __float2bfloat16_rn(0.0f);
        if (k < g.K) {
            const int tap = k / g.Cin, ci = k - tap * g.Cin;
            const int hi = 2 * ho + tap / 3 - 1, wi = 2 * wo + tap % 3 - 1;
            if (hi >= 0 && hi < g.H && wi >= 0 && wi < g.H) e[j] = x[(((int64_t)b * g.H + hi) * g.H + wi) * g.Cin + ci];
        }
    }
    memcpy(&v, e, 16);
    return v;
}

// Forward: y[m][co] = relu(sum_k im2col(m, k) w[co][k] + bias[co]), m = (b, ho, wo).
__global__ void __launch_bounds__(kThreads) conv_fwd_kernel(const bf16 *__restrict__ x, const bf16 *__restrict__ w,
                                                            const float *__restrict__ bias, bf16 *__restrict__ y,
                                                            const ConvGeom g) {
    __shared__ __align__(16) bf16 As[BM * LDS];
    __shared__ __align__(16) bf16 Bs[BN * LDS];
    const int M = g.n * g.Ho * g.Ho;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int warp = threadIdx.x >> 5, wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4] = {};
    for (int k0 = 0; k0 < g.Kp; k0 += BK) {
#pragma unroll
        for (int rep = 0; rep < 2; rep++) {
            const int c = threadIdx.x + rep * kThreads;
            const int row = c >> 2, k8 = k0 + (c & 3) * 8;
            const int m = m0 + row;
            uint4 va = make_uint4(0, 0, 0, 0);
            if (m < M) {
                const int b = m / (g.Ho * g.Ho), r = m - b * g.Ho * g.Ho, ho = r / g.Ho, wo = r - ho * g.Ho;
                va = im2col8(x, g, b, ho, wo, k8);
            }
            *reinterpret_cast<uint4 *>(As + row * LDS + (c & 3) * 8) = va;
            const int co = n0 + row;
            uint4 vb = make_uint4(0, 0, 0, 0);
            if (co < g.Cout) vb = *reinterpret_cast<const uint4 *>(w + (int64_t)co * g.Kp + k8);
            *reinterpret_cast<uint4 *>(Bs + row * LDS + (c & 3) * 8) = vb;
        }
        __syncthreads();
        warp_mma(As, Bs, wm, wn, acc);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r += 2) {
                int m, co;
                acc_coord(m0, n0, wm, wn, i, j, r, m, co);
                if (m < M && co < g.Cout) {
                    const float v0 = fmaxf(acc[i][j][r] + bias[co], 0.0f);
                    const float v1 = fmaxf(acc[i][j][r + 1] + bias[co + 1], 0.0f);
                    *reinterpret_cast<__nv_bfloat162 *>(y + (int64_t)m * g.Cout + co) = __floats2bfloat162_rn(v0, v1);
                }
            }
}

// ---------------------------------------------------------------- forward on tcgen05 (UMMA)
//
// The forward convolution as an implicit GEMM on the 5th-generation tensor cores: D[m][co] =
// sum_k A[m][k] B[co][k], m = (b, ho, wo) output pixels, k = (tap, ci).  A (gathered, im2col)
// and B (the BF16 weights, [Cout][Kp]) are staged in shared memory by the CTA's 512 threads
// with cp.async; one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M = 128, N =
// the CTA's channels, Cout or 64, K = 16 per instruction) into a TMEM accumulator of N columns,
// completion tracked by tcgen05.commit on an mbarrier per stage (two stages: the next K slice is
// gathered while the tensor cores work on the current one).  The epilogue reads the accumulator
// back with tcgen05.ld (warp w owns TMEM lanes 32 (w % 4) .. + 31, i.e. output rows, and every
// fourth group of 32 columns from w / 4), adds the bias, applies ReLU and stores BF16.
//
// Shared-memory operands use the UMMA K-major layout without swizzle: 16-byte chunks of 8
// consecutive k of one row, chunk (row, kc) at 16 (kc * ROWS + row) bytes, so 8 consecutive
// rows of a chunk column form one 128-byte core matrix; descriptor strides: between row
// groups of 8 (SBO) 128 bytes, between the two 8-k halves of a K = 16 instruction (LBO)
// 16 ROWS bytes.
constexpr int kUmmaM = 128, kUmmaBK = 64;  // rows per tile, k per stage (up to four K = 16 instructions)
constexpr int kUmmaT = 512;                 // threads per CTA: 4 per output row for the gathers

// 16-byte global -> shared copy (cp.async, L2 only); bytes = 0 fills the 16 bytes with zeros.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(bytes)
                 : "memory");
}

// Shared-memory matrix descriptor: start address, leading and stride byte offsets (16-byte
// units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// BWD = false: the forward, x = the layer's input, w = [Cout][Kp], y = relu(conv + bias).
// BWD = true: the data gradient, x = the output gradient dy [n][Ho][Ho][Cout], w = the transposed
// weights [Cin][9 Cout], mask = the previous layer's output (ReLU mask), y = dx [n][H][H][Cin].
// With stride 2 an input pixel (hi, wi) receives only the taps ky = hi + 1 (mod 2), kx = wi + 1
// (mod 2), so the rows are split by parity class (py, px) = (hi, wi) mod 2 (blockIdx.z, the four-tap
// class first): a class's rows are the pixels (2i + py, 2j + px) and its K = (1 + py)(1 + px) Cout,
// k = (t, co) over the class's taps t = (ty, tx), ky = py ? 2 ty : 1, kx = px ? 2 tx : 1, which
// read dy at (i + py (1 - ty), j + px (1 - tx)) where that is inside the output.
template <int N, bool BWD>
__global__ void __launch_bounds__(kUmmaT) conv_umma_kernel(const bf16 *__restrict__ x, const bf16 *__restrict__ w,
                                                           const float *__restrict__ bias,
                                                           const bf16 *__restrict__ mask, bf16 *__restrict__ y,
                                                           const ConvGeom g, unsigned int *__restrict__ status) {
    static_assert(N % 16 == 0 && N >= 32 && N <= 256 && (N & (N - 1)) == 0, "TMEM columns: a power of two, 32..256");
    constexpr int kA = kUmmaM * kUmmaBK * 2, kB = N * kUmmaBK * 2;  // bytes per stage
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sA[2] = {smem, smem + kA};
    unsigned char *sB[2] = {smem + 2 * kA, smem + 2 * kA + kB};
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * kA + 2 * kB);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
    volatile int *gave_up = reinterpret_cast<volatile int *>(tslot + 1);  // a bounded wait gave up
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int side = BWD ? g.H >> 1 : g.Ho;  // rows: output pixels, or one parity class of input pixels
    const int M = g.n * side * side;
    const int ph = BWD ? 3 - (int)blockIdx.z : 0, py = ph >> 1, px = ph & 1, ntx = 1 + px;
    const int KT = BWD ? (1 + py) * ntx * g.Cout : g.Kp;  // GEMM K (a multiple of 32; of 64 for BWD)
    const int wstride = BWD ? 9 * g.Cout : g.Kp;           // B row stride
    const int CO = BWD ? g.Cin : g.Cout;                   // GEMM N: the output's channels
    const int m0 = blockIdx.x * kUmmaM, co0 = blockIdx.y * N;  // this CTA: rows m0.., channels co0 .. co0 + N
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        *gave_up = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tacc = *tslot;
    const int nk = (KT + kUmmaBK - 1) / kUmmaBK;  // KT is a multiple of 32: the last slice may be half
    constexpr uint32_t idesc = umma_idesc_bf16(kUmmaM, N);
    // this thread's output row (its im2col row), decoded once; its chunks kc = part + 4 j
    const int row = threadIdx.x & (kUmmaM - 1), part = threadIdx.x >> 7, m = m0 + row;
    const bool mvalid = m < M;
    int b = 0, ho = 0, wo = 0;
    if (mvalid) {
        b = m / (side * side);
        const int r = m - b * side * side;
        ho = r / side;  // (i, j) of the parity class for the data gradient
        wo = r - ho * side;
    }
    // one K slice into stage st2: A chunks by cp.async (16 bytes of one tap's channels; zero
    // fill outside the image and past K), or gathered through registers where 8 consecutive k
    // span taps (Cin = 2: four taps of two channels; other Cin not a multiple of 8: element by
    // element); B chunks by cp.async
    auto load_slice = [&](int kb2, int st2) {
        const int k0 = kb2 * kUmmaBK;
        const int kchunks = min(kUmmaBK, KT - k0) >> 3;
        int woff = 0;  // BWD: a slice lies inside one tap t (64 divides Cout); B reads wt's block of tap(t)
        if constexpr (BWD) {
            const int t = k0 / g.Cout, ty = t / ntx, tx = t - ty * ntx;
            woff = (3 * (py ? 2 * ty : 1) + (px ? 2 * tx : 1) - t) * g.Cout;
        }
#pragma unroll
        for (int j = 0; j < kUmmaBK / 8 / (kUmmaT / kUmmaM); j++) {
            const int kc = part + (kUmmaT / kUmmaM) * j;
            unsigned char *dst = sA[st2] + 16 * (kc * kUmmaM + row);
            const int k8 = k0 + kc * 8;
            if constexpr (BWD) {
                // 8 consecutive k = 8 output channels of one tap (Cout is a multiple of 8)
                const bf16 *src = x;
                uint32_t bytes = 0;
                if (mvalid && kc < kchunks) {
                    const int t = k8 / g.Cout, co = k8 - t * g.Cout, ty = t / ntx, tx = t - ty * ntx;
                    const int ho2 = ho + py * (1 - ty), wo2 = wo + px * (1 - tx);
                    if (ho2 < g.Ho && wo2 < g.Ho) {
                        src = x + (((int64_t)b * g.Ho + ho2) * g.Ho + wo2) * g.Cout + co;
                        bytes = 16;
                    }
                }
                cp_async16(dst, src, bytes);
            } else if ((g.Cin & 7) == 0) {
                const bf16 *src = x;
                uint32_t bytes = 0;
                if (mvalid && kc < kchunks && k8 < g.K) {
                    const int tap = k8 / g.Cin, ci = k8 - tap * g.Cin;
                    const int hi = 2 * ho + tap / 3 - 1, wi = 2 * wo + tap % 3 - 1;
                    if (hi >= 0 && hi < g.H && wi >= 0 && wi < g.H) {
                        src = x + (((int64_t)b * g.H + hi) * g.H + wi) * g.Cin + ci;
                        bytes = 16;
                    }
                }
                cp_async16(dst, src, bytes);
            } else if (g.Cin == 2) {
                // 8 consecutive k = 4 taps x 2 channels: four 4-byte loads
                uint32_t v[4] = {0u, 0u, 0u, 0u};
                if (mvalid && kc < kchunks) {
#pragma unroll
                    for (int t = 0; t < 4; t++) {
                        const int tap = (k8 >> 1) + t;
                        if (2 * tap < g.K) {
                            const int hi = 2 * ho + tap / 3 - 1, wi = 2 * wo + tap % 3 - 1;
                            if (hi >= 0 && hi < g.H && wi >= 0 && wi < g.H)
                                v[t] = *reinterpret_cast<const uint32_t *>(x + (((int64_t)b * g.H + hi) * g.H + wi) * 2);
                        }
                    }
                }
                *reinterpret_cast<uint4 *>(dst) = make_uint4(v[0], v[1], v[2], v[3]);
            } else {
                uint4 va = make_uint4(0, 0, 0, 0);
                if (mvalid && kc < kchunks) va = im2col8(x, g, b, ho, wo, k8);
                *reinterpret_cast<uint4 *>(dst) = va;
            }
        }
        for (int c = threadIdx.x; c < N * (kUmmaBK / 8); c += kUmmaT) {
            const int co = c % N, kc = c / N;
            const bool v = kc < kchunks;
            cp_async16(sB[st2] + 16 * (kc * N + co),
                       v ? w + (int64_t)(co0 + co) * wstride + woff + k0 + kc * 8 : w, v ? 16u : 0u);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    load_slice(0, 0);
    for (int kb = 0; kb < nk; kb++) {
        const int st = kb & 1;
        const int kchunks = min(kUmmaBK, KT - kb * kUmmaBK) >> 3;
        if (kb + 1 < nk) {
            // stage (kb + 1) & 1 is free once the MMAs of slice kb - 1 are done
            if (kb >= 1 && !*gave_up &&
                !mbar_wait_bounded(&bars[(kb + 1) & 1], (uint32_t)((kb - 1) >> 1) & 1u, kWaitLimitNs))
                *gave_up = 1;
            load_slice(kb + 1, (kb + 1) & 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");  // slice kb has landed
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        fence_proxy_async_smem();  // this thread's copies and stores, before the tensor cores read them
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (threadIdx.x == 0 && !*gave_up) {
#pragma unroll
            for (int j = 0; j < kUmmaBK / 16; j++) {
                if (2 * j >= kchunks) break;  // a half slice: two instructions
                const uint64_t da = umma_smem_desc(smem_addr(sA[st]) + j * 2 * 16 * kUmmaM, 16 * kUmmaM, 128);
                const uint64_t db = umma_smem_desc(smem_addr(sB[st]) + j * 2 * 16 * N, 16 * N, 128);
                const uint32_t acc = (kb > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tacc),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&bars[st]))
                         : "memory");
        }
    }
    // the last commit tracks every MMA issued before it
    const int last = nk - 1;
    if (!*gave_up && !mbar_wait_bounded(&bars[last & 1], (uint32_t)(last >> 1) & 1u, kWaitLimitNs)) *gave_up = 1;
    const bool ok = __syncthreads_and(*gave_up == 0) != 0;  // the same decision in every warp
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        // a wait gave up: the tensor cores may still be writing the accumulator; give the last
        // commit one more bounded wait before the columns are freed
        if (threadIdx.x == 0) {
            atomicOr(status, 1u);
            mbar_wait_bounded(&bars[last & 1], (uint32_t)(last >> 1) & 1u, kWaitLimitNs);
        }
    } else {
        // warp w reads TMEM lanes 32 (w % 4) .. + 31 (its output rows) and every (T / 128)-th group
        // of 32 columns from group w / 4
        const int mr = m0 + 32 * (warp & 3) + lane;  // the row; its pixel mo
        int mo = mr;
        if constexpr (BWD) {
            const int bb = mr / (side * side), r = mr - bb * side * side, i = r / side, j = r - i * side;
            mo = (bb * g.H + 2 * i + py) * g.H + 2 * j + px;
        }
#pragma unroll 1
        for (int c0 = 32 * (warp >> 2); c0 < N; c0 += 32 * (kUmmaT / kUmmaM)) {
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(tacc + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (mr < M) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int64_t o0 = (int64_t)mo * CO + co0 + c0 + 8 * q;
                    __nv_bfloat162 o[4];
                    if constexpr (BWD) {  // the previous layer's ReLU mask
                        const uint4 pv = *reinterpret_cast<const uint4 *>(mask + o0);
                        const __nv_bfloat162 *pm = reinterpret_cast<const __nv_bfloat162 *>(&pv);
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            const float2 pf = __bfloat1622float2(pm[i]);
                            const int c = 8 * q + 2 * i;
                            o[i] = __floats2bfloat162_rn(pf.x > 0.0f ? __uint_as_float(r[c]) : 0.0f,
                                                         pf.y > 0.0f ? __uint_as_float(r[c + 1]) : 0.0f);
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            const int c = 8 * q + 2 * i;
                            o[i] = __floats2bfloat162_rn(fmaxf(__uint_as_float(r[c]) + bias[co0 + c0 + c], 0.0f),
                                                         fmaxf(__uint_as_float(r[c + 1]) + bias[co0 + c0 + c + 1], 0.0f));
                        }
                    }
                    *reinterpret_cast<uint4 *>(y + o0) = *reinterpret_cast<const uint4 *>(o);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tacc), "r"(N));
}

// Dynamic shared memory of conv_umma_kernel<N, BWD>: two stages of A and B, the barriers and the
// TMEM address, rounded up where needed so that at most 512 / N CTAs share an SM (the TMEM
// columns of all resident CTAs then fit; no allocation waits).  At 512 threads per CTA at most 4
// CTAs are resident anyway.
static size_t umma_fwd_smem(int N) {
    const size_t need = 2 * (size_t)(kUmmaM + N) * kUmmaBK * 2 + 64;
    const size_t per_sm = 228 * 1024, cap = (size_t)(512 / N);
    if (cap >= (size_t)(2048 / kUmmaT)) return need;
    const size_t floor_for_cap = per_sm / (cap + 1) + 1024;
    return std::max(need, std::min(floor_for_cap, (size_t)227 * 1024));
}

template <int N, bool BWD>
static cudaError_t launch_umma_n(const bf16 *x, const bf16 *w, const float *bias, const bf16 *mask, bf16 *y,
                                 const ConvGeom &g, int blocks, int channels, unsigned int *status, cudaStream_t s) {
    const size_t smem = umma_fwd_smem(N);
    cudaError_t e = cudaFuncSetAttribute(conv_umma_kernel<N, BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    conv_umma_kernel<N, BWD><<<dim3(blocks, channels / N, BWD ? 4 : 1), kUmmaT, smem, s>>>(x, w, bias, mask, y, g,
                                                                                           status);
    return cudaGetLastError();
}

// One layer's forward convolution (bwd = false: x, w = [Cout][Kp], bias -> y) or data gradient
// (bwd = true: dy, w = [Cin][9 Cout], ReLU mask -> dx) on the tensor cores; output channels 32,
// 64, 128 or 256.  Layers with fewer than two row tiles per SM split their channels over CTAs
// of 64 (the A tile is then gathered once per channel tile).
static cudaError_t launch_conv_umma(bool bwd, const bf16 *x, const bf16 *w, const float *bias, const bf16 *mask,
                                    bf16 *y, const ConvGeom &g, unsigned int *status, cudaStream_t s, int sms) {
    // the data gradient runs the four parity classes of input pixels as grid.z (stride 2, H even)
    if (bwd && ((g.H & 1) || g.Ho != g.H / 2 || (g.Cout & 63))) return cudaErrorInvalidValue;
    const int side = bwd ? g.H / 2 : g.Ho, channels = bwd ? g.Cin : g.Cout;
    const int blocks = (g.n * side * side + kUmmaM - 1) / kUmmaM;
    const int nt = (channels > 64 && blocks * (bwd ? 4 : 1) < 2 * sms) ? 64 : channels;
    if (bwd) {
        switch (nt) {
            case 32: return launch_umma_n<32, true>(x, w, bias, mask, y, g, blocks, channels, status, s);
            case 64: return launch_umma_n<64, true>(x, w, bias, mask, y, g, blocks, channels, status, s);
            case 128: return launch_umma_n<128, true>(x, w, bias, mask, y, g, blocks, channels, status, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (nt) {
        case 32: return launch_umma_n<32, false>(x, w, bias, mask, y, g, blocks, channels, status, s);
        case 64: return launch_umma_n<64, false>(x, w, bias, mask, y, g, blocks, channels, status, s);
        case 128: return launch_umma_n<128, false>(x, w, bias, mask, y, g, blocks, channels, status, s);
        case 256: return launch_umma_n<256, false>(x, w, bias, mask, y, g, blocks, channels, status, s);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------- weight gradient on tcgen05
//
// D[k][co] = sum_p A[k][p] dy[p][co] for one tile of 128 im2col columns k (blockIdx.x) over the
// pixels of one split (blockIdx.z), in slices of 64 pixels; A[k][p] = im2col(p, k) for k < K, 0
// for K <= k < Kp, and 1 for k = Kp, so that accumulator row Kp is the bias gradient.  Both
// operands are MN-major in shared memory: the natural 16-byte chunk (8 consecutive k, or 8
// channels, of one pixel) is one row of a core matrix, chunk (pixel p, chunk column c) at
// 1024 c + 16 p bytes; descriptor strides: between pixel groups of 8 (LBO, the K direction) 128
// bytes, between chunk columns (SBO, the M / N direction) 1024 bytes.  The epilogue writes
// part[z][co][k] (k < Kp) and partb[z][co] (k = Kp), summed over splits in a fixed order after.
template <int N>
__global__ void __launch_bounds__(kUmmaT) conv_wgrad_umma_kernel(const bf16 *__restrict__ dy,
                                                                 const bf16 *__restrict__ x, float *__restrict__ part,
                                                                 float *__restrict__ partb, const ConvGeom g,
                                                                 int slices_per_split,
                                                                 unsigned int *__restrict__ status) {
    static_assert(N >= 32 && N <= 256 && (N & (N - 1)) == 0, "TMEM columns: a power of two, 32..256");
    constexpr int kA = kUmmaM * 64 * 2, kB = N * 64 * 2;  // bytes per stage: 128 rows k / N channels x 64 pixels
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sA[2] = {smem, smem + kA};
    unsigned char *sB[2] = {smem + 2 * kA, smem + 2 * kA + kB};
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * kA + 2 * kB);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
    volatile int *gave_up = reinterpret_cast<volatile int *>(tslot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int P = g.n * g.Ho * g.Ho, k0 = blockIdx.x * kUmmaM;
    const int s_begin = blockIdx.z * slices_per_split;
    const int ns = min(slices_per_split, (P + 63) / 64 - s_begin);  // >= 1 by the launch's split count
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        *gave_up = 0;
    }
    // chunk columns of A past K hold the same values for every pixel: zeros, and the 1 of row Kp
    const int pl = threadIdx.x & 63, cg = threadIdx.x >> 6;  // this thread's pixel in a slice, first chunk column
    const int kreal = (g.K - k0 + 7) >> 3;                    // chunk columns with im2col values (may be <= 0)
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int c = cg + 8 * j;
        if (c >= kreal) {
            const int kb = k0 + 8 * c;
            const uint32_t one = (g.Kp >= kb && g.Kp < kb + 8) ? 0x3F80u << (16 * ((g.Kp - kb) & 1)) : 0u;
            const int word = (g.Kp - kb) >> 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (one) {
                if (word == 0) v.x = one;
                else if (word == 1) v.y = one;
                else if (word == 2) v.z = one;
                else v.w = one;
            }
            *reinterpret_cast<uint4 *>(sA[0] + 1024 * c + 16 * pl) = v;
            *reinterpret_cast<uint4 *>(sA[1] + 1024 * c + 16 * pl) = v;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tacc = *tslot;
    constexpr uint32_t idesc = umma_idesc_bf16(kUmmaM, N) | (1u << 15) | (1u << 16);  // A and B MN-major
    // one slice of 64 pixels into stage st2: A's im2col chunks and B's dy chunks by cp.async
    // (zero fill outside the image and past the last pixel), Cin = 2 through registers
    auto load_slice = [&](int si, int st2) {
        const int p = (s_begin + si) * 64 + pl;
        const bool pv = p < P;
        int b = 0, ho = 0, wo = 0;
        if (pv) {
            b = p / (g.Ho * g.Ho);
            const int r = p - b * g.Ho * g.Ho;
            ho = r / g.Ho;
            wo = r - ho * g.Ho;
        }
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int c = cg + 8 * j;
            if (c < kreal) {
                unsigned char *dst = sA[st2] + 1024 * c + 16 * pl;
                const int k8 = k0 + 8 * c;
                if ((g.Cin & 7) == 0) {
                    const bf16 *src = x;
                    uint32_t bytes = 0;
                    if (pv) {
                        const int tap = k8 / g.Cin, ci = k8 - tap * g.Cin;
                        const int hi = 2 * ho + tap / 3 - 1, wi = 2 * wo + tap % 3 - 1;
                        if (hi >= 0 && hi < g.H && wi >= 0 && wi < g.H) {
                            src = x + (((int64_t)b * g.H + hi) * g.H + wi) * g.Cin + ci;
                            bytes = 16;
                        }
                    }
                    cp_async16(dst, src, bytes);
                } else if (g.Cin == 2) {
                    uint32_t v[4] = {0u, 0u, 0u, 0u};
                    if (pv) {
#pragma unroll
                        for (int t = 0; t < 4; t++) {
                            const int tap = (k8 >> 1) + t;
                            if (2 * tap < g.K) {
                                const int hi = 2 * ho + tap / 3 - 1, wi = 2 * wo + tap % 3 - 1;
                                if (hi >= 0 && hi < g.H && wi >= 0 && wi < g.H)
                                    v[t] = *reinterpret_cast<const uint32_t *>(
                                        x + (((int64_t)b * g.H + hi) * g.H + wi) * 2);
                            }
                        }
                    }
                    *reinterpret_cast<uint4 *>(dst) = make_uint4(v[0], v[1], v[2], v[3]);
                } else {
                    *reinterpret_cast<uint4 *>(dst) = pv ? im2col8(x, g, b, ho, wo, k8) : make_uint4(0, 0, 0, 0);
                }
            }
        }
        for (int c = cg; c < N / 8; c += 8)
            cp_async16(sB[st2] + 1024 * c + 16 * pl, pv ? dy + (int64_t)p * g.Cout + 8 * c : dy, pv ? 16u : 0u);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    load_slice(0, 0);
    for (int si = 0; si < ns; si++) {
        const int st = si & 1;
        if (si + 1 < ns) {
            // stage (si + 1) & 1 is free once the MMAs of slice si - 1 are done
            if (si >= 1 && !*gave_up &&
                !mbar_wait_bounded(&bars[(si + 1) & 1], (uint32_t)((si - 1) >> 1) & 1u, kWaitLimitNs))
                *gave_up = 1;
            load_slice(si + 1, (si + 1) & 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        fence_proxy_async_smem();
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (threadIdx.x == 0 && !*gave_up) {
#pragma unroll
            for (int j = 0; j < 4; j++) {  // K = 16 pixels per instruction: pixel groups 2 j, 2 j + 1
                const uint64_t da = umma_smem_desc(smem_addr(sA[st]) + 256 * j, 128, 1024);
                const uint64_t db = umma_smem_desc(smem_addr(sB[st]) + 256 * j, 128, 1024);
                const uint32_t acc = (si > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tacc),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&bars[st]))
                         : "memory");
        }
    }
    const int last = ns - 1;
    if (!*gave_up && !mbar_wait_bounded(&bars[last & 1], (uint32_t)(last >> 1) & 1u, kWaitLimitNs)) *gave_up = 1;
    const bool ok = __syncthreads_and(*gave_up == 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (threadIdx.x == 0) {
            atomicOr(status, 1u);
            mbar_wait_bounded(&bars[last & 1], (uint32_t)(last >> 1) & 1u, kWaitLimitNs);
        }
    } else {
        const int k = k0 + 32 * (warp & 3) + lane;  // this thread's accumulator row
        float *out = part + (int64_t)blockIdx.z * g.Cout * g.Kp;
#pragma unroll 1
        for (int c0 = 32 * (warp >> 2); c0 < N; c0 += 32 * (kUmmaT / kUmmaM)) {
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(tacc + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (k < g.Kp) {
#pragma unroll
                for (int i = 0; i < 32; i++) out[(int64_t)(c0 + i) * g.Kp + k] = __uint_as_float(r[i]);
            } else if (k == g.Kp) {
#pragma unroll
                for (int i = 0; i < 32; i++) partb[(int64_t)blockIdx.z * g.Cout + c0 + i] = __uint_as_float(r[i]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tacc), "r"(N));
}

// Splits of the pixel slices for conv_wgrad_umma_kernel: about two CTAs per SM over the k tiles,
// at least four slices per split.
static int wgrad_umma_splits(const ConvGeom &g, int sms, int *slices_per_split) {
    const int slices = (g.n * g.Ho * g.Ho + 63) / 64, ktiles = g.Kp / kUmmaM + 1;
    int splits = std::max(1, std::min(slices / 4, (2 * sms + ktiles - 1) / ktiles));
    *slices_per_split = (slices + splits - 1) / splits;
    return (slices + *slices_per_split - 1) / *slices_per_split;
}

template <int N>
static cudaError_t launch_wgrad_n(const bf16 *dy, const bf16 *x, float *part, float *partb, const ConvGeom &g,
                                  int splits, int sps, unsigned int *status, cudaStream_t s) {
    const size_t smem = umma_fwd_smem(N);
    cudaError_t e = cudaFuncSetAttribute(conv_wgrad_umma_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    conv_wgrad_umma_kernel<N><<<dim3(g.Kp / kUmmaM + 1, 1, splits), kUmmaT, smem, s>>>(dy, x, part, partb, g, sps,
                                                                                       status);
    return cudaGetLastError();
}

// One layer's weight and bias gradient partials on the tensor cores (Cout 32, 64, 128 or 256).
static cudaError_t launch_conv_wgrad_umma(const bf16 *dy, const bf16 *x, float *part, float *partb,
                                          const ConvGeom &g, int splits, int sps, unsigned int *status,
                                          cudaStream_t s) {
    switch (g.Cout) {
        case 32: return launch_wgrad_n<32>(dy, x, part, partb, g, splits, sps, status, s);
        case 64: return launch_wgrad_n<64>(dy, x, part, partb, g, splits, sps, status, s);
        case 128: return launch_wgrad_n<128>(dy, x, part, partb, g, splits, sps, status, s);
        case 256: return launch_wgrad_n<256>(dy, x, part, partb, g, splits, sps, status, s);
        default: return cudaErrorInvalidValue;
    }
}

// Data gradient: dx[m][ci] = sum_{tap, co} dy[pixel reached by tap][co] wt[ci][tap][co], m =
// (b, hi, wi) an input pixel; masked by the previous layer's ReLU (xprev > 0) and stored as
// that layer's output gradient.  Cout is a multiple of 8, so 8 consecutive k share a tap.
__global__ void __launch_bounds__(kThreads) conv_bwd_data_kernel(const bf16 *__restrict__ dy,
                                                                 const bf16 *__restrict__ wt,
                                                                 const bf16 *__restrict__ xprev,
                                                                 bf16 *__restrict__ dx, const ConvGeom g) {
    __shared__ __align__(16) bf16 As[BM * LDS];
    __shared__ __align__(16) bf16 Bs[BN * LDS];
    const int M = g.n * g.H * g.H;
    const int KD = 9 * g.Cout;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int warp = threadIdx.x >> 5, wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4] = {};
    for (int k0 = 0; k0 < KD; k0 += BK) {
#pragma unroll
        for (int rep = 0; rep < 2; rep++) {
            const int c = threadIdx.x + rep * kThreads;
            const int row = c >> 2, k8 = k0 + (c & 3) * 8;
            const int m = m0 + row;
            uint4 va = make_uint4(0, 0, 0, 0);
            if (m < M) {
                const int b = m / (g.H * g.H), r = m - b * g.H * g.H, hi = r / g.H, wi = r - hi * g.H;
                const int tap = k8 / g.Cout, co = k8 - tap * g.Cout;
                const int ho2 = hi + 1 - tap / 3, wo2 = wi + 1 - tap % 3;
                if (ho2 >= 0 && wo2 >= 0 && !(ho2 & 1) && !(wo2 & 1) && (ho2 >> 1) < g.Ho && (wo2 >> 1) < g.Ho)
                    va = *reinterpret_cast<const uint4 *>(
                        dy + (((int64_t)b * g.Ho + (ho2 >> 1)) * g.Ho + (wo2 >> 1)) * g.Cout + co);
            }
            *reinterpret_cast<uint4 *>(As + row * LDS + (c & 3) * 8) = va;
            const int ci = n0 + row;
            uint4 vb = make_uint4(0, 0, 0, 0);
            if (ci < g.Cin) vb = *reinterpret_cast<const uint4 *>(wt + (int64_t)ci * KD + k8);
            *reinterpret_cast<uint4 *>(Bs + row * LDS + (c & 3) * 8) = vb;
        }
        __syncthreads();
        warp_mma(As, Bs, wm, wn, acc);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r += 2) {
                int m, ci;
                acc_coord(m0, n0, wm, wn, i, j, r, m, ci);
                if (m < M && ci < g.Cin) {
                    const int64_t o = (int64_t)m * g.Cin + ci;
                    const float p0 = __bfloat162float(xprev[o]), p1 = __bfloat162float(xprev[o + 1]);
                    *reinterpret_cast<__nv_bfloat162 *>(dx + o) =
                        __floats2bfloat162_rn(p0 > 0.0f ? acc[i][j][r] : 0.0f, p1 > 0.0f ? acc[i][j][r + 1] : 0.0f);
                }
            }
}

// Weight gradient, split over pixels: part[z][co][k] = sum over pixel tiles of split z of
// dy[p][co] im2col(p, k).  M' = Cout, N' = Kp, K' = pixels; both operands are gathered with
// pixels innermost in shared memory.
__global__ void __launch_bounds__(kThreads) conv_bwd_weight_kernel(const bf16 *__restrict__ dy,
                                                                   const bf16 *__restrict__ x, float *__restrict__ part,
                                                                   const ConvGeom g, int tiles_per_split) {
    __shared__ __align__(16) bf16 As[BM * LDS];
    __shared__ __align__(16) bf16 Bs[BN * LDS];
    const int P = g.n * g.Ho * g.Ho;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int warp = threadIdx.x >> 5, wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4] = {};
    const int t_begin = blockIdx.z * tiles_per_split;
    const int t_end = min(t_begin + tiles_per_split, (P + BK - 1) / BK);
    for (int tile = t_begin; tile < t_end; tile++) {
        const int p0 = tile * BK;
        // each thread: pixel pl = tid % 32, 8-wide channel groups (tid / 32) + 4 * rep
#pragma unroll
        for (int rep = 0; rep < 2; rep++) {
            const int pl = threadIdx.x & 31, grp = (threadIdx.x >> 5) + rep * 4;  // 8 groups of 8 rows
            const int p = p0 + pl;
            const bool pv = p < P;
            int b = 0, ho = 0, wo = 0;
            if (pv) {
                b = p / (g.Ho * g.Ho);
                const int r = p - b * g.Ho * g.Ho;
                ho = r / g.Ho;
                wo = r - ho * g.Ho;
            }
            const int co = m0 + grp * 8;
            uint4 va = make_uint4(0, 0, 0, 0);
            if (pv && co < g.Cout) va = *reinterpret_cast<const uint4 *>(dy + (int64_t)p * g.Cout + co);
            const bf16 *ea = reinterpret_cast<const bf16 *>(&va);
#pragma unroll
            for (int j = 0; j < 8; j++) As[(grp * 8 + j) * LDS + pl] = ea[j];
            const int k8 = n0 + grp * 8;
            uint4 vb = make_uint4(0, 0, 0, 0);
            if (pv) vb = im2col8(x, g, b, ho, wo, k8);
            const bf16 *eb = reinterpret_cast<const bf16 *>(&vb);
#pragma unroll
            for (int j = 0; j < 8; j++) Bs[(grp * 8 + j) * LDS + pl] = eb[j];
        }
        __syncthreads();
        warp_mma(As, Bs, wm, wn, acc);
        __syncthreads();
    }
    float *out = part + (int64_t)blockIdx.z * g.Cout * g.Kp;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) {
                int co, k;
                acc_coord(m0, n0, wm, wn, i, j, r, co, k);
                if (co < g.Cout && k < g.Kp) out[(int64_t)co * g.Kp + k] = acc[i][j][r];
            }
}

// dst[i] = sum_z part[z][i] in split order (deterministic).
__global__ void sum_splits_kernel(const float *__restrict__ part, int splits, int64_t n, float *__restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float s = 0.0f;
        int z = 0;
        for (; z + 8 <= splits; z += 8) {  // eight loads in flight, added in split order
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = part[(int64_t)(z + u) * n + i];
#pragma unroll
            for (int u = 0; u < 8; u++) s += v[u];
        }
        for (; z < splits; z++) s += part[(int64_t)z * n + i];
        dst[i] = s;
    }
}

// Bias gradient partials: part[chunk][c] = sum of dy[p][c] over the chunk's pixels.
__global__ void bias_grad_kernel(const bf16 *__restrict__ dy, int P, int C, int chunk, float *__restrict__ part) {
    const int c = threadIdx.x;
    if (c >= C) return;
    const int p0 = blockIdx.x * chunk, p1 = min(P, p0 + chunk);
    float s = 0.0f;
    for (int p = p0; p < p1; p++) s += __bfloat162float(dy[(int64_t)p * C + c]);
    part[(int64_t)blockIdx.x * C + c] = s;
}

// ---------------------------------------------------------------- input, pooling, MLP, loss

// x0[b][y][x][0] = fixed, [..][1] = moving, each the s x s box average of an (s 128)^2 image,
// normalised as (v - 127.5) / 64.
__global__ void input_kernel(const float *__restrict__ fixed, const float *__restrict__ moving, int n, int s,
                             bf16 *__restrict__ x0) {
    const int64_t total = (int64_t)n * kSide * kSide;
    const int side = kSide * s;
    const float inv = 1.0f / (float)(s * s);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / (kSide * kSide));
        const int r = (int)(i - (int64_t)b * kSide * kSide), yy = r / kSide, xx = r - yy * kSide;
        float f = 0.0f, m = 0.0f;
        for (int dy = 0; dy < s; dy++)
            for (int dx = 0; dx < s; dx++) {
                const int64_t o = ((int64_t)b * side + yy * s + dy) * side + xx * s + dx;
                f += fixed[o];
                m += moving[o];
            }
        x0[2 * i] = __float2bfloat16_rn((f * inv - 127.5f) * (1.0f / 64.0f));
        x0[2 * i + 1] = __float2bfloat16_rn((m * inv - 127.5f) * (1.0f / 64.0f));
    }
}

// feat[b][c] = mean of y5[b][16 positions][c].
__global__ void gap_kernel(const bf16 *__restrict__ y5, int n, float *__restrict__ feat) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kFeat) return;
    const int b = i / kFeat, c = i - b * kFeat;
    float s = 0.0f;
    for (int p = 0; p < 16; p++) s += __bfloat162float(y5[((int64_t)b * 16 + p) * kFeat + c]);
    feat[i] = s * (1.0f / 16.0f);
}

// out[b][j] = act(sum_i w[j][i] in[b][i] + bias[j]); act = ReLU when relu != 0.
__global__ void fc_kernel(const float *__restrict__ in, const float *__restrict__ w, const float *__restrict__ bias,
                          int n, int nin, int nout, int relu, float *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * nout) return;
    const int b = i / nout, j = i - b * nout;
    float s = bias[j];
    for (int k = 0; k < nin; k++) s = fmaf(w[(int64_t)j * nin + k], in[(int64_t)b * nin + k], s);
    out[i] = relu ? fmaxf(s, 0.0f) : s;
}

constexpr float kSMin = -6.0f, kSMax = 4.0f;

// Laplace NLL per (sample, parameter) and its gradient w.r.t. the 16 outputs; lossp[b] = the
// sample's share of the mean loss.
__global__ void loss_kernel(const float *__restrict__ out, const float *__restrict__ labels, int n,
                            float *__restrict__ dout, float *__restrict__ lossp) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const float scale = 1.0f / (float)(n * kParams8);
    float L = 0.0f;
    for (int a = 0; a < kParams8; a++) {
        const float c = out[b * kOut + a], sr = out[b * kOut + 8 + a], y = labels[b * kParams8 + a];
        const float s = fminf(fmaxf(sr, kSMin), kSMax);
        const float e = fabsf(c - y), is = expf(-s);
        L += (e * is + s) * scale;
        dout[b * kOut + a] = (c > y ? is : (c < y ? -is : 0.0f)) * scale;
        dout[b * kOut + 8 + a] = (sr > kSMin && sr < kSMax) ? (1.0f - e * is) * scale : 0.0f;
    }
    lossp[b] = L;
}

// Backward of a dense layer (one thread per output): din[b][i] = mask * sum_j w[j][i] dout[b][j]
// with mask = (in > 0) when the input came through a ReLU; dw[j][i] = sum_b dout[b][j] in[b][i];
// db[j] = sum_b dout[b][j].
__global__ void fc_bwd_input_kernel(const float *__restrict__ dout, const float *__restrict__ w,
                                    const float *__restrict__ in, int n, int nin, int nout, int relu_in,
                                    float *__restrict__ din) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * nin) return;
    const int b = i / nin, k = i - b * nin;
    float s = 0.0f;
    for (int j = 0; j < nout; j++) s = fmaf(w[(int64_t)j * nin + k], dout[(int64_t)b * nout + j], s);
    din[i] = (!relu_in || in[i] > 0.0f) ? s : 0.0f;
}

__global__ void fc_bwd_weight_kernel(const float *__restrict__ dout, const float *__restrict__ in, int n, int nin,
                                     int nout, float *__restrict__ dw, float *__restrict__ db) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nout * (nin + 1)) return;
    const int j = i / (nin + 1), k = i - j * (nin + 1);
    // summed over the batch in order; the loads of 8 batch rows are issued before their 8
    // multiply-adds, so the loop waits on memory once per 8 rows instead of once per row
    float s = 0.0f;
    if (k < nin) {
        int b = 0;
        for (; b + 8 <= n; b += 8) {
            float u[8], v[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                u[t] = dout[(int64_t)(b + t) * nout + j];
                v[t] = in[(int64_t)(b + t) * nin + k];
            }
#pragma unroll
            for (int t = 0; t < 8; t++) s = fmaf(u[t], v[t], s);
        }
        for (; b < n; b++) s = fmaf(dout[(int64_t)b * nout + j], in[(int64_t)b * nin + k], s);
        dw[(int64_t)j * nin + k] = s;
    } else {
        int b = 0;
        for (; b + 8 <= n; b += 8) {
            float u[8];
#pragma unroll
            for (int t = 0; t < 8; t++) u[t] = dout[(int64_t)(b + t) * nout + j];
#pragma unroll
            for (int t = 0; t < 8; t++) s += u[t];
        }
        for (; b < n; b++) s += dout[(int64_t)b * nout + j];
        db[j] = s;
    }
}

// Pooling backward through layer 5's ReLU: dy5[b][p][c] = (y5 > 0) dfeat[b][c] / 16.
__global__ void gap_bwd_kernel(const float *__restrict__ dfeat, const bf16 *__restrict__ y5, int n,
                               bf16 *__restrict__ dy5) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 16 * kFeat) return;
    const int b = i / (16 * kFeat), c = i % kFeat;
    const float v = __bfloat162float(y5[i]) > 0.0f ? dfeat[b * kFeat + c] * (1.0f / 16.0f) : 0.0f;
    dy5[i] = __float2bfloat16_rn(v);
}

// Adam (bias-corrected) on the flat parameters; conv weights are then copied to BF16, row-major
// [Cout][Kp] and transposed [Cin][9][Cout] (for the data gradient).
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ gr, float *__restrict__ m1,
                            float *__restrict__ m2, int64_t n, float lr, float c1, float c2) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = gr[i];
        const float a = b1 * m1[i] + (1.0f - b1) * gi;
        const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = v;
        p[i] -= lr * (a * c1) / (sqrtf(v * c2) + eps);
    }
}

__global__ void to_bf16_kernel(const float *__restrict__ w, int cout, int kp, int cin, bf16 *__restrict__ wb,
                               bf16 *__restrict__ wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cout * kp) return;
    const int co = i / kp, k = i - co * kp;
    const bf16 v = __float2bfloat16_rn(w[i]);
    wb[i] = v;
    if (wt && k < 9 * cin) {
        const int tap = k / cin, ci = k - tap * cin;
        wt[((int64_t)ci * 9 + tap) * cout + co] = v;
    }
}

}  // namespace net
}  // namespace cgs

using namespace cgs;
using namespace cgs::net;

// The network: parameters, Adam moments, gradients (flat FP32), BF16 weight copies and the
// activations and gradients of one batch of up to max_batch pairs.
struct cgs_net {
    int dev = -1;
    int sms = 0;
    int max_batch = 0;
    int n = 0;     // batch size of the last forward
    int64_t step = 0;
    Layout L;
    char *mem = nullptr;
    float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
    bf16 *wb[kLayers] = {}, *wt[kLayers] = {};
    bf16 *act[kLayers + 1] = {};  // act[0] = input, act[l + 1] = conv layer l output
    bf16 *dya = nullptr, *dyb = nullptr;  // ping-pong output gradients
    float *feat = nullptr, *hid = nullptr, *out = nullptr, *dout = nullptr, *dhid = nullptr, *dfeat = nullptr;
    float *lossp = nullptr;
    float *ws = nullptr;
    size_t ws_floats = 0;
    unsigned int *status = nullptr;  // tcgen05 forward: bit 0 = a bounded wait gave up
    bool conv_mma_sync = false;      // CGS_NET_CONV=mma_sync: the mma.sync forward and data gradient (comparisons)
    bool wgrad_mma_sync = false;     // CGS_NET_CONV=mma_sync or CGS_NET_WGRAD=mma_sync: the mma.sync weight gradient
};

namespace cgs {
namespace net {

static cgs_status sync_bf16(cgs_net *nt, cudaStream_t s) {
    for (int l = 0; l < kLayers; l++) {
        const int cnt = kCout[l] * kpad(l);
        to_bf16_kernel<<<(cnt + 255) / 256, 256, 0, s>>>(nt->params + nt->L.w[l], kCout[l], kpad(l), kCin[l], nt->wb[l],
                                                         l > 0 ? nt->wt[l] : nullptr);
    }
    CGS_CUDA(cudaGetLastError(), "to_bf16_kernel");
    return CGS_SUCCESS;
}

static ConvGeom geom(int l, int n) {
    ConvGeom g;
    g.n = n;
    g.H = side_in(l);
    g.Ho = side_out(l);
    g.Cin = kCin[l];
    g.Cout = kCout[l];
    g.K = kdim(l);
    g.Kp = kpad(l);
    return g;
}

// Splits of the weight-gradient GEMM: enough blocks to fill the GPU twice, at least 4 pixel
// tiles each.
static int wgrad_splits(const ConvGeom &g, int sms, int *tiles_per_split) {
    const int tiles = (g.n * g.Ho * g.Ho + BK - 1) / BK;
    const int base = ((g.Cout + BM - 1) / BM) * ((g.Kp + BN - 1) / BN);
    int splits = std::max(1, std::min(tiles / 4, (2 * sms + base - 1) / base));
    *tiles_per_split = (tiles + splits - 1) / splits;
    splits = (tiles + *tiles_per_split - 1) / *tiles_per_split;
    return splits;
}

static size_t ws_need(int n, int sms) {
    size_t need = 0;
    for (int l = 0; l < kLayers; l++) {
        const ConvGeom g = geom(l, n);
        int tps;
        const int sp = wgrad_splits(g, sms, &tps);
        need = std::max(need, (size_t)sp * g.Cout * g.Kp);
        const int P = n * g.Ho * g.Ho, chunk = 1024;
        need = std::max(need, (size_t)((P + chunk - 1) / chunk) * g.Cout);
        const int su = wgrad_umma_splits(g, sms, &tps);
        need = std::max(need, (size_t)su * g.Cout * (g.Kp + 1));
    }
    return need;
}

}  // namespace net
}  // namespace cgs

extern "C" {

int64_t cgs_net_param_count(void) { return Layout().total; }

cgs_status cgs_net_create(int32_t max_batch, uint64_t seed, cgs_net **out) {
    if (!out) return fail(CGS_ERROR_INVALID_VALUE, "out is null");
    *out = nullptr;
    if (max_batch < 1 || max_batch > 4096) return fail(CGS_ERROR_INVALID_VALUE, "max_batch must be 1..4096");
    cgs_status s;
    DeviceInfo di;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;
    cgs_net *nt = new cgs_net();
    nt->dev = di.dev;
    nt->sms = di.sms;
    nt->max_batch = max_batch;
    {
        const char *fv = std::getenv("CGS_NET_CONV");
        nt->conv_mma_sync = fv && std::string(fv) == "mma_sync";
        const char *wv = std::getenv("CGS_NET_WGRAD");
        nt->wgrad_mma_sync = nt->conv_mma_sync || (wv && std::string(wv) == "mma_sync");
    }
    const int64_t P = nt->L.total;
    const int64_t B = max_batch;
    // sizes in bytes, each block 256-aligned
    std::vector<size_t> sz;
    sz.push_back(4 * P * 4);  // params, grads, m1, m2
    size_t wbytes = 0;
    for (int l = 0; l < kLayers; l++) wbytes += 2 * ((size_t)kCout[l] * kpad(l) * 2 + 256);
    sz.push_back(wbytes);
    size_t abytes = (size_t)B * kSide * kSide * 2 * 2 + 256;
    size_t dmax = 0;
    for (int l = 0; l < kLayers; l++) {
        const size_t e = (size_t)B * side_out(l) * side_out(l) * kCout[l];
        abytes += e * 2 + 256;
        dmax = std::max(dmax, e);
    }
    sz.push_back(abytes);
    sz.push_back(2 * (dmax * 2 + 256));
    sz.push_back(((size_t)B * (2 * kFeat + 2 * kHid + 2 * kOut + 1)) * 4 + 7 * 256);
    nt->ws_floats = ws_need(max_batch, di.sms);
    sz.push_back(nt->ws_floats * 4 + 256);
    sz.push_back(256);  // status word
    size_t total = 0;
    for (size_t v : sz) total += (v + 255) / 256 * 256;
    cudaError_t e = cudaMalloc(&nt->mem, total);
    if (e != cudaSuccess) {
        delete nt;
        return cuda_fail(e, "cudaMalloc (network)");
    }
    char *p = nt->mem;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) / 256 * 256;
        return r;
    };
    nt->params = reinterpret_cast<float *>(take(P * 4));
    nt->grads = reinterpret_cast<float *>(take(P * 4));
    nt->m1 = reinterpret_cast<float *>(take(P * 4));
    nt->m2 = reinterpret_cast<float *>(take(P * 4));
    for (int l = 0; l < kLayers; l++) {
        nt->wb[l] = reinterpret_cast<bf16 *>(take((size_t)kCout[l] * kpad(l) * 2));
        nt->wt[l] = reinterpret_cast<bf16 *>(take((size_t)kCout[l] * kpad(l) * 2));
    }
    nt->act[0] = reinterpret_cast<bf16 *>(take((size_t)B * kSide * kSide * 2 * 2));
    for (int l = 0; l < kLayers; l++)
        nt->act[l + 1] = reinterpret_cast<bf16 *>(take((size_t)B * side_out(l) * side_out(l) * kCout[l] * 2));
    nt->dya = reinterpret_cast<bf16 *>(take(dmax * 2));
    nt->dyb = reinterpret_cast<bf16 *>(take(dmax * 2));
    nt->feat = reinterpret_cast<float *>(take((size_t)B * kFeat * 4));
    nt->dfeat = reinterpret_cast<float *>(take((size_t)B * kFeat * 4));
    nt->hid = reinterpret_cast<float *>(take((size_t)B * kHid * 4));
    nt->dhid = reinterpret_cast<float *>(take((size_t)B * kHid * 4));
    nt->out = reinterpret_cast<float *>(take((size_t)B * kOut * 4));
    nt->dout = reinterpret_cast<float *>(take((size_t)B * kOut * 4));
    nt->lossp = reinterpret_cast<float *>(take((size_t)B * 4));
    nt->ws = reinterpret_cast<float *>(take(nt->ws_floats * 4));
    nt->status = reinterpret_cast<unsigned int *>(take(4));

    // He-normal initialisation (std sqrt(2 / fan_in)); the last layer small so the first
    // proposals sit at the grid centre with radius ~1 (half the range)
    std::vector<float> h((size_t)P, 0.0f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    for (int l = 0; l < kLayers; l++) {
        const float sd = std::sqrt(2.0f / (float)kdim(l));
        for (int co = 0; co < kCout[l]; co++)
            for (int k = 0; k < kdim(l); k++) h[nt->L.w[l] + (int64_t)co * kpad(l) + k] = sd * nd(rng);
    }
    for (int64_t i = 0; i < (int64_t)kHid * kFeat; i++) h[nt->L.fc1w + i] = std::sqrt(2.0f / kFeat) * nd(rng);
    for (int64_t i = 0; i < (int64_t)kOut * kHid; i++) h[nt->L.fc2w + i] = 0.01f * nd(rng);
    e = cudaMemcpy(nt->params, h.data(), P * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(nt->m1, 0, P * 4);
    if (e == cudaSuccess) e = cudaMemset(nt->m2, 0, P * 4);
    if (e == cudaSuccess) e = cudaMemset(nt->grads, 0, P * 4);
    if (e == cudaSuccess) e = cudaMemset(nt->status, 0, 4);
    for (int l = 1; l < kLayers && e == cudaSuccess; l++) e = cudaMemset(nt->wt[l], 0, (size_t)kCout[l] * kpad(l) * 2);
    if (e != cudaSuccess) {
        cudaFree(nt->mem);
        delete nt;
        return cuda_fail(e, "network init");
    }
    if ((s = sync_bf16(nt, 0)) != CGS_SUCCESS || (e = cudaDeviceSynchronize()) != cudaSuccess) {
        cudaFree(nt->mem);
        delete nt;
        return s != CGS_SUCCESS ? s : cuda_fail(e, "network init");
    }
    *out = nt;
    return CGS_SUCCESS;
}

cgs_status cgs_net_destroy(cgs_net *nt) {
    if (!nt) return CGS_SUCCESS;
    cudaDeviceSynchronize();
    cudaFree(nt->mem);
    delete nt;
    return CGS_SUCCESS;
}

cgs_status cgs_net_get_params(const cgs_net *nt, float *host) {
    if (!nt || !host) return fail(CGS_ERROR_INVALID_VALUE, "network or buffer is null");
    CGS_CUDA(cudaMemcpy(host, nt->params, nt->L.total * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    unsigned int st = 0;
    CGS_CUDA(cudaMemcpy(&st, nt->status, 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (st) return fail(CGS_ERROR_DEVICE_TIMEOUT, "a tensor-core forward pass gave up waiting on its barriers");
    return CGS_SUCCESS;
}

cgs_status cgs_net_set_params(cgs_net *nt, const float *host) {
    if (!nt || !host) return fail(CGS_ERROR_INVALID_VALUE, "network or buffer is null");
    CGS_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    CGS_CUDA(cudaMemcpy(nt->params, host, nt->L.total * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    cgs_status s = sync_bf16(nt, 0);
    if (s != CGS_SUCCESS) return s;
    CGS_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    return CGS_SUCCESS;
}

cgs_status cgs_net_get_grads(const cgs_net *nt, float *host) {
    if (!nt || !host) return fail(CGS_ERROR_INVALID_VALUE, "network or buffer is null");
    CGS_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    CGS_CUDA(cudaMemcpy(host, nt->grads, nt->L.total * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CGS_SUCCESS;
}

cgs_status cgs_net_forward(cgs_net *nt, const float *fixed, const float *moving, int32_t n, int32_t side, float *out,
                           cgs_stream_t stream_) {
    if (!nt || !fixed || !moving) return fail(CGS_ERROR_INVALID_VALUE, "network or images are null");
    if (n < 1 || n > nt->max_batch) return fail(CGS_ERROR_INVALID_VALUE, "batch size out of range");
    if (side < kSide || side % kSide) return fail(CGS_ERROR_INVALID_VALUE, "image side must be a multiple of 128");
    cudaStream_t s = (cudaStream_t)stream_;
    nt->n = n;
    const int64_t tot = (int64_t)n * kSide * kSide;
    input_kernel<<<(int)std::min<int64_t>((tot + 255) / 256, nt->sms * 16), 256, 0, s>>>(fixed, moving, n,
                                                                                          side / kSide, nt->act[0]);
    for (int l = 0; l < kLayers; l++) {
        const ConvGeom g = geom(l, n);
        const int M = n * g.Ho * g.Ho;
        if (nt->conv_mma_sync) {  // the warp-level mma.sync forward, kept for comparison
            conv_fwd_kernel<<<dim3((M + BM - 1) / BM, (g.Cout + BN - 1) / BN), kThreads, 0, s>>>(
                nt->act[l], nt->wb[l], nt->params + nt->L.b[l], nt->act[l + 1], g);
            continue;
        }
        cudaError_t e = launch_conv_umma(false, nt->act[l], nt->wb[l], nt->params + nt->L.b[l], nullptr,
                                         nt->act[l + 1], g, nt->status, s, nt->sms);
        if (e != cudaSuccess) return cuda_fail(e, "conv_umma_kernel (forward)");
    }
    gap_kernel<<<(n * kFeat + 255) / 256, 256, 0, s>>>(nt->act[kLayers], n, nt->feat);
    fc_kernel<<<(n * kHid + 255) / 256, 256, 0, s>>>(nt->feat, nt->params + nt->L.fc1w, nt->params + nt->L.fc1b, n,
                                                     kFeat, kHid, 1, nt->hid);
    fc_kernel<<<(n * kOut + 255) / 256, 256, 0, s>>>(nt->hid, nt->params + nt->L.fc2w, nt->params + nt->L.fc2b, n,
                                                     kHid, kOut, 0, nt->out);
    CGS_CUDA(cudaGetLastError(), "network forward");
    if (out) CGS_CUDA(cudaMemcpyAsync(out, nt->out, (size_t)n * kOut * 4, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
    return CGS_SUCCESS;
}

cgs_status cgs_net_backward(cgs_net *nt, const float *labels, float *loss, cgs_stream_t stream_) {
    if (!nt || !labels) return fail(CGS_ERROR_INVALID_VALUE, "network or labels are null");
    if (nt->n < 1) return fail(CGS_ERROR_INVALID_VALUE, "no forward pass to differentiate");
    cudaStream_t s = (cudaStream_t)stream_;
    const int n = nt->n;
    float *G = nt->grads;
    loss_kernel<<<(n + 127) / 128, 128, 0, s>>>(nt->out, labels, n, nt->dout, nt->lossp);
    // fc2, fc1
    fc_bwd_weight_kernel<<<(kOut * (kHid + 1) + 255) / 256, 256, 0, s>>>(nt->dout, nt->hid, n, kHid, kOut,
                                                                         G + nt->L.fc2w, G + nt->L.fc2b);
    fc_bwd_input_kernel<<<(n * kHid + 255) / 256, 256, 0, s>>>(nt->dout, nt->params + nt->L.fc2w, nt->hid, n, kHid,
                                                               kOut, 1, nt->dhid);
    fc_bwd_weight_kernel<<<(kHid * (kFeat + 1) + 255) / 256, 256, 0, s>>>(nt->dhid, nt->feat, n, kFeat, kHid,
                                                                          G + nt->L.fc1w, G + nt->L.fc1b);
    fc_bwd_input_kernel<<<(n * kFeat + 255) / 256, 256, 0, s>>>(nt->dhid, nt->params + nt->L.fc1w, nt->feat, n,
                                                                kFeat, kHid, 0, nt->dfeat);
    gap_bwd_kernel<<<(n * 16 * kFeat + 255) / 256, 256, 0, s>>>(nt->dfeat, nt->act[kLayers], n, nt->dya);
    bf16 *dy = nt->dya, *dx = nt->dyb;
    for (int l = kLayers - 1; l >= 0; l--) {
        const ConvGeom g = geom(l, n);
        const int64_t wn = (int64_t)g.Cout * g.Kp;
        if (nt->wgrad_mma_sync) {  // the warp-level mma.sync weight gradient, kept for comparison
            int tps;
            const int splits = wgrad_splits(g, nt->sms, &tps);
            conv_bwd_weight_kernel<<<dim3((g.Cout + BM - 1) / BM, (g.Kp + BN - 1) / BN, splits), kThreads, 0, s>>>(
                dy, nt->act[l], nt->ws, g, tps);
            sum_splits_kernel<<<(int)std::min<int64_t>((wn + 255) / 256, 1024), 256, 0, s>>>(nt->ws, splits, wn,
                                                                                              G + nt->L.w[l]);
            const int P = n * g.Ho * g.Ho, chunk = 1024, chunks = (P + chunk - 1) / chunk;
            bias_grad_kernel<<<chunks, 256, 0, s>>>(dy, P, g.Cout, chunk, nt->ws);
            sum_splits_kernel<<<1, 256, 0, s>>>(nt->ws, chunks, g.Cout, G + nt->L.b[l]);
        } else {
            int sps;
            const int splits = wgrad_umma_splits(g, nt->sms, &sps);
            float *partb = nt->ws + (int64_t)splits * wn;
            cudaError_t e = launch_conv_wgrad_umma(dy, nt->act[l], nt->ws, partb, g, splits, sps, nt->status, s);
            if (e != cudaSuccess) return cuda_fail(e, "conv_wgrad_umma_kernel");
            sum_splits_kernel<<<(int)std::min<int64_t>((wn + 255) / 256, 1024), 256, 0, s>>>(nt->ws, splits, wn,
                                                                                              G + nt->L.w[l]);
            sum_splits_kernel<<<(g.Cout + 255) / 256, 256, 0, s>>>(partb, splits, g.Cout, G + nt->L.b[l]);
        }
        if (l > 0) {
            const int Min = n * g.H * g.H;
            if (nt->conv_mma_sync) {  // the warp-level mma.sync data gradient, kept for comparison
                conv_bwd_data_kernel<<<dim3((Min + BM - 1) / BM, (g.Cin + BN - 1) / BN), kThreads, 0, s>>>(
                    dy, nt->wt[l], nt->act[l], dx, g);
            } else {
                cudaError_t e = launch_conv_umma(true, dy, nt->wt[l], nullptr, nt->act[l], dx, g, nt->status, s, nt->sms);
                if (e != cudaSuccess) return cuda_fail(e, "conv_umma_kernel (data gradient)");
            }
            std::swap(dy, dx);
        }
    }
    CGS_CUDA(cudaGetLastError(), "network backward");
    if (loss) {
        sum_splits_kernel<<<1, 32, 0, s>>>(nt->lossp, n, 1, nt->ws);
        CGS_CUDA(cudaMemcpyAsync(loss, nt->ws, 4, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
    }
    return CGS_SUCCESS;
}

cgs_status cgs_net_adam_step(cgs_net *nt, float lr, cgs_stream_t stream_) {
    if (!nt) return fail(CGS_ERROR_INVALID_VALUE, "network is null");
    cudaStream_t s = (cudaStream_t)stream_;
    nt->step++;
    const float c1 = 1.0f / (1.0f - std::pow(0.9f, (float)nt->step));
    const float c2 = 1.0f / (1.0f - std::pow(0.999f, (float)nt->step));
    adam_kernel<<<nt->sms * 8, 256, 0, s>>>(nt->params, nt->grads, nt->m1, nt->m2, nt->L.total, lr, c1, c2);
    CGS_CUDA(cudaGetLastError(), "adam_kernel");
    return sync_bf16(nt, s);
}

}  // extern "C"

extern "C" {

cgs_status cgs_grid_window(const cgs_grid *full, const int32_t first[8], const int32_t count[8], cgs_grid *window) {
    cgs_status s = check_grid(full);
    if (s != CGS_SUCCESS) return s;
    if (!first || !count || !window) return fail(CGS_ERROR_INVALID_VALUE, "first, count or window is null");
    cgs_grid g = *full;
    for (int a = 0; a < full->dims; a++) {
        const float cnt = full->count[a];
        if (cnt != std::floor(cnt)) return fail(CGS_ERROR_INVALID_VALUE, "grid windows need integral counts");
        if (count[a] < 1 || first[a] < 0 || first[a] + count[a] > (int32_t)cnt)
            return fail(CGS_ERROR_INVALID_VALUE, "window outside the grid on axis " + std::to_string(a));
        // the full grid's own decode of the first and last index (CudaGrid::indexToGridPoint)
        g.start[a] = std::fmaf((float)first[a], full->resolution[a], full->start[a]);
        g.end[a] = std::fmaf((float)(first[a] + count[a] - 1), full->resolution[a], full->start[a]);
        g.count[a] = (float)count[a];
    }
    if ((s = cgs_grid_update(&g, -1)) != CGS_SUCCESS) return s;
    *window = g;
    return CGS_SUCCESS;
}

cgs_status cgs_proposal_window(const cgs_grid *full, const float out[16], int32_t min_values, int32_t max_values,
                               int32_t first[8], int32_t count[8]) {
    cgs_status s = check_grid(full);
    if (s != CGS_SUCCESS) return s;
    if (!out || !first || !count) return fail(CGS_ERROR_INVALID_VALUE, "out, first or count is null");
    if (min_values < 1 || max_values > 63 || min_values > max_values || !(min_values & 1) || !(max_values & 1))
        return fail(CGS_ERROR_INVALID_VALUE, "min_values <= max_values, both odd, at most 63");
    for (int a = 0; a < 8; a++) {
        first[a] = 0;
        count[a] = 1;
    }
    for (int a = 0; a < full->dims; a++) {
        const float cnt = full->count[a];
        if (cnt != std::floor(cnt)) return fail(CGS_ERROR_INVALID_VALUE, "proposal windows need integral counts");
        const int nv = (int)cnt;
        count[a] = nv;
        if (nv <= 1) continue;
        const double res = full->resolution[a], range = res * (nv - 1);
        if (!(res > 0.0)) return fail(CGS_ERROR_INVALID_VALUE, "proposal windows need increasing axes");
        const double c = std::isfinite(out[a]) ? std::min(1.0, std::max(-1.0, (double)out[a])) : 0.0;
        const double sr = std::isfinite(out[8 + a]) ? std::min(4.0, std::max(-6.0, (double)out[8 + a])) : 4.0;
        const int ic = (int)std::lround((c + 1.0) * 0.5 * (nv - 1));
        const double radius = std::exp(sr) * 0.5 * range;
        // every grid value within the radius of the centre: |i - ic| <= radius / res + 1/2
        int w = (int)std::floor(radius / res + 0.5);
        w = std::max((min_values - 1) / 2, std::min((max_values - 1) / 2, w));
        int i0 = ic - w, i1 = ic + w;
        if (i0 < 0) { i1 -= i0; i0 = 0; }
        if (i1 > nv - 1) { i0 -= i1 - (nv - 1); i1 = nv - 1; }
        i0 = std::max(i0, 0);
        first[a] = i0;
        count[a] = i1 - i0 + 1;
    }
    return CGS_SUCCESS;
}

}  // extern "C"
