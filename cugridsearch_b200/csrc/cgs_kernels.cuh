// cgs_kernels.cuh -- the fused grid-search kernel (pixel-loop costs) and its helpers.
//
// Layout of the work.  A CTA of NW warps runs persistently over "tasks"; a task is
// NW * G consecutive grid ordinals, G per warp.  Ordinals enumerate the grid in a
// locality order chosen on the host (the axes whose steps move the sampled footprint
// least vary fastest), so the G points of a warp and the NW*G points of a CTA sample
// nearly the same region of the moving image: the moving image is read through L1
// with 4 gathers per sample that mostly hit.  The fixed image streams through shared
// memory in chunks of rows, loaded by bulk (TMA) copies into a 2-stage mbarrier
// pipeline; every warp sweeps the same chunk, each lane owning every 32nd pixel, and
// evaluates all G grid points at that pixel.  Sums are kept per lane in two levels
// (per chunk, then per task) and reduced with warp shuffles; the argmin is fused: a
// 64-bit (cost, index) key per point, warp min, CTA min, one atomicMin per CTA, and
// the last CTA to finish decodes the winner.
//
// Exact decisions, fast samples.  The reference's discrete decisions -- whether a pixel
// maps inside the moving image and, for MI, the histogram bin of each sample -- are
// reproduced bit for bit; the sample VALUES only need FP32 accuracy.  So each pixel is
// mapped with fused multiply-adds and an approximate reciprocal, and a per-grid-point
// error bound (map_guard) says how far that fast coordinate can be from the reference's
// correctly rounded one.  A pixel whose fast coordinate is farther than the bound from
// every decision boundary takes the fast path; the rare rest (a band about a thousandth
// of a pixel wide around the overlap's edge, samples near an MI bin edge, and every
// pixel of an ill-conditioned homography) is recomputed with the reference's exact
// operation sequence.
#pragma once
#include "cgs_device.cuh"
#include "../../include/cugridsearch_b200.h"

namespace cgs {

constexpr int kMaxTrig = 256;
constexpr int kStages = 2;
constexpr uint64_t kWaitLimitNs = 4000000000ull;  // 4 s per bounded wait
constexpr float kMagic = 12582912.0f;            // 1.5 * 2^23: round-down add leaves floor(x) in the mantissa
constexpr int kMagicBits = 0x4B400000;

struct SearchParams {
    // grid: reference decode tables and the evaluation order
    float start[8], res[8];
    int32_t inc[8];      // CudaGrid dimensional increments (int32, reference arithmetic)
    int32_t ocount[8];   // integer count of axis perm[j]
    int32_t perm[8];     // evaluation order, perm[0] varies fastest
    int32_t dims;
    int32_t natural;     // 1: ordinal == grid index (non-integer counts or forced)
    int32_t cost;        // cgs_cost (read by the batch kernel to pick the task body)
    uint32_t n;          // number of grid points
    uint32_t num_tasks;  // tasks of this search; the one that completes the count writes the result
    // images
    Plane mov, fix;
    float mov_wf, mov_hf;
    float cx, cy;        // parametersToHomography centre: (float)W_m / 2, (float)H_m / 2
    int32_t chunk_rows, num_chunks;
    int32_t exact_only;  // 1: every pixel takes the exact path (verification)
    // outputs and scratch
    float *costs;
    unsigned long long *key;
    unsigned int *done;
    unsigned int *status;
    const float *vmax;   // max |moving pixel| (from the staging kernel)
    const float *shifts; // {fixed, moving} image means (staging kernel): the shifts of the ZNCC sums
    cudaTextureObject_t mov_tex;  // the staged moving planes as one (W+1) x C(H+1) texture
    const float4 *mov_quad;       // per channel, W x H taps {(y, x), (y+1, x), (y, x+1) - (y, x), (y+1, x+1) - (y+1, x)}
                                  // (the span kernel's form: PrepParams::quad_form 1, less the moving shift)
    int32_t quad_pitch;           // quads per row
    int64_t quad_plane;           // quads per channel
    const float *row_table;       // calcMIAlt's row values (the float recurrence row += 1/(H_f-1))
    int32_t n_rows;
    cgs_argmin *result;
    // span kernel (cgs_span.cuh): rows per tile, tiles per row and column, 16-byte units per stage
    // (the tile's fixed rows, then its window), window row pitch modulo 8
    int32_t tile_h, tiles_x, tiles_y, win_cap, win_pitch_mod;
    const double2 *fix_prefix;    // span kernel: FP64 {sum f, sum f^2} prefix sums of each fixed row, W + 1 per row
    const float *span_rows;       // MI span kernel: the fixed bins times (B + 1), int32, the fixed plane's pitch
    const float *span_rows_header;  // MI span kernel: the quads' largest slope bound (written by its staging step)
    // cost options
    int32_t mi_bins;
    float gate_n;        // minimum overlap terms for ZNCC / MI
    float total_terms;   // W_f * H_f * C_f
    float2 trig[kMaxTrig];
};

// The span kernel's staging step of one pair, after prep_kernel (cgs_span.cuh).
struct SpanPrepArgs {
    const float *fix;
    int fpitch, fw, fh;
    double2 *prefix;
    int row_blocks;  // blocks [0, row_blocks) write the prefix sums, the others shift the quads
    float4 *quads;
    int64_t nquads;
    const float *shifts;
};

// Launch parameters of the multi-pair span kernel (cgs_span.cuh).
struct SpanBatchParams {
    const SearchParams *pairs;    // [n_pairs], device
    const uint32_t *task_begin;   // [n_pairs + 1]
    const uint32_t *slot;         // [n_pairs]: index of the pair's time stamps
    uint32_t n_pairs, total_tasks;
    unsigned int *next_task;      // zero at launch
    unsigned long long *t_start;  // first task start per slot (atomicMin), or null
    unsigned long long *t_end;    // last task end per slot (atomicMax), or null
    int32_t tile_h, tiles, cap;
};


// ---------------------------------------------------------------- the map of a grid point

// General projective map of fixed pixel (x, y) to moving coordinates, in the reference's
// association: w = ((A*x + B*y) + P) - Q,  X = ((C1*x + C2*y) + R) - S,
// Y = ((D1*x + D2*y) + T) - U,  mx = X / w,  my = Y / w.  It covers
//  * calcNewCoordH's adjugate map (cudaImageFunctions.cuh:277-285),
//  * averageAbsoluteDifferenceH's raw map (cudaErrorFunctions.cuh:205-207): A = H6, B = H7,
//    P = 1 (the +1.0), C1 = H0, C2 = H1, R = H2, D1 = H3, D2 = H4, T = H5, Q = S = U = 0,
//  * the translation of sumOfAbsoluteDifferences (:99-100): w = 1, X = x + tx, Y = y + ty.
// Subtracting a zero and dividing by one are exact, so each form rounds as the reference.
struct MapCoef {
    float A, B, P, Q, C1, C2, R, S, D1, D2, T, U;
};

__device__ __forceinline__ MapCoef coef_from_h(const Homog &h) {
    InvMap m;
    m.set(h);
    return MapCoef{m.A, m.B, m.P, m.Q, m.C1, m.C2, m.R, m.S, m.D1, m.D2, m.T, m.U};
}

template <int COST>
__device__ __forceinline__ MapCoef make_coef(const float *q, float2 cs, const SearchParams &p) {
    if constexpr (COST == CGS_COST_SAD_AVG) {
        return coef_from_h(h_uncentred(q, cs.x, cs.y));
    } else if constexpr (COST == CGS_COST_SAD_AVG_H) {
        return MapCoef{q[6], q[7], 1.0f, 0.0f, q[0], q[1], q[2], 0.0f, q[3], q[4], q[5], 0.0f};
    } else if constexpr (COST == CGS_COST_SAD_SUM_T || COST == CGS_COST_SAD_SUM_T_REF) {
        return MapCoef{0.0f, 0.0f, 1.0f, 0.0f, 1.0f, 0.0f, q[0], 0.0f, 0.0f, 1.0f, q[1], 0.0f};
    } else {
        return coef_from_h(h_centred(q, cs.x, cs.y, p.cx, p.cy));
    }
}

// The reference's correctly rounded coordinates.
__device__ __forceinline__ void exact_map(const MapCoef &k, float x, float y, float &mx, float &my) {
    const float w = xs(xa(xa(xm(k.A, x), xm(k.B, y)), k.P), k.Q);
    const float X = xs(xa(xa(xm(k.C1, x), xm(k.C2, y)), k.R), k.S);
    const float Y = xs(xa(xa(xm(k.D1, x), xm(k.D2, y)), k.T), k.U);
    mx = xd(X, w);
    my = xd(Y, w);
}

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Fast-path state of one grid point (registers).  The per-row terms (B, P - Q, C2, R - S,
// D2, T - U) live in shared memory and are read once per row.
struct FastMap {
    float A, C1, D1;
    float li_x, lo_x, li_y, lo_y;  // |m - half| < li: clearly inside; > lo: clearly outside
};

struct RowTerms {
    float B, PQ, C2, RS, D2, TU;
};

// Error bound of the fast coordinates against the exact ones, over the whole fixed image.
// With u = 2^-24 and M_w = |A|(W_f-1) + |B|(H_f-1) + |P| + |Q| (M_X, M_Y alike), both the
// exact and the fast w lie within 4u*M_w of the real-valued w (standard bounds for a sum of
// four rounded terms), likewise X and Y; the divisions add at most 4u relative (one
// correctly rounded division; one approximate reciprocal of at most 1 ulp plus a rounded
// product).  Hence, for |mx| <= B_x = max(W_m, H_m) + 1, where the in/out decisions lie,
//     |mx_fast - mx_exact| <= 7.2u (M_X + B_x M_w) / w_lo + 4.1u B_x = g_x,
// w_lo being a lower bound of |w| over the image (w is linear: its extremes are at the
// corners).  The guard is twice that.  Beyond B_x the bound grows with slope
// 7.2u M_w / w_lo + 4.1u, which must stay small for "clearly outside" to hold there.  A
// point whose w may change sign over the image, or whose bound is not small, takes the
// exact path everywhere.
__device__ __forceinline__ void map_guard(const MapCoef &k, const SearchParams &p, FastMap &f, RowTerms &rt,
                                          float &gx_out, float &gy_out) {
    f.A = k.A;
    f.C1 = k.C1;
    f.D1 = k.D1;
    rt = RowTerms{k.B, k.P - k.Q, k.C2, k.R - k.S, k.D2, k.T - k.U};
    const double u = 5.9604644775390625e-8;  // 2^-24
    const double X1 = (double)p.fix.w - 1.0, Y1 = (double)p.fix.h - 1.0;
    const double A = k.A, B = k.B, PQ = (double)k.P - (double)k.Q;
    const double Mw = fabs(A) * X1 + fabs(B) * Y1 + fabs((double)k.P) + fabs((double)k.Q);
    const double MX = fabs((double)k.C1) * X1 + fabs((double)k.C2) * Y1 + fabs((double)k.R) + fabs((double)k.S);
    const double MY = fabs((double)k.D1) * X1 + fabs((double)k.D2) * Y1 + fabs((double)k.T) + fabs((double)k.U);
    const double w00 = PQ, w10 = A * X1 + PQ, w01 = B * Y1 + PQ, w11 = A * X1 + B * Y1 + PQ;
    const double wmn = fmin(fmin(w00, w10), fmin(w01, w11));
    const double wmx = fmax(fmax(w00, w10), fmax(w01, w11));
    const double werr = 8.0 * u * Mw;
    bool ok = (wmn > werr) || (wmx < -werr);
    const double wlo = fmin(fabs(wmn), fabs(wmx)) - werr;
    const double Bx = fmax((double)p.mov_wf, (double)p.mov_hf) + 1.0;
    double gx = 0, gy = 0;
    if (ok) {
        const double slope = 7.2 * u * Mw / wlo + 4.1 * u;
        gx = 2.0 * (7.2 * u * (MX + Bx * Mw) / wlo + 4.1 * u * Bx);
        gy = 2.0 * (7.2 * u * (MY + Bx * Mw) / wlo + 4.1 * u * Bx);
        ok = slope < 1e-4 && gx < 0.125 && gy < 0.125;
    }
    const float hw = 0.5f * p.mov_wf, hh = 0.5f * p.mov_hf;
    if (ok && !p.exact_only) {
        f.li_x = (float)((double)hw - gx);
        f.lo_x = (float)((double)hw + gx);
        f.li_y = (float)((double)hh - gy);
        f.lo_y = (float)((double)hh + gy);
    } else {  // never clearly inside, never clearly outside: every pixel goes exact
        f.li_x = f.li_y = -1.0f;
        f.lo_x = f.lo_y = __int_as_float(0x7f800000);
    }
    gx_out = (float)gx;
    gy_out = (float)gy;
}

// ---------------------------------------------------------------- costs

// Accumulators: NA floats per grid point plus an integer term count.
template <int COST> struct AccN { static constexpr int value = 1; };
template <> struct AccN<CGS_COST_SQD_REF> { static constexpr int value = 3; };
template <> struct AccN<CGS_COST_NCC_REF> { static constexpr int value = 3; };
template <> struct AccN<CGS_COST_ZNCC> { static constexpr int value = 5; };
template <> struct AccN<CGS_COST_MI> { static constexpr int value = 1; };

// Zero-mean NCC sums one-pass moments of shifted values f' = f - s_f, m' = m - s_m, the shifts
// being the images' means (from a fixed subsample, computed by the staging kernel); near the data
// the moments cancel little.  FP32 partial sums per lane are reduced and accumulated in FP64, and
// the cost is formed in FP64.  An overlap whose fixed or moving variance is below kZnccDegenerate
// of its sum of squares around the image mean (a constant region: the variance is then below the
// resolution of the FP32 partial sums) has no correlation: +inf.
constexpr double kZnccDegenerate = 1e-6;

// Per-pixel quantities of the fixed value, shared by the G grid points.
struct FixTerms {
    float f;    // fixed value
    float a;    // cost-specific: f/255 (NCC/SQD), f - shift (ZNCC)
    float b;    // cost-specific: (f/255*f)/255 (NCC/SQD), (f - shift)^2 (ZNCC)
    int bin;    // MI: fixed bin
};

template <int COST>
__device__ __forceinline__ FixTerms fix_terms(float f, float sB, int bins, float fshift) {
    FixTerms t;
    t.f = f;
    t.a = 0.0f;
    t.b = 0.0f;
    t.bin = 0;
    if constexpr (COST == CGS_COST_NCC_REF || COST == CGS_COST_SQD_REF) {
        t.a = xd(f, 255.0f);
        t.b = xd(xm(t.a, f), 255.0f);
    } else if constexpr (COST == CGS_COST_ZNCC) {
        t.a = f - fshift;
        t.b = t.a * t.a;
    } else if constexpr (COST == CGS_COST_MI) {
        t.bin = min(max((int)floorf(f * sB), 0), bins - 1);  // sB = bins / 256
    }
    return t;
}

// Accumulate one (fixed, moving value v) term; mshift: the moving shift of ZNCC.
template <int COST>
__device__ __forceinline__ void accumulate(float *a, const FixTerms &t, float v, float mshift) {
    if constexpr (COST == CGS_COST_SAD_AVG || COST == CGS_COST_SAD_AVG_H || COST == CGS_COST_SAD_SUM_T ||
                  COST == CGS_COST_SAD_SUM_T_REF) {
        a[0] += fabsf(v - t.f);
    } else if constexpr (COST == CGS_COST_NCC_REF) {
        // calcNCC: i1 += (f/255*f)/255, i2 += (m/255)^2, ic += (f/255)(m/255)
        const float m = v * (1.0f / 255.0f);
        a[0] += t.b;
        a[1] = fmaf(m, m, a[1]);
        a[2] = fmaf(t.a, m, a[2]);
    } else if constexpr (COST == CGS_COST_SQD_REF) {
        // calcSQD: out += (m/255 - f/255)^2, i1 += (m/255)^2, i2 += (f/255*f)/255
        const float m = v * (1.0f / 255.0f);
        const float d = m - t.a;
        a[0] = fmaf(d, d, a[0]);
        a[1] = fmaf(m, m, a[1]);
        a[2] += t.b;
    } else if constexpr (COST == CGS_COST_ZNCC) {
        const float ms = v - mshift;
        a[0] += t.a;
        a[1] += ms;
        a[2] += t.b;
        a[3] = fmaf(ms, ms, a[3]);
        a[4] = fmaf(t.a, ms, a[4]);
    }
}

// Final cost from the warp-reduced sums (one lane per grid point).
template <int COST>
__device__ __forceinline__ float finalize(const float *a, int n, const SearchParams &p) {
    if constexpr (COST == CGS_COST_SAD_AVG || COST == CGS_COST_SAD_AVG_H) {
        return xd(a[0], (float)n);  // float / int: 0 / 0 is NaN, as in the reference
    } else if constexpr (COST == CGS_COST_SAD_SUM_T || COST == CGS_COST_SAD_SUM_T_REF) {
        return a[0];
    } else if constexpr (COST == CGS_COST_NCC_REF) {
        return n > 0 ? xd(-a[2], sqrtf(xm(a[0], a[1]))) : 0.0f;
    } else if constexpr (COST == CGS_COST_SQD_REF) {
        return n > 0 ? xd(a[0], sqrtf(xm(a[1], a[2]))) : 123123.0f;
    } else {
        return 0.0f;
    }
}

// Zero-mean NCC from the FP64 moments {sum f', sum m', sum f'^2, sum m'^2, sum f'm'} of n terms.
__device__ __forceinline__ float zncc_cost(const double *a, int n, const SearchParams &p) {
    if (n == 0 || (float)n < p.gate_n) return __int_as_float(0x7f800000);
    const double dn = (double)n;
    const double cov = a[4] - a[0] * a[1] / dn;
    const double vf = a[2] - a[0] * a[0] / dn;
    const double vm = a[3] - a[1] * a[1] / dn;
    if (!(vf > kZnccDegenerate * a[2]) || !(vm > kZnccDegenerate * a[3])) return __int_as_float(0x7f800000);
    return (float)(-cov / sqrt(vf * vm));
}

// MI cost of histogram h (B x B counts, row = fixed bin, with a marginal row and column at
// index B; row stride `hstride`) over n terms; one warp, every lane calls it.  The marginals
// are written into h.  The pixel-loop and span kernels share it, so equal counts give equal
// costs.
__device__ __forceinline__ float mi_from_hist(uint32_t *h, int n, int B, int hstride, const SearchParams &p) {
    const int lane = threadIdx.x & 31;
    // marginals: fixed (row sums) into column B, moving (column sums) into row B
    for (int i = lane; i < B; i += 32) {
        uint32_t rs = 0, cs = 0;
        for (int j = 0; j < B; j++) {
            rs += h[i * hstride + j];
            cs += h[j * hstride + i];
        }
        h[i * hstride + B] = rs;
        h[B * hstride + i] = cs;
    }
    __syncwarp();
    const float nf = (float)n;
    float s = 0.0f;
    for (int j = lane; j < B; j += 32) {
        const float hm = (float)h[B * hstride + j];
        for (int i = 0; i < B; i++) {
            const uint32_t v = h[i * hstride + j];
            if (v) {
                const float vf = (float)v;
                const float hf = (float)h[i * hstride + B];
                s += vf * log2f((vf * nf) / (hf * hm));
            }
        }
    }
    s = warp_sum(s);
    return (n == 0 || nf < p.gate_n) ? __int_as_float(0x7f800000) : -s / p.total_terms;
}

// ---------------------------------------------------------------- grid decode// ---------------------------------------------------------------- grid decode

// Ordinal in the evaluation order -> grid index and per-axis indices.
__device__ __forceinline__ uint32_t ordinal_to_index(const SearchParams &p, uint32_t o, int32_t *ax) {
    if (p.natural) {
        int32_t rem = (int32_t)o;
#pragma unroll
        for (int a = 7; a >= 0; a--) {  // indexToGridPoint, cudaGridSearch.cuh:174-180
            if (a < p.dims) {
                ax[a] = rem / p.inc[a];
                rem -= ax[a] * p.inc[a];
            }
        }
        return o;
    }
    uint32_t index = 0;
    int32_t r[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        r[j] = 0;
        if (j < p.dims) {
            const uint32_t c = (uint32_t)p.ocount[j];
            const uint32_t q = o / c;
            r[j] = (int32_t)(o - q * c);
            o = q;
            index += (uint32_t)r[j] * (uint32_t)p.inc[p.perm[j]];
        }
    }
#pragma unroll
    for (int a = 0; a < 8; a++) {
        int32_t v = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) v = (p.perm[j] == a && j < p.dims) ? r[j] : v;
        ax[a] = v;
    }
    return index;
}

// Grid value start + i * res as the reference's device decode forms it (contracted).
__device__ __forceinline__ void grid_values(const SearchParams &p, const int32_t *ax, float *q) {
#pragma unroll
    for (int a = 0; a < 8; a++) q[a] = (a < p.dims) ? __fmaf_rn((float)ax[a], p.res[a], p.start[a]) : 0.0f;
}

// Writes the decoded argmin.  Runs in the last CTA to finish.
static __device__ void write_result(const SearchParams &p) {
    const unsigned long long k = atomicAdd(p.key, 0ull);
    cgs_argmin r;
    r.status = (int32_t)atomicAdd(p.status, 0u);
    clear_verify_fields(r);
#pragma unroll
    for (int a = 0; a < 8; a++) r.params[a] = 0.0f;
    if (k == ~0ull) {
        r.valid = 0;
        r.index = -1;
        r.cost = __int_as_float(0x7f800000);
    } else {
        r.valid = 1;
        const uint32_t idx = (uint32_t)(k & 0xffffffffull);
        r.index = (int64_t)idx;
        r.cost = key_cost(k);
        int32_t ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int32_t rem = (int32_t)idx;
        for (int a = p.dims - 1; a >= 0; a--) {
            ax[a] = rem / p.inc[a];
            rem -= ax[a] * p.inc[a];
        }
        grid_values(p, ax, r.params);
    }
    *p.result = r;
}

// ---------------------------------------------------------------- one task of a persistent CTA

// How a fast-path sample reads its 2x2 taps from the staged moving image: one texture gather,
// four cached scalar loads, or one 16-byte load of the pixel's pre-gathered quad.
enum Taps : int { kTapsTexture = 0, kTapsLoads = 1, kTapsQuad = 2 };

__host__ __device__ constexpr int default_taps(int cost) { return cost == CGS_COST_MI ? kTapsLoads : kTapsTexture; }

// MI bin guard of one grid point: coordinate bounds scaled to bin units (sgx, sgy) and the
// widest fractional tap weight that keeps the sample in its cell (hx, hy).
struct MiGuard {
    float sgx, sgy, hx, hy;
};

// Shared-memory copy of a grid point's exact-path coefficients, guards and row terms.
struct ExactSlot {
    float P, Q, R, S, T, U, gx, gy;
    RowTerms rt;
    float B, C2, D2, pad;
};

// Shared memory of a persistent search CTA: kStages mbarriers, the per-warp argmin keys, the
// abort flag, kStages fixed-image stages, the grid points' exact-path slots [NW][G], the
// per-(warp, point) term counts [NW][G], then the running sums [NW][G][NA][32] or the MI
// histograms ([NW][G] of them when each warp owns its points, [G] when the warps share them).
struct CtaSmem {
    uint64_t *bars;
    unsigned long long *wbest;
    int *abort_flag;
    float *stages;
    int stage_floats;
    ExactSlot *slots;
    int *cnts;
    float *acc;
};

__host__ __device__ constexpr size_t cta_smem_head(int NW) { return 128 + 8 * (size_t)NW; }

// Bytes of dynamic shared memory of a CTA; acc_bytes is the sums or histograms region.
__host__ __device__ constexpr size_t cta_smem_bytes(int G, int NW, size_t stage_bytes, size_t acc_bytes) {
    return cta_smem_head(NW) + kStages * stage_bytes + (size_t)NW * G * (sizeof(ExactSlot) + sizeof(int)) + acc_bytes;
}

template <int G, int NW>
__device__ __forceinline__ CtaSmem carve_smem(unsigned char *smem, int stage_floats) {
    CtaSmem s;
    s.bars = reinterpret_cast<uint64_t *>(smem);
    s.wbest = reinterpret_cast<unsigned long long *>(smem + 64);
    s.abort_flag = reinterpret_cast<int *>(smem + 64 + 8 * NW);
    s.stages = reinterpret_cast<float *>(smem + cta_smem_head(NW));
    s.stage_floats = stage_floats;
    s.slots = reinterpret_cast<ExactSlot *>(s.stages + kStages * stage_floats);
    s.cnts = reinterpret_cast<int *>(s.slots + NW * G);
    s.acc = reinterpret_cast<float *>(s.cnts + NW * G);
    return s;
}

// Bulk copy of chunk `chunk` of a pair's staged fixed image (rows chunk * R ..) into stage
// it % kStages; plane c of the chunk lands at c * R * pitch.  Thread 0 only.
template <int C>
__device__ __forceinline__ void issue_chunk(const SearchParams &p, const CtaSmem &sm, uint32_t it, int chunk) {
    const int R = p.chunk_rows, fpitch = p.fix.pitch;
    const int r0 = chunk * R;
    const int rows = min(R, p.fix.h - r0);
    const uint32_t bytes = (uint32_t)rows * (uint32_t)fpitch * 4u;
    float *dst = sm.stages + (it % kStages) * sm.stage_floats;
    uint64_t *bar = &sm.bars[it % kStages];
    fence_proxy_async_smem();  // the stage's previous reads (generic proxy) before the async refill
    mbar_arrive_expect_tx(bar, bytes * C);
#pragma unroll
    for (int c = 0; c < C; c++)
        bulk_g2s(dst + c * R * fpitch, p.fix.data + c * p.fix.plane + (int64_t)r0 * fpitch, bytes, bar);
}

// Completion of a task (thread 0, after the CTA barrier that follows the task's argmin):
// fold the CTA's key into the pair's, count the task, and let the pair's last task write the
// decoded result.  `tasks` > 1 retires tasks that an aborted CTA will not run.
__device__ __forceinline__ void retire_tasks(const SearchParams &p, unsigned long long key, uint32_t tasks,
                                             bool timed_out) {
    if (key != ~0ull) atomicMin(p.key, key);
    if (timed_out) atomicOr(p.status, (unsigned)CGS_ERROR_DEVICE_TIMEOUT);
    __threadfence();
    const unsigned int old = atomicAdd(p.done, tasks);
    if (old + tasks == p.num_tasks) {
        __threadfence();
        write_result(p);
    }
}

// One task: the G (BSPLIT) or NW * G grid points of ordinals task * points-per-task .., over
// every chunk of the fixed image.
//   BSPLIT = false: warp w owns G consecutive points and sweeps every pixel for them (lane l
//                   takes every 32nd pixel); MI histograms are private to a (warp, point).
//   BSPLIT = true:  the NW warps share G points and split the pixels (lane l of warp w takes
//                   pixels w * 32 + l + k * 32 NW); MI histograms are per (block, point).
// Per-lane partial sums are folded per chunk into shared memory (two-level summation).  With
// BSPLIT = false the summation order of a point does not depend on G or NW, so costs are
// bit-identical across those tunings.  Thread 0 calls prod.after_chunk(it) after each chunk's
// barrier to refill the released stage.  Returns false if a bounded wait gave up (the CTA
// stops; the task is not retired).
template <int COST, int C, int G, int NW, int TAPS, bool BSPLIT, class Prod>
__device__ __forceinline__ bool run_task(const SearchParams &p, uint32_t task, const CtaSmem &sm, uint32_t &it,
                                         Prod &prod) {
    constexpr int NA = AccN<COST>::value;
    constexpr bool kMI = (COST == CGS_COST_MI);
    constexpr bool kZ = (COST == CGS_COST_ZNCC);  // FP64 totals (see kZnccDegenerate)
    constexpr bool kAllPixels = (COST == CGS_COST_SAD_SUM_T_REF);  // outside samples count as 0
    constexpr bool kTexTaps = (TAPS == kTapsTexture);
    constexpr int PSTEP = BSPLIT ? NW * 32 : 32;  // pixel stride of a lane
    constexpr bool kPacked = (G % 2 == 0);         // fast path on pairs of points (FP32x2)
    constexpr int GP = kPacked ? G / 2 : 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int fw = p.fix.w, fh = p.fix.h;
    const int fpitch = p.fix.pitch;
    const int R = p.chunk_rows;
    const int num_chunks = p.num_chunks;
    const int mpitch = p.mov.pitch;
    const int64_t mplane = p.mov.plane;
    const float mrows = (float)(p.mov.h + 1);  // texture rows per plane
    const float *__restrict__ mdata = p.mov.data;
    const cudaTextureObject_t mtex = p.mov_tex;
    const float4 *__restrict__ mquad = p.mov_quad;
    const int qpitch = p.quad_pitch;
    const int64_t qplane = p.quad_plane;
    const float mov_wf = p.mov_wf, mov_hf = p.mov_hf;
    const float hw = 0.5f * mov_wf, hh = 0.5f * mov_hf;
    const int B = p.mi_bins;
    const int hstride = B + 1;            // row stride (bank-conflict padding)
    const int hsize = (B + 1) * (B + 1);  // + a row/column for the marginals
    const float sB = (float)B * (1.0f / 256.0f);
    // value-rounding allowance of the MI bin guard: fast and exact bilinear values of the
    // same coordinates differ by at most 8u * max|v| (bin units, twice for safety)
    const float gv0 = kMI ? sB * 2.0f * 8.0f * 5.9604645e-8f * (*p.vmax) + 1e-6f : 0.0f;

    const uint32_t ord0 = BSPLIT ? task * G : (task * NW + warp) * G;
    const float fshift = kZ ? p.shifts[0] : 0.0f, mshift = kZ ? p.shifts[1] : 0.0f;
    double dz[2] = {0.0, 0.0};  // ZNCC: lane l holds the warp's totals l and l + 32 of index g * NA + j

    FastMap fm[G];
    MiGuard mg[G];  // used by the MI instantiations only
    uint32_t gidx[G];
    bool gvalid[G];
    ExactSlot *my_slots = sm.slots + warp * G;  // BSPLIT: every warp keeps its own copy
#pragma unroll
    for (int g = 0; g < G; g++) {
        const uint32_t o = ord0 + g;
        gvalid[g] = o < p.n;
        int32_t ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        gidx[g] = gvalid[g] ? ordinal_to_index(p, o, ax) : 0u;
        float q[8];
        grid_values(p, ax, q);
        const float2 cs = p.trig[min(ax[0], kMaxTrig - 1)];
        const MapCoef kc = make_coef<COST>(q, cs, p);
        float gx, gy;
        RowTerms rt;
        map_guard(kc, p, fm[g], rt, gx, gy);
        mg[g].sgx = sB * gx;
        mg[g].sgy = sB * gy;
        mg[g].hx = 0.5f - gx;
        mg[g].hy = 0.5f - gy;
        if (lane == 0) my_slots[g] = ExactSlot{kc.P, kc.Q, kc.R, kc.S, kc.T, kc.U, gx, gy, rt, kc.B, kc.C2, kc.D2, 0.0f};
    }

    // packed per-task constants of the fast path (pairs of points)
    float2 A2[GP], C12[GP], D12[GP];
    if constexpr (kPacked) {
#pragma unroll
        for (int h = 0; h < GP; h++) {
            A2[h] = make_float2(fm[2 * h].A, fm[2 * h + 1].A);
            C12[h] = make_float2(fm[2 * h].C1, fm[2 * h + 1].C1);
            D12[h] = make_float2(fm[2 * h].D1, fm[2 * h + 1].D1);
        }
    }
    const float2 nhw2 = make_float2(-hw, -hw), nhh2 = make_float2(-hh, -hh);
    const float2 magic2 = make_float2(kMagic, kMagic), nmagic2 = make_float2(-kMagic, -kMagic);
    const float2 minus1 = make_float2(-1.0f, -1.0f);

    float *tot = sm.acc + warp * G * NA * 32 + lane;
    int cnt[G];
#pragma unroll
    for (int g = 0; g < G; g++) {
        cnt[g] = 0;
        if constexpr (!kMI) {
#pragma unroll
            for (int j = 0; j < NA; j++) tot[(g * NA + j) * 32] = 0.0f;
        }
    }
    uint32_t *hist = reinterpret_cast<uint32_t *>(sm.acc) + (BSPLIT ? 0 : (size_t)warp * G * hsize);
    if constexpr (kMI) {
        if constexpr (BSPLIT) {
            for (int i = threadIdx.x; i < G * hsize; i += NW * 32) hist[i] = 0u;
        } else {
            for (int i = lane; i < G * hsize; i += 32) hist[i] = 0u;
        }
    }
    if constexpr (BSPLIT && kMI) __syncthreads();
    else __syncwarp();

    const int pstart = BSPLIT ? warp * 32 + lane : lane;
    for (int ch = 0; ch < num_chunks; ch++, it++) {
        const int stage = (int)(it % kStages);
        const uint32_t parity = (it / kStages) & 1u;
        if (!mbar_wait_bounded(&sm.bars[stage], parity, kWaitLimitNs)) *sm.abort_flag = 1;
        const float *sfix = sm.stages + stage * sm.stage_floats;
        const int r0 = ch * R;
        const int rows = min(R, fh - r0);

        float part[G][NA];
#pragma unroll
        for (int g = 0; g < G; g++)
#pragma unroll
            for (int j = 0; j < NA; j++) part[g][j] = 0.0f;

        if (p.exact_only) {
            // Exact sampling: coordinates, tap weights and values in the reference's
            // operation order (calcNewCoordH + valueAt_bilinear), so every sample is the
            // reference's bit for bit.  Row products B*y, C2*y, D2*y are formed once per row.
            float ek[G][9];  // A, C1, D1, P, Q, R, S, T, U
#pragma unroll
            for (int g = 0; g < G; g++) {
                const ExactSlot &sl = my_slots[g];
                ek[g][0] = fm[g].A; ek[g][1] = fm[g].C1; ek[g][2] = fm[g].D1;
                ek[g][3] = sl.P; ek[g][4] = sl.Q; ek[g][5] = sl.R; ek[g][6] = sl.S; ek[g][7] = sl.T; ek[g][8] = sl.U;
            }
            int xx = pstart, yy = 0;
            while (xx >= fw) { xx -= fw; yy++; }
            float xf = (float)xx;
            float eb[G][3];
            auto set_row_e = [&](int yrow) {
                const float yf = (float)(r0 + yrow);
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const ExactSlot &sl = my_slots[g];
                    eb[g][0] = xm(sl.B, yf);
                    eb[g][1] = xm(sl.C2, yf);
                    eb[g][2] = xm(sl.D2, yf);
                }
            };
            set_row_e(yy);
            while (yy < rows) {
                FixTerms ft[C];
#pragma unroll
                for (int c = 0; c < C; c++) ft[c] = fix_terms<COST>(sfix[c * R * fpitch + yy * fpitch + xx], sB, B, fshift);
                float ex[G], ey[G];
                bool ins[G];
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const float w = xs(xa(xa(xm(ek[g][0], xf), eb[g][0]), ek[g][3]), ek[g][4]);
                    const float X = xs(xa(xa(xm(ek[g][1], xf), eb[g][1]), ek[g][5]), ek[g][6]);
                    const float Y = xs(xa(xa(xm(ek[g][2], xf), eb[g][2]), ek[g][7]), ek[g][8]);
                    ex[g] = xd(X, w);
                    ey[g] = xd(Y, w);
                    ins[g] = in_image(ey[g], ex[g], mov_wf, mov_hf);
                }
                float v[G][C];
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const float fx = ins[g] ? floorf(ex[g]) : 0.0f, fy = ins[g] ? floorf(ey[g]) : 0.0f;
                    const float ax = xs(ex[g], fx), ay = xs(ey[g], fy);
                    const float omx = xs(1.0f, ax), omy = xs(1.0f, ay);
                    const float u = ins[g] ? fx + 1.0f : -4.0f;
                    const int base = (int)fx + mpitch * (int)fy;
#pragma unroll
                    for (int c = 0; c < C; c++) {
                        float v00, v01, v10, v11;
                        if constexpr (kTexTaps) {
                            const float4 t4 = tex2Dgather<float4>(mtex, u, fy + 1.0f + (float)c * mrows, 0);
                            v00 = t4.w; v01 = t4.z; v10 = t4.x; v11 = t4.y;
                        } else {
                            const float *pl = mdata + c * mplane + base;
                            v00 = __ldg(pl); v01 = __ldg(pl + 1);
                            v10 = __ldg(pl + mpitch); v11 = __ldg(pl + mpitch + 1);
                        }
                        const float top = xa(xm(omx, v00), xm(ax, v01));
                        const float bot = xa(xm(omx, v10), xm(ax, v11));
                        v[g][c] = ins[g] ? xa(xm(omy, top), xm(ay, bot)) : 0.0f;
                    }
                }
#pragma unroll
                for (int g = 0; g < G; g++) {
                    if (ins[g] || kAllPixels) {
#pragma unroll
                        for (int c = 0; c < C; c++) {
                            if constexpr (kMI) {
                                const int bm = min(max((int)floorf(v[g][c] * sB), 0), B - 1);
                                atomicAdd(&hist[g * hsize + ft[c].bin * hstride + bm], 1u);
                            } else {
                                accumulate<COST>(part[g], ft[c], v[g][c], mshift);
                            }
                        }
                        cnt[g] += C;
                    }
                }
                xx += PSTEP;
                xf += (float)PSTEP;
                if (xx >= fw) {
                    do { xx -= fw; yy++; } while (xx >= fw);
                    xf = (float)xx;
                    if (yy < rows) set_row_e(yy);
                }
            }
        } else {
            int xx = pstart, yy = 0;
            while (xx >= fw) { xx -= fw; yy++; }
            float xf = (float)xx;
            // per-row terms of the map; with an even G they are kept as pairs of points for the
            // packed FP32x2 operations below (each component rounds as the scalar operation)
            float byw[G], byx[G], byy[G];
            float2 byw2[GP], byx2[GP], byy2[GP];
            auto set_row = [&](int yrow) {
                const float yf = (float)(r0 + yrow);
                if constexpr (kPacked) {
                    const float2 yf2 = make_float2(yf, yf);
#pragma unroll
                    for (int h = 0; h < GP; h++) {
                        const RowTerms ra = my_slots[2 * h].rt, rb = my_slots[2 * h + 1].rt;
                        byw2[h] = __ffma2_rn(make_float2(ra.B, rb.B), yf2, make_float2(ra.PQ, rb.PQ));
                        byx2[h] = __ffma2_rn(make_float2(ra.C2, rb.C2), yf2, make_float2(ra.RS, rb.RS));
                        byy2[h] = __ffma2_rn(make_float2(ra.D2, rb.D2), yf2, make_float2(ra.TU, rb.TU));
                    }
                } else {
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        const RowTerms rt = my_slots[g].rt;
                        byw[g] = fmaf(rt.B, yf, rt.PQ);
                        byx[g] = fmaf(rt.C2, yf, rt.RS);
                        byy[g] = fmaf(rt.D2, yf, rt.TU);
                    }
                }
            };
            set_row(yy);
            while (yy < rows) {
                FixTerms ft[C];
#pragma unroll
                for (int c = 0; c < C; c++) ft[c] = fix_terms<COST>(sfix[c * R * fpitch + yy * fpitch + xx], sB, B, fshift);
                // 1. fast coordinates, decisions and cell coordinates of all G points
                //    (independent chains): tx = floor + 1.5 * 2^23 (round-down add), fx = floor,
                //    ax = fraction
                bool fin[G], amb[G];
                float mxs[G], mys[G], txs[G], tys[G], fxs[G], fys[G], axs[G], ays[G];
                auto decide = [&](int g, float dx, float dy) {
                    fin[g] = (dx < fm[g].li_x) & (dy < fm[g].li_y);              // clearly inside
                    amb[g] = !fin[g] & !((dx > fm[g].lo_x) | (dy > fm[g].lo_y)); // undecided: exact path
                };
                if constexpr (kPacked) {
                    const float2 xf2 = make_float2(xf, xf);
#pragma unroll
                    for (int h = 0; h < GP; h++) {
                        const int g = 2 * h;
                        const float2 w = __ffma2_rn(A2[h], xf2, byw2[h]);
                        const float2 X = __ffma2_rn(C12[h], xf2, byx2[h]);
                        const float2 Y = __ffma2_rn(D12[h], xf2, byy2[h]);
                        const float2 rw = make_float2(rcp_approx(w.x), rcp_approx(w.y));
                        const float2 mx = __fmul2_rn(X, rw), my = __fmul2_rn(Y, rw);
                        const float2 dx = __fadd2_rn(mx, nhw2), dy = __fadd2_rn(my, nhh2);
                        decide(g, fabsf(dx.x), fabsf(dy.x));
                        decide(g + 1, fabsf(dx.y), fabsf(dy.y));
                        const float2 tx = __fadd2_rd(mx, magic2), ty = __fadd2_rd(my, magic2);
                        const float2 fx = __fadd2_rn(tx, nmagic2), fy = __fadd2_rn(ty, nmagic2);
                        const float2 ax = __ffma2_rn(fx, minus1, mx), ay = __ffma2_rn(fy, minus1, my);
                        mxs[g] = mx.x; mxs[g + 1] = mx.y; mys[g] = my.x; mys[g + 1] = my.y;
                        txs[g] = tx.x; txs[g + 1] = tx.y; tys[g] = ty.x; tys[g + 1] = ty.y;
                        fxs[g] = fx.x; fxs[g + 1] = fx.y; fys[g] = fy.x; fys[g + 1] = fy.y;
                        axs[g] = ax.x; axs[g + 1] = ax.y; ays[g] = ay.x; ays[g + 1] = ay.y;
                    }
                } else {
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        const float w = fmaf(fm[g].A, xf, byw[g]);
                        const float X = fmaf(fm[g].C1, xf, byx[g]);
                        const float Y = fmaf(fm[g].D1, xf, byy[g]);
                        const float rw = rcp_approx(w);
                        mxs[g] = X * rw;
                        mys[g] = Y * rw;
                        decide(g, fabsf(mxs[g] - hw), fabsf(mys[g] - hh));
                        txs[g] = __fadd_rd(mxs[g], kMagic);
                        tys[g] = __fadd_rd(mys[g], kMagic);
                        fxs[g] = txs[g] - kMagic;
                        fys[g] = tys[g] - kMagic;
                        axs[g] = mxs[g] - fxs[g];
                        ays[g] = mys[g] - fys[g];
                    }
                }
                // 2. taps of all G points.  Texture: one gather returns the 2x2 footprint; the
                //    gather coordinate is the footprint's centre, (floor + 1) in texel units, so
                //    the texture unit's fixed-point coordinate rounding cannot change the cell;
                //    points not clearly inside read zeros from the border.  Quads: one 16-byte
                //    load of the footprint (points not clearly inside read quad 0, unused).
                float v[G][C];
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const float tx = txs[g], ty = tys[g], fx = fxs[g], fy = fys[g], ax = axs[g], ay = ays[g];
                    const float u = fin[g] ? fx + 1.0f : -4.0f;
                    const int ix = __float_as_int(tx) - kMagicBits, iy = __float_as_int(ty) - kMagicBits;
                    const int base = fin[g] ? ix + mpitch * iy : 0;
                    const int qbase = fin[g] ? ix + qpitch * iy : 0;
#pragma unroll
                    for (int c = 0; c < C; c++) {
                        float v00, v01, v10, v11, d0, d1, dy;  // dy: bound of the column differences
                        if constexpr (TAPS == kTapsQuad) {
                            // quad = {left column (v00, v10), its differences to the right column
                            // (v01 - v00, v11 - v10), rounded once as here}: the two row lerps as
                            // one packed pair
                            const float4 q4 = __ldg(mquad + c * qplane + qbase);
                            v00 = q4.x; v10 = q4.y; d0 = q4.z; d1 = q4.w;
                            const float2 left = make_float2(q4.x, q4.y), dd = make_float2(q4.z, q4.w);
                            const float2 tb = __ffma2_rn(make_float2(ax, ax), dd, left);  // (top, bottom)
                            v[g][c] = fmaf(ay, tb.y - tb.x, tb.x);
                            if constexpr (kMI) {
                                // |v11 - v01| <= |v10 - v00| + |v11 - v10| + |v01 - v00|; the factor
                                // covers the roundings of the differences and of this sum
                                dy = (fabsf(v10 - v00) + fabsf(d0) + fabsf(d1)) * (1.0f + 0x1p-20f);
                            }
                        } else {
                            if constexpr (kTexTaps) {
                                const float4 t4 = tex2Dgather<float4>(mtex, u, fy + 1.0f + (float)c * mrows, 0);
                                // gather order: x = (i0, j1), y = (i1, j1), z = (i1, j0), w = (i0, j0)
                                v00 = t4.w; v01 = t4.z; v10 = t4.x; v11 = t4.y;
                            } else {
                                const float *pl = mdata + c * mplane + base;
                                v00 = __ldg(pl); v01 = __ldg(pl + 1);
                                v10 = __ldg(pl + mpitch); v11 = __ldg(pl + mpitch + 1);
                            }
                            d0 = v01 - v00;
                            d1 = v11 - v10;
                            const float top = fmaf(ax, d0, v00), bot = fmaf(ax, d1, v10);
                            v[g][c] = fmaf(ay, bot - top, top);
                            if constexpr (kMI) dy = fmaxf(fabsf(v10 - v00), fabsf(v11 - v01));
                        }
                        if constexpr (kMI) {
                            // the bin is exact unless the sample could lie across a bin edge (or the
                            // coordinate across a cell edge) from the reference's sample
                            const float t = v[g][c] * sB;
                            const float fr = t - floorf(t);
                            const float Dx = fmaxf(fabsf(d0), fabsf(d1));
                            const float gb = fmaf(dy, mg[g].sgy, fmaf(Dx, mg[g].sgx, gv0));
                            const bool near = (fabsf(fr - 0.5f) > 0.5f - gb) | (fabsf(ax - 0.5f) > mg[g].hx) |
                                              (fabsf(ay - 0.5f) > mg[g].hy);
                            if (fin[g] & near) {
                                fin[g] = false;
                                amb[g] = true;
                            }
                        }
                    }
                }
                // 3. rare: undecided points through the reference's exact operation sequence
                bool any_amb = false;
#pragma unroll
                for (int g = 0; g < G; g++) any_amb |= amb[g];
                if (any_amb) {
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        if (amb[g]) {
                            const ExactSlot &sl = my_slots[g];
                            const MapCoef kc{fm[g].A, sl.B, sl.P, sl.Q, fm[g].C1, sl.C2, sl.R, sl.S,
                                             fm[g].D1, sl.D2, sl.T, sl.U};
                            float ex, ey;
                            exact_map(kc, xf, (float)(r0 + yy), ex, ey);
                            if (in_image(ey, ex, mov_wf, mov_hf)) {
                                fin[g] = true;
#pragma unroll
                                for (int c = 0; c < C; c++) v[g][c] = bilinear_in(mdata + c * mplane, mpitch, ey, ex);
                            }
                        }
                    }
                }
                // 4. accumulate (predicated)
#pragma unroll
                for (int g = 0; g < G; g++) {
                    if (fin[g]) {
#pragma unroll
                        for (int c = 0; c < C; c++) {
                            if constexpr (kMI) {
                                const int bm = min(max((int)floorf(v[g][c] * sB), 0), B - 1);
                                atomicAdd(&hist[g * hsize + ft[c].bin * hstride + bm], 1u);
                            } else {
                                accumulate<COST>(part[g], ft[c], v[g][c], mshift);
                            }
                        }
                        cnt[g] += C;
                    } else if constexpr (kAllPixels) {
#pragma unroll
                        for (int c = 0; c < C; c++) accumulate<COST>(part[g], ft[c], 0.0f, mshift);
                        cnt[g] += C;
                    }
                }
                xx += PSTEP;
                xf += (float)PSTEP;
                if (xx >= fw) {
                    do { xx -= fw; yy++; } while (xx >= fw);
                    xf = (float)xx;
                    if (yy < rows) set_row(yy);
                }
            }
        }  // fast sampling
        if constexpr (kZ) {
            // the chunk's warp sums into the FP64 totals
#pragma unroll
            for (int g = 0; g < G; g++)
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    const float sw = warp_sum(part[g][j]);
                    const int idx = g * NA + j;
                    if (lane == (idx & 31)) dz[idx >> 5] += (double)sw;
                }
        } else if constexpr (!kMI) {
#pragma unroll
            for (int g = 0; g < G; g++)
#pragma unroll
                for (int j = 0; j < NA; j++) tot[(g * NA + j) * 32] += part[g][j];
        }

        __syncthreads();
        if (*sm.abort_flag) return false;
        if (threadIdx.x == 0) prod.after_chunk(it);
    }

    // ---- per grid point: reduce, finalise, dump, argmin key ----
    auto mi_cost = [&](uint32_t *h, int n) -> float { return mi_from_hist(h, n, B, hstride, p); };

    unsigned long long kk = ~0ull;
    if constexpr (!BSPLIT) {
        float my_cost = 0.0f;
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int n = warp_sum_i(cnt[g]);
            float cost;
            if constexpr (kMI) {
                __syncwarp();
                cost = mi_cost(hist + g * hsize, n);
            } else if constexpr (kZ) {
                double a[NA];
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    const int idx = g * NA + j;
                    a[j] = __shfl_sync(0xffffffffu, dz[idx >> 5], idx & 31);
                }
                cost = zncc_cost(a, n, p);
            } else {
                float a[NA];
#pragma unroll
                for (int j = 0; j < NA; j++) a[j] = warp_sum(tot[(g * NA + j) * 32]);
                cost = finalize<COST>(a, n, p);
            }
            if (lane == g) my_cost = cost;
        }
        // lanes 0..G-1 hold the costs of the warp's points
        if (lane < G) {
            bool valid = false;
            uint32_t idx = 0;
#pragma unroll
            for (int g = 0; g < G; g++)
                if (lane == g) { valid = gvalid[g]; idx = gidx[g]; }
            if (valid) {
                if (p.costs) p.costs[idx] = my_cost;
                kk = make_key(my_cost, idx);
            }
        }
    } else {
        // the warps' counts, then warp g (mod NW) finalises point g from every warp's sums
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int n = warp_sum_i(cnt[g]);
            if (lane == 0) sm.cnts[warp * G + g] = n;
        }
        double *dacc = reinterpret_cast<double *>(sm.acc);  // ZNCC: [NW][G * NA] FP64 totals
        if constexpr (kZ) {
#pragma unroll
            for (int i = 0; i < G * NA; i++)
                if (lane == (i & 31)) dacc[warp * G * NA + i] = dz[i >> 5];
        }
        __syncthreads();
#pragma unroll
        for (int g = 0; g < G; g++) {
            if (g % NW != warp) continue;
            int n = 0;
            for (int w = 0; w < NW; w++) n += sm.cnts[w * G + g];
            float cost;
            if constexpr (kMI) {
                cost = mi_cost(hist + g * hsize, n);
            } else if constexpr (kZ) {
                double a[NA];
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    double v = 0.0;
                    for (int w = 0; w < NW; w++) v += dacc[w * G * NA + g * NA + j];
                    a[j] = v;
                }
                cost = zncc_cost(a, n, p);
            } else {
                float a[NA];
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    float v = 0.0f;
                    for (int w = 0; w < NW; w++) v += sm.acc[(w * G + g) * NA * 32 + j * 32 + lane];
                    a[j] = warp_sum(v);
                }
                cost = finalize<COST>(a, n, p);
            }
            if (lane == 0 && gvalid[g]) {
                if (p.costs) p.costs[gidx[g]] = cost;
                const unsigned long long k = make_key(cost, gidx[g]);
                kk = k < kk ? k : kk;
            }
        }
    }
    kk = warp_min_u64(kk);
    if (lane == 0) sm.wbest[warp] = kk;
    __syncthreads();  // keys complete; slots, sums and histograms are free for the next task
    if (threadIdx.x == 0) {
        unsigned long long b = ~0ull;
        for (int w = 0; w < NW; w++) b = sm.wbest[w] < b ? sm.wbest[w] : b;
        retire_tasks(p, b, 1u, false);
    }
    return true;
}

// ---------------------------------------------------------------- the single-pair kernel

// Producer of the single-pair kernel: the CTA's tasks are blockIdx.x + k * gridDim.x, each
// with the pair's num_chunks chunks, so iteration `it` is chunk it % num_chunks.
template <int C>
struct StaticProducer {
    const SearchParams *p;
    const CtaSmem *sm;
    uint32_t total_it;
    __device__ __forceinline__ void issue(uint32_t it) {
        issue_chunk<C>(*p, *sm, it, (int)(it % (uint32_t)p->num_chunks));
    }
    __device__ __forceinline__ void after_chunk(uint32_t it) {
        if (it + kStages < total_it) issue(it + kStages);
    }
};

// NW warps per CTA; 512 / (32 NW) CTAs share an SM (two CTAs of 8 warps hide each
// other's chunk barriers).  Tasks are dealt round-robin over the persistent CTAs.
template <int COST, int C, int G, int NW, int TAPS = default_taps(COST)>
__global__ void __launch_bounds__(NW * 32, 16 / NW) search_kernel(const __grid_constant__ SearchParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const CtaSmem sm = carve_smem<G, NW>(smem, p.chunk_rows * p.fix.pitch * C);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(&sm.bars[s], 1);
        fence_mbar_init();
        *sm.abort_flag = 0;
    }
    __syncthreads();

    const uint32_t my_tasks =
        (p.num_tasks > blockIdx.x) ? (p.num_tasks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    StaticProducer<C> prod{&p, &sm, my_tasks * (uint32_t)p.num_chunks};
    if (threadIdx.x == 0) {
        for (uint32_t it = 0; it < (uint32_t)kStages && it < prod.total_it; it++) prod.issue(it);
    }

    uint32_t it = 0;
    for (uint32_t k = 0; k < my_tasks; k++) {
        if (!run_task<COST, C, G, NW, TAPS, false>(p, blockIdx.x + k * gridDim.x, sm, it, prod)) {
            // a bounded wait gave up: retire this CTA's remaining tasks with the timeout status
            if (threadIdx.x == 0) retire_tasks(p, ~0ull, my_tasks - k, true);
            return;
        }
    }
}

}  // namespace cgs
