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
#pragma once
#include "cgs_device.cuh"
#include "../../include/cugridsearch_b200.h"

namespace cgs {

constexpr int kMaxTrig = 256;
constexpr int kStages = 2;
constexpr uint64_t kWaitLimitNs = 4000000000ull;  // 4 s per bounded wait

struct SearchParams {
    // grid: reference decode tables and the evaluation order
    float start[8], res[8];
    int32_t inc[8];      // CudaGrid dimensional increments (int32, reference arithmetic)
    int32_t ocount[8];   // integer count of axis perm[j]
    int32_t perm[8];     // evaluation order, perm[0] varies fastest
    int32_t dims;
    int32_t natural;     // 1: ordinal == grid index (non-integer counts or forced)
    uint32_t n;          // number of grid points
    uint32_t num_tasks;
    // images
    Plane mov, fix;
    float mov_wf, mov_hf;
    float cx, cy;        // parametersToHomography centre: (float)W_m / 2, (float)H_m / 2
    int32_t chunk_rows, num_chunks;
    // outputs and scratch
    float *costs;
    unsigned long long *key;
    unsigned int *done;
    unsigned int *status;
    cgs_argmin *result;
    // cost options
    int32_t mi_bins;
    float gate_n;        // minimum overlap terms for ZNCC / MI
    float total_terms;   // W_f * H_f * C_f
    float2 trig[kMaxTrig];
};

// Per-grid-point state of each cost family.
template <int COST>
struct Mapper;

template <>
struct Mapper<CGS_COST_SAD_AVG> {
    InvMap m;
    __device__ void set(const float *q, float2 cs, const SearchParams &) { m.set(h_uncentred(q, cs.x, cs.y)); }
    __device__ __forceinline__ void map(float x, float y, float &mx, float &my) const { m.map(x, y, mx, my); }
};
template <>
struct Mapper<CGS_COST_SAD_AVG_H> {
    RawMap m;
    __device__ void set(const float *q, float2, const SearchParams &) {
#pragma unroll
        for (int i = 0; i < 8; i++) m.H[i] = q[i];
    }
    __device__ __forceinline__ void map(float x, float y, float &mx, float &my) const { m.map(x, y, mx, my); }
};
struct ShiftMap {
    float tx, ty;
    __device__ void set(const float *q, float2, const SearchParams &) { tx = q[0]; ty = q[1]; }
    __device__ __forceinline__ void map(float x, float y, float &mx, float &my) const {
        mx = xa(x, tx);
        my = xa(y, ty);
    }
};
template <> struct Mapper<CGS_COST_SAD_SUM_T> : ShiftMap {};
template <> struct Mapper<CGS_COST_SAD_SUM_T_REF> : ShiftMap {};
struct CentredMap {
    InvMap m;
    __device__ void set(const float *q, float2 cs, const SearchParams &p) { m.set(h_centred(q, cs.x, cs.y, p.cx, p.cy)); }
    __device__ __forceinline__ void map(float x, float y, float &mx, float &my) const { m.map(x, y, mx, my); }
};
template <> struct Mapper<CGS_COST_SQD_REF> : CentredMap {};
template <> struct Mapper<CGS_COST_NCC_REF> : CentredMap {};
template <> struct Mapper<CGS_COST_ZNCC> : CentredMap {};
template <> struct Mapper<CGS_COST_MI> : CentredMap {};

// Accumulators: NA floats per grid point plus an integer term count.
template <int COST> struct AccN { static constexpr int value = 1; };
template <> struct AccN<CGS_COST_SQD_REF> { static constexpr int value = 3; };
template <> struct AccN<CGS_COST_NCC_REF> { static constexpr int value = 3; };
template <> struct AccN<CGS_COST_ZNCC> { static constexpr int value = 5; };
template <> struct AccN<CGS_COST_MI> { static constexpr int value = 0; };

constexpr float kZnccShift = 127.5f;  // centre of the [0, 255] range: keeps the one-pass
                                      // variance sums well conditioned

// Accumulate one (fixed value f, moving value v) term.
template <int COST>
__device__ __forceinline__ void accumulate(float *a, float f, float v) {
    if constexpr (COST == CGS_COST_SAD_AVG || COST == CGS_COST_SAD_AVG_H || COST == CGS_COST_SAD_SUM_T ||
                  COST == CGS_COST_SAD_SUM_T_REF) {
        a[0] += fabsf(xs(v, f));  // |m - f| exactly as the reference forms it
    } else if constexpr (COST == CGS_COST_NCC_REF) {
        // calcNCC: i1 += (f/255*f)/255, i2 += t*t, ic += (f/255)*t with t = m/255
        const float t = xd(v, 255.0f);
        const float fn = xd(f, 255.0f);
        a[0] += xd(xm(fn, f), 255.0f);
        a[1] = fmaf(t, t, a[1]);
        a[2] = fmaf(fn, t, a[2]);
    } else if constexpr (COST == CGS_COST_SQD_REF) {
        // calcSQD: out += (t - f/255)^2, i1 += t*t, i2 += (f/255*f)/255
        const float t = xd(v, 255.0f);
        const float fn = xd(f, 255.0f);
        const float d = xs(t, fn);
        a[0] = fmaf(d, d, a[0]);
        a[1] = fmaf(t, t, a[1]);
        a[2] += xd(xm(fn, f), 255.0f);
    } else if constexpr (COST == CGS_COST_ZNCC) {
        const float fs = f - kZnccShift, ms = v - kZnccShift;
        a[0] += fs;
        a[1] += ms;
        a[2] = fmaf(fs, fs, a[2]);
        a[3] = fmaf(ms, ms, a[3]);
        a[4] = fmaf(fs, ms, a[4]);
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
    } else if constexpr (COST == CGS_COST_ZNCC) {
        if (n == 0 || (float)n < p.gate_n) return __int_as_float(0x7f800000);
        const float dn = (float)n;
        const float cov = a[4] - a[0] * a[1] / dn;
        const float vf = a[2] - a[0] * a[0] / dn;
        const float vm = a[3] - a[1] * a[1] / dn;
        if (!(vf > 0.0f) || !(vm > 0.0f)) return __int_as_float(0x7f800000);
        return -cov / sqrtf(vf * vm);
    } else {
        return 0.0f;
    }
}

// Ordinal in the evaluation order -> grid index and per-axis indices.
__device__ __forceinline__ uint32_t ordinal_to_index(const SearchParams &p, uint32_t o, int32_t *ax) {
    if (p.natural) {
        int32_t rem = (int32_t)o;
        for (int a = p.dims - 1; a >= 0; a--) {  // indexToGridPoint, cudaGridSearch.cuh:174-180
            ax[a] = rem / p.inc[a];
            rem -= ax[a] * p.inc[a];
        }
        return o;
    }
    uint32_t index = 0;
    for (int j = 0; j < p.dims; j++) {
        const int a = p.perm[j];
        const uint32_t c = (uint32_t)p.ocount[j];
        const uint32_t q = o / c;
        const uint32_t r = o - q * c;
        o = q;
        ax[a] = (int32_t)r;
        index += r * (uint32_t)p.inc[a];
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
    r.reserved = 0;
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

template <int COST, int C, int G, int NW>
__global__ void __launch_bounds__(NW * 32, 1) search_kernel(const __grid_constant__ SearchParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int NA = AccN<COST>::value;
    constexpr bool kMI = (COST == CGS_COST_MI);

    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    unsigned long long *wbest = reinterpret_cast<unsigned long long *>(smem + 64);
    int *abort_flag = reinterpret_cast<int *>(smem + 64 + 8 * NW);
    float *stages = reinterpret_cast<float *>(smem + 128 + 8 * NW);
    const int fpitch = p.fix.pitch;
    const int R = p.chunk_rows;
    const int stage_floats = R * fpitch * C;
    uint32_t *hist_base = reinterpret_cast<uint32_t *>(stages + kStages * stage_floats);
    const int B = p.mi_bins;
    const int hstride = B + 1;                 // row stride (bank-conflict padding)
    const int hsize = (B + 1) * (B + 1);       // + a row/column for the marginals

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int fw = p.fix.w, fh = p.fix.h;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(&bars[s], 1);
        fence_mbar_init();
        *abort_flag = 0;
    }
    __syncthreads();

    const uint32_t my_tasks =
        (p.num_tasks > blockIdx.x) ? (p.num_tasks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    const uint32_t total_it = my_tasks * (uint32_t)p.num_chunks;

    auto issue = [&](uint32_t it) {
        const int chunk = (int)(it % (uint32_t)p.num_chunks);
        const int r0 = chunk * R;
        const int rows = min(R, fh - r0);
        const uint32_t bytes = (uint32_t)rows * (uint32_t)fpitch * 4u;
        float *dst = stages + (it % kStages) * stage_floats;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bars[it % kStages], bytes * C);
#pragma unroll
        for (int c = 0; c < C; c++)
            bulk_g2s(dst + c * R * fpitch, p.fix.data + c * p.fix.plane + (int64_t)r0 * fpitch, bytes,
                     &bars[it % kStages]);
    };

    if (threadIdx.x == 0) {
        for (uint32_t it = 0; it < (uint32_t)kStages && it < total_it; it++) issue(it);
    }

    unsigned long long best = ~0ull;
    uint32_t it = 0;
    bool aborted = false;

    for (uint32_t k = 0; k < my_tasks && !aborted; k++) {
        const uint32_t task = blockIdx.x + k * gridDim.x;
        const uint32_t ord0 = (task * NW + warp) * G;

        Mapper<COST> mp[G];
        uint32_t gidx[G];
        bool gvalid[G];
#pragma unroll
        for (int g = 0; g < G; g++) {
            const uint32_t o = ord0 + g;
            gvalid[g] = o < p.n;
            int32_t ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            gidx[g] = gvalid[g] ? ordinal_to_index(p, o, ax) : 0u;
            float q[8];
            grid_values(p, ax, q);
            const float2 cs = p.trig[min(ax[0], kMaxTrig - 1)];
            mp[g].set(q, cs, p);
        }

        float acc[G][NA > 0 ? NA : 1];
        int cnt[G];
#pragma unroll
        for (int g = 0; g < G; g++) {
            cnt[g] = 0;
#pragma unroll
            for (int j = 0; j < (NA > 0 ? NA : 1); j++) acc[g][j] = 0.0f;
        }
        uint32_t *hist = hist_base + (size_t)warp * G * hsize;
        if constexpr (kMI) {
            for (int i = lane; i < G * hsize; i += 32) hist[i] = 0u;
            __syncwarp();
        }

        for (int ch = 0; ch < p.num_chunks; ch++, it++) {
            const int stage = (int)(it % kStages);
            const uint32_t parity = (it / kStages) & 1u;
            if (!mbar_wait_bounded(&bars[stage], parity, kWaitLimitNs)) *abort_flag = 1;
            const float *sfix = stages + stage * stage_floats;
            const int r0 = ch * R;
            const int rows = min(R, fh - r0);

            float part[G][NA > 0 ? NA : 1];
#pragma unroll
            for (int g = 0; g < G; g++)
#pragma unroll
                for (int j = 0; j < (NA > 0 ? NA : 1); j++) part[g][j] = 0.0f;

            int xx = lane, yy = 0;
            while (xx >= fw) { xx -= fw; yy++; }
            while (yy < rows) {
                const float xf = (float)xx, yf = (float)(r0 + yy);
                float fv[C];
#pragma unroll
                for (int c = 0; c < C; c++) fv[c] = sfix[c * R * fpitch + yy * fpitch + xx];
#pragma unroll
                for (int g = 0; g < G; g++) {
                    float mx, my;
                    mp[g].map(xf, yf, mx, my);
                    const bool inside = in_image(my, mx, p.mov_wf, p.mov_hf);
                    if constexpr (COST == CGS_COST_SAD_SUM_T_REF) {
                        // by-reference SAD: every pixel counts, outside samples read 0
#pragma unroll
                        for (int c = 0; c < C; c++) {
                            const float v = inside ? bilinear_in(p.mov.data + c * p.mov.plane, p.mov.w, my, mx) : 0.0f;
                            accumulate<COST>(part[g], fv[c], v);
                        }
                        cnt[g] += C;
                    } else if (inside) {
#pragma unroll
                        for (int c = 0; c < C; c++) {
                            const float v = bilinear_in(p.mov.data + c * p.mov.plane, p.mov.w, my, mx);
                            if constexpr (kMI) {
                                const float bs = (float)B * (1.0f / 256.0f);
                                int bf = (int)floorf(fv[c] * bs), bm = (int)floorf(v * bs);
                                bf = min(max(bf, 0), B - 1);
                                bm = min(max(bm, 0), B - 1);
                                atomicAdd(&hist[g * hsize + bf * hstride + bm], 1u);
                            } else {
                                accumulate<COST>(part[g], fv[c], v);
                            }
                        }
                        cnt[g] += C;
                    }
                }
                xx += 32;
                while (xx >= fw) { xx -= fw; yy++; }
            }
#pragma unroll
            for (int g = 0; g < G; g++)
#pragma unroll
                for (int j = 0; j < NA; j++) acc[g][j] += part[g][j];

            __syncthreads();
            if (*abort_flag) {
                aborted = true;
                break;
            }
            if (threadIdx.x == 0 && it + kStages < total_it) issue(it + kStages);
        }
        if (aborted) break;

        // ---- per grid point: reduce, finalise, dump, argmin ----
        float my_cost = 0.0f;
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int n = warp_sum_i(cnt[g]);
            float cost;
            if constexpr (kMI) {
                __syncwarp();
                uint32_t *h = hist + g * hsize;
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
                cost = (n == 0 || nf < p.gate_n) ? __int_as_float(0x7f800000) : -s / p.total_terms;
            } else {
                float a[NA];
#pragma unroll
                for (int j = 0; j < NA; j++) a[j] = warp_sum(acc[g][j]);
                cost = finalize<COST>(a, n, p);
            }
            if (lane == g) my_cost = cost;
        }
        // lanes 0..G-1 hold the costs of the warp's points
        unsigned long long kk = ~0ull;
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
        kk = warp_min_u64(kk);
        best = kk < best ? kk : best;
    }

    // ---- CTA argmin, one atomic per CTA, last CTA writes the result ----
    if (lane == 0) wbest[warp] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long b = ~0ull;
        for (int w = 0; w < NW; w++) b = wbest[w] < b ? wbest[w] : b;
        if (b != ~0ull) atomicMin(p.key, b);
        if (*abort_flag) atomicOr(p.status, (unsigned)CGS_ERROR_DEVICE_TIMEOUT);
        __threadfence();
        const unsigned int ticket = atomicAdd(p.done, 1u);
        if (ticket == gridDim.x - 1) {
            __threadfence();
            write_result(p);
        }
    }
}

}  // namespace cgs
