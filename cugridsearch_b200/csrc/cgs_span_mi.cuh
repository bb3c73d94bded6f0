// cgs_span_mi.cuh -- the span kernel for mutual information: exact joint-histogram counts over
// fast samples, with the in/out decisions taken per image row.
//
// Decisions per row as in the zero-mean NCC span kernel (cgs_span.cuh): per (row, point) an
// inner span (inside for the reference too, no test), an outer span, and the band between them
// sampled with the reference's exact operation sequence in the span pass.
//
// Bins.  Every fast sample inside the inner span is interpolated from its quad (the bilinear
// polynomial's coefficients, three FMAs) and binned, floor(B v / 256) clamped to [0, B).  The
// bin is the reference's unless the sample may lie across a bin edge from the reference's
// sample: its distance to the nearest edge (0 and B excepted: the bin is clamped there) is below
// the bound on their difference, the fast coordinates' guard g times the interpolant's slopes
// plus the rounding of both interpolations.  The slopes are the quad's own (3|c10| + |c01| +
// 2|c11| bounds both partial derivatives' sum in the cell) unless the coordinates lie within g of
// a cell edge: the reference may then interpolate the neighbouring cell, and since the bilinear
// interpolant is continuous across the edge the image's largest such slope (span_prep_mi_kernel)
// bounds the difference instead.  Undecided samples are queued per warp and re-sampled with the
// reference's exact sequence by all 32 lanes at once when the queue fills and at the end of each
// band of rows, so the counts are exactly the reference's.
//
// Layout.  Each warp keeps two grid points (one FP32x2 pair) and their (B + 1) x (B + 1) u32
// histograms in shared memory (row = fixed bin, the last row and column for the marginals),
// filled with shared-memory atomics.  The fixed image's bins, premultiplied by the row stride,
// come from a plane written by span_prep_mi_kernel; the taps come from the quad plane in
// global memory through L1 (the histograms take the shared memory that windows would need).
// The warps of a CTA meet at a barrier per band of rows, so that their points (neighbours in the
// locality order) read the same region of the quad plane while it is in L1.
#pragma once
#include "cgs_span.cuh"

namespace cgs {

constexpr int kMiQueue = 192;  // deferred samples per warp (a block adds at most 64 before the check)

__host__ __device__ constexpr size_t span_mi_smem_bytes(int NW, int TH, int B) {
    return span_head_bytes(NW) + (size_t)NW * 2 * sizeof(SpanSlot) + (size_t)NW * sizeof(PairRow) +
           (size_t)NW * 2 * TH * sizeof(InnerSpan) + (size_t)NW * TH * sizeof(RowRun) +
           (size_t)NW * 2 * sizeof(int) + (size_t)NW * sizeof(int) + (size_t)NW * kMiQueue * sizeof(uint32_t) +
           (size_t)NW * 2 * (B + 1) * (B + 1) * sizeof(uint32_t) + 16;
}

struct SpanMiSmem {
    unsigned long long *wbest;
    int *bounds_flag;
    SpanSlot *slots;   // [NW * 2]
    PairRow *prow;     // [NW]
    InnerSpan *spans;  // [NW][2][TH]
    RowRun *runs;      // [NW][TH]
    int *cnt;          // [NW][2] overlap counts
    int *qcnt;         // [NW] queued samples
    uint32_t *queue;   // [NW][kMiQueue] x | y << 15 | g << 30
    uint32_t *hist;    // [NW * 2][(B + 1)^2]
};

template <int NW>
__device__ __forceinline__ SpanMiSmem carve_span_mi(unsigned char *smem, int TH, int B) {
    SpanMiSmem s;
    s.wbest = reinterpret_cast<unsigned long long *>(smem + 64);
    s.bounds_flag = reinterpret_cast<int *>(smem + 64 + 8 * NW);
    unsigned char *q = smem + span_head_bytes(NW);
    s.slots = reinterpret_cast<SpanSlot *>(q);
    q += (size_t)NW * 2 * sizeof(SpanSlot);
    s.prow = reinterpret_cast<PairRow *>(q);
    q += (size_t)NW * sizeof(PairRow);
    s.spans = reinterpret_cast<InnerSpan *>(q);
    q += (size_t)NW * 2 * TH * sizeof(InnerSpan);
    s.runs = reinterpret_cast<RowRun *>(q);
    q += (size_t)NW * TH * sizeof(RowRun);
    s.cnt = reinterpret_cast<int *>(q);
    q += (size_t)NW * 2 * sizeof(int);
    s.qcnt = reinterpret_cast<int *>(q);
    q += (size_t)NW * sizeof(int);
    s.queue = reinterpret_cast<uint32_t *>(q);
    q += (size_t)NW * kMiQueue * sizeof(uint32_t);
    s.hist = reinterpret_cast<uint32_t *>(q);
    return s;
}

// One count into a shared-memory histogram.  No compiler memory clobber: the counts are read only
// after a __syncwarp or __syncthreads, and the loads of the next samples may move ahead of it.
__device__ __forceinline__ void red_shared_add1(uint32_t addr) {
    asm volatile("red.shared.add.u32 [%0], 1;" ::"r"(addr));
}

// The reference's bin of value v: min(max(floor(v B / 256), 0), B - 1).
__device__ __forceinline__ int mi_bin(float v, float sB, int B) { return min(max((int)floorf(v * sB), 0), B - 1); }

// One task: the two grid points of each warp over every row of the fixed image.
template <int NW, bool CHECK>
__device__ __forceinline__ void run_span_mi_task(const SearchParams &p, uint32_t task, const SpanMiSmem &ss) {
    constexpr int G = 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int fw = p.fix.w, fh = p.fix.h;
    const int TH = p.tile_h;
    const float mov_wf = p.mov_wf, mov_hf = p.mov_hf;
    const float *__restrict__ mdata = p.mov.data;
    const int mpitch = p.mov.pitch;
    const float *__restrict__ fdata = p.fix.data;
    const int fpitch = p.fix.pitch;
    const int32_t *__restrict__ fbins = reinterpret_cast<const int32_t *>(p.span_rows);  // bin (B + 1)
    const int B = p.mi_bins;
    const int hstride = B + 1, hsize = (B + 1) * (B + 1);
    const float sB = (float)B * (1.0f / 256.0f);
    const float Bh = (float)B - 0.5f;
    // rounding allowance: the fast (three FMAs on pre-differenced taps) and the exact
    // interpolations of the same coordinates differ by at most 16u max|v| (twice that here)
    const float gv0 = sB * 2.0f * 16.0f * 5.9604645e-8f * (*p.vmax) + 1e-6f;
    const float lmax = *reinterpret_cast<const float *>(p.span_rows_header);  // largest quad slope bound

    // ---- the warp's two points
    const uint32_t ord0 = (task * NW + warp) * G;
    float2 A2, C12, D12, sg2, gl2, hh2;
    SpanSlot *my_slots = ss.slots + warp * G;
#pragma unroll
    for (int g = 0; g < G; g++) {
        const uint32_t o = ord0 + g;
        const bool gvalid = o < p.n;
        int32_t ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const uint32_t gidx = gvalid ? ordinal_to_index(p, o, ax) : 0u;
        float q[8];
        grid_values(p, ax, q);
        const float2 cs = p.trig[min(ax[0], kMaxTrig - 1)];
        const MapCoef kc = make_coef<CGS_COST_MI>(q, cs, p);
        FastMap fm;
        RowTerms rt;
        float gx, gy;
        map_guard(kc, p, fm, rt, gx, gy);
        const bool ok = gvalid && fm.li_x > 0.0f;
        if (lane == 0)
            my_slots[g] = SpanSlot{kc.A, rt.B, rt.PQ, kc.C1, rt.C2, rt.RS, kc.D1, rt.D2, rt.TU, kc.P, kc.Q, kc.R,
                                   kc.S, kc.T, kc.U, gx, gy, ok ? 1 : 0, gvalid ? 1 : 0, gidx};
        // slope factor of the bin guard: |v_fast - v_exact| <= (3|c10| + |c01| + 2|c11|) max(gx, gy)
        // (in bin units with sB), the factor covering the roundings of the sum
        const float sg = sB * fmaxf(gx, gy) * (1.0f + 0x1p-18f);
        const float gl = fmaf(lmax, sg, gv0);  // the bound near a cell edge
        const float hh = 0.5f - fmaxf(gx, gy);  // fraction farther than this from 0.5: near a cell edge
        if (g == 0) {
            A2.x = kc.A; C12.x = kc.C1; D12.x = kc.D1; sg2.x = sg; gl2.x = gl; hh2.x = hh;
        } else {
            A2.y = kc.A; C12.y = kc.C1; D12.y = kc.D1; sg2.y = sg; gl2.y = gl; hh2.y = hh;
        }
    }
    __syncwarp();
    if (lane == 0) {
        const SpanSlot &a = my_slots[0], &b = my_slots[1];
        ss.prow[warp] = PairRow{make_float2(a.B, b.B), make_float2(a.PQ, b.PQ), make_float2(a.C2, b.C2),
                                make_float2(a.RS, b.RS), make_float2(a.D2, b.D2), make_float2(a.TU, b.TU)};
    }
    uint32_t *my_hist = ss.hist + (size_t)warp * G * hsize;
    for (int i = lane; i < G * hsize; i += 32) my_hist[i] = 0u;
    int *my_cnt = ss.cnt + warp * G;
    int *my_qcnt = ss.qcnt + warp;
    uint32_t *my_queue = ss.queue + warp * kMiQueue;
    if (lane < G) my_cnt[lane] = 0;
    if (lane == 0) *my_qcnt = 0;
    __syncwarp();
    const uint32_t hist_s = smem_addr(my_hist);

    // one sample of point g at (x, y) by the reference's exact sequence, counted if inside
    auto exact_sample = [&](int g, int x, int y, bool count) {
        const SpanSlot &sl = my_slots[g];
        const MapCoef kc{sl.A, sl.B, sl.P, sl.Q, sl.C1, sl.C2, sl.R, sl.S, sl.D1, sl.D2, sl.T, sl.U};
        float ex, ey;
        exact_map(kc, (float)x, (float)y, ex, ey);
        if (in_image(ey, ex, mov_wf, mov_hf)) {
            const int bm = mi_bin(bilinear_in(mdata, mpitch, ey, ex), sB, B);
            const int bf = mi_bin(fdata[(int64_t)y * fpitch + x], sB, B);
            red_shared_add1(hist_s + 4u * (uint32_t)(g * hsize + bf * hstride + bm));
            return count ? 1 : 0;
        }
        return 0;
    };
    // the queued samples, all lanes at once (inside for the reference: no count)
    auto drain = [&]() {
        __syncwarp();
        const int nq = *my_qcnt;
        for (int e = lane; e < nq; e += 32) {
            const uint32_t v = my_queue[e];
            exact_sample((int)(v >> 30), (int)(v & 0x7fffu), (int)((v >> 15) & 0x7fffu), false);
        }
        __syncwarp();
        if (lane == 0) *my_qcnt = 0;
        __syncwarp();
    };

    InnerSpan *my_spans = ss.spans + warp * G * TH;
    RowRun *my_runs = ss.runs + warp * TH;
    const float2 magic2 = make_float2(kMagic, kMagic), nmagic2 = make_float2(-kMagic, -kMagic);
    const float2 minus1 = make_float2(-1.0f, -1.0f), mhalf2 = make_float2(-0.5f, -0.5f);
    const uint64_t mqbase = reinterpret_cast<uint64_t>(p.mov_quad) - 16ull * (uint64_t)(uint32_t)kMagicBits;
    const float2 qpitch2 = make_float2((float)p.quad_pitch, (float)p.quad_pitch);
    const int nblocks = (fw + 31) >> 5;

    for (int y0 = 0; y0 < fh; y0 += TH) {
        __syncthreads();  // the CTA's warps start each band together (L1 locality of the quads)
        // ---- the band's spans and band pixels (lanes: entries g TH + r)
        for (int k = 0; 32 * k < G * TH; k++) {
            const int i = lane + 32 * k;
            const bool act = i < G * TH;
            const int g = act ? i / TH : 0, r = i - g * TH;
            int n = 0;
            if (act) {
                const SpanSlot &sl = my_slots[g];
                const int y = y0 + r;
                InnerSpan is{0, 0};
                if (y < fh && sl.valid) {
                    const float yf = (float)y;
                    int xa = 0, len = 0, pa = 0, plen = fw;  // ill-conditioned: every pixel exact
                    if (sl.ok) {
                        const float wm = fmaf(sl.A, 0.5f * (float)(fw - 1), fmaf(sl.B, yf, sl.PQ));
                        const float s = wm > 0.0f ? 1.0f : -1.0f;
                        row_span(sl, yf, s, fw, mov_wf, mov_hf, 1.5f * sl.gx, 1.5f * sl.gy, xa, len);
                        row_span(sl, yf, s, fw, mov_wf, mov_hf, -1.5f * sl.gx, -1.5f * sl.gy, pa, plen);
                        if (len > 0 && plen > 0) {
                            const int lo = min(pa, xa), hi = max(pa + plen, xa + len);
                            pa = lo;
                            plen = hi - lo;
                        } else if (len > 0) {
                            pa = xa;
                            plen = len;
                        }
                    }
                    is = InnerSpan{xa, len};
                    n = len;
                    const int e0 = len > 0 ? xa : pa + plen, e1 = len > 0 ? xa + len : pa + plen;
                    for (int x = pa; x < e0; x++) n += exact_sample(g, x, y, true);
                    for (int x = e1; x < pa + plen; x++) n += exact_sample(g, x, y, true);
                }
                my_spans[g * TH + r] = is;
            }
            for (int o = 1; o < TH && o < 32; o <<= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
            if (act && r == 0) my_cnt[g] += n;
        }
        __syncwarp();
        if (lane < TH) {
            int ia = 0, ib = fw - 1, ua = 1 << 30, ub = -1;
#pragma unroll
            for (int g = 0; g < G; g++) {
                const InnerSpan is = my_spans[g * TH + lane];
                if (is.len > 0) {
                    ia = max(ia, is.xa);
                    ib = min(ib, is.xa + is.len - 1);
                    ua = min(ua, is.xa);
                    ub = max(ub, is.xa + is.len - 1);
                } else {
                    ib = -1;
                }
            }
            my_runs[lane] = RowRun{ia, ib, ua, ub};
        }
        __syncwarp();

        // ---- the band's rows
        for (int r = 0; r < TH && y0 + r < fh; r++) {
            const RowRun run = my_runs[r];
            if (run.ua > run.ub) continue;
            const int y = y0 + r;
            const float2 yf2 = make_float2((float)y, (float)y);
            const PairRow pr = ss.prow[warp];
            const float2 byw = __ffma2_rn(pr.B, yf2, pr.PQ);
            const float2 byx = __ffma2_rn(pr.C2, yf2, pr.RS);
            const float2 byy = __ffma2_rn(pr.D2, yf2, pr.TU);
            const int32_t *brow = fbins + (int64_t)y * fpitch;
            // NB consecutive blocks of 32 columns from block c (the lane's columns 32 c + lane + 32 k);
            // EDGE: some column may lie outside a point's inner span
            auto column = [&](int c, auto edge_tag, auto nb_tag) {
                constexpr bool EDGE = decltype(edge_tag)::value;
                constexpr int NB = decltype(nb_tag)::value;
                int x[NB], fb[NB];
                bool in0[NB], in1[NB], amb0[NB], amb1[NB];
#pragma unroll
                for (int k = 0; k < NB; k++) {
                    x[k] = 32 * (c + k) + lane;
                    in0[k] = true;
                    in1[k] = true;
                    if constexpr (EDGE) {
                        const InnerSpan a = my_spans[r], b = my_spans[TH + r];
                        in0[k] = (unsigned)(x[k] - a.xa) < (unsigned)a.len;
                        in1[k] = (unsigned)(x[k] - b.xa) < (unsigned)b.len;
                    }
                    fb[k] = __ldg(brow + min(x[k], fw - 1));  // fixed bin x (B + 1)
                }
#pragma unroll
                for (int k = 0; k < NB; k++) {
                    const float xf = (float)x[k];
                    const float2 xf2 = make_float2(xf, xf);
                    const float2 w = __ffma2_rn(A2, xf2, byw);
                    const float2 X = __ffma2_rn(C12, xf2, byx);
                    const float2 Y = __ffma2_rn(D12, xf2, byy);
                    const float2 rw = make_float2(rcp_approx(w.x), rcp_approx(w.y));
                    const float2 mx = __fmul2_rn(X, rw), my = __fmul2_rn(Y, rw);
                    const float2 tx2 = __fadd2_rd(mx, magic2), ty2 = __fadd2_rd(my, magic2);
                    const float2 fx2 = __fadd2_rn(tx2, nmagic2), fy2 = __fadd2_rn(ty2, nmagic2);
                    const float2 ax2 = __ffma2_rn(fx2, minus1, mx), ay2 = __ffma2_rn(fy2, minus1, my);
                    const float2 qi = __ffma2_rn(fy2, qpitch2, tx2);
                    uint32_t q0b = __float_as_uint(qi.x), q1b = __float_as_uint(qi.y);
                    if constexpr (EDGE) {
                        q0b = in0[k] ? q0b : (uint32_t)kMagicBits;
                        q1b = in1[k] ? q1b : (uint32_t)kMagicBits;
                    }
                    if constexpr (CHECK) {  // inside the moving image, else recorded and skipped
                        const int ix0 = (int)(__float_as_uint(tx2.x) - (uint32_t)kMagicBits);
                        const int iy0 = (int)(__float_as_uint(ty2.x) - (uint32_t)kMagicBits);
                        const int ix1 = (int)(__float_as_uint(tx2.y) - (uint32_t)kMagicBits);
                        const int iy1 = (int)(__float_as_uint(ty2.y) - (uint32_t)kMagicBits);
                        const bool b0 = in0[k] && ((unsigned)ix0 >= (unsigned)p.mov.w || (unsigned)iy0 >= (unsigned)p.mov.h);
                        const bool b1 = in1[k] && ((unsigned)ix1 >= (unsigned)p.mov.w || (unsigned)iy1 >= (unsigned)p.mov.h);
                        if (b0 | b1) *ss.bounds_flag = 1;
                        q0b = b0 ? (uint32_t)kMagicBits : q0b;
                        q1b = b1 ? (uint32_t)kMagicBits : q1b;
                        in0[k] = in0[k] && !b0;
                        in1[k] = in1[k] && !b1;
                    }
                    const float4 q0 = __ldg(reinterpret_cast<const float4 *>(mqbase + 16ull * q0b));
                    const float4 q1 = __ldg(reinterpret_cast<const float4 *>(mqbase + 16ull * q1b));
                    // values: quad = {c00, c10, c01, c11}, m = (c00 + ax c10) + ay (c01 + ax c11)
                    const float v0 = fmaf(ay2.x, fmaf(ax2.x, q0.w, q0.z), fmaf(ax2.x, q0.y, q0.x));
                    const float v1 = fmaf(ay2.y, fmaf(ax2.y, q1.w, q1.z), fmaf(ax2.y, q1.y, q1.x));
                    const float2 t = __fmul2_rn(make_float2(v0, v1), make_float2(sB, sB));
                    const float2 tb = __fadd2_rd(t, magic2);  // floor(t) in the mantissa (|t| < 2^22)
                    const float2 fr = __ffma2_rn(__fadd2_rn(tb, nmagic2), minus1, t);
                    // bin-edge guard: the sample's distance to the nearer edge against the bound
                    const float s0 = fmaf(2.0f, fabsf(q0.w), fmaf(3.0f, fabsf(q0.y), fabsf(q0.z)));
                    const float s1 = fmaf(2.0f, fabsf(q1.w), fmaf(3.0f, fabsf(q1.y), fabsf(q1.z)));
                    float2 gb = __ffma2_rn(make_float2(s0, s1), sg2, make_float2(gv0, gv0));
                    const float2 dfr = __fadd2_rn(fr, mhalf2);
                    const float2 dax = __fadd2_rn(ax2, mhalf2), day = __fadd2_rn(ay2, mhalf2);
                    // within the guard of a cell edge: the image's largest slope bounds the difference
                    if (fmaxf(fabsf(dax.x), fabsf(day.x)) > hh2.x) gb.x = fmaxf(gb.x, gl2.x);
                    if (fmaxf(fabsf(dax.y), fabsf(day.y)) > hh2.y) gb.y = fmaxf(gb.y, gl2.y);
                    // an edge at 0 or B is no edge: the bin is clamped there
                    amb0[k] = in0[k] && (fabsf(dfr.x) > 0.5f - gb.x) && (t.x > 0.5f) && (t.x < Bh);
                    amb1[k] = in1[k] && (fabsf(dfr.y) > 0.5f - gb.y) && (t.y > 0.5f) && (t.y < Bh);
                    const int bm0 = min(max(__float2int_rd(t.x), 0), B - 1);
                    const int bm1 = min(max(__float2int_rd(t.y), 0), B - 1);
                    if (in0[k] && !amb0[k]) red_shared_add1(hist_s + 4u * (uint32_t)(fb[k] + bm0));
                    if (in1[k] && !amb1[k]) red_shared_add1(hist_s + 4u * (uint32_t)(hsize + fb[k] + bm1));
                }
                // undecided samples: queued for the exact sequence
#pragma unroll
                for (int k = 0; k < NB; k++) {
                    const unsigned m0 = __ballot_sync(0xffffffffu, amb0[k]), m1 = __ballot_sync(0xffffffffu, amb1[k]);
                    if (m0 | m1) {
                        const unsigned lt = (1u << lane) - 1u;
                        const int base = *my_qcnt;
                        const int c0 = __popc(m0);
                        const uint32_t enc = (uint32_t)x[k] | ((uint32_t)y << 15);
                        if (amb0[k]) my_queue[base + __popc(m0 & lt)] = enc;
                        if (amb1[k]) my_queue[base + c0 + __popc(m1 & lt)] = enc | (1u << 30);
                        __syncwarp();
                        if (lane == 0) *my_qcnt = base + c0 + __popc(m1);
                        __syncwarp();
                        if (base + c0 + __popc(m1) > kMiQueue - 64) drain();
                    }
                }
            };
            const int cu0 = max(0, run.ua >> 5), cu1 = min(nblocks - 1, run.ub >> 5);
            int cf0 = cu1 + 1, cf1 = cu1;
            if (run.ia <= run.ib) {
                const int a = max(cu0, (run.ia + 31) >> 5), b = min(cu1, ((run.ib + 1) >> 5) - 1);
                if (a <= b) {
                    cf0 = a;
                    cf1 = b;
                }
            }
            using One = std::integral_constant<int, 1>;
            using Two = std::integral_constant<int, 2>;
#pragma unroll 1
            for (int c = cu0; c < cf0; c++) column(c, std::true_type{}, One{});
            int c = cf0;
#pragma unroll 1
            for (; c + 1 <= cf1; c += 2) column(c, std::false_type{}, Two{});  // two blocks in flight
            if (c <= cf1) column(c, std::false_type{}, One{});
#pragma unroll 1
            for (int c2 = cf1 + 1; c2 <= cu1; c2++) column(c2, std::true_type{}, One{});
        }
        drain();
    }

    // ---- per grid point: MI from the exact counts, dump, argmin key
    __syncwarp();
    float my_cost = 0.0f;
#pragma unroll
    for (int g = 0; g < G; g++) {
        const float c = mi_from_hist(my_hist + g * hsize, my_cnt[g], B, hstride, p);
        if (lane == g) my_cost = c;
        __syncwarp();
    }
    unsigned long long kk = ~0ull;
    if (lane < G) {
        const SpanSlot &sl = my_slots[lane];
        if (sl.valid) {
            if (p.costs) p.costs[sl.index] = my_cost;
            kk = make_key(my_cost, sl.index);
        }
    }
    kk = warp_min_u64(kk);
    if (lane == 0) ss.wbest[warp] = kk;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long b = ~0ull;
        for (int w = 0; w < NW; w++) b = ss.wbest[w] < b ? ss.wbest[w] : b;
        if (CHECK && *ss.bounds_flag) atomicOr(p.status, kStatusSpanBounds);
        retire_tasks(p, b, 1u, false);
    }
    __syncthreads();  // the next task reuses the slots
}

template <int NW, bool CHECK>
__global__ void __launch_bounds__(NW * 32, 1) span_mi_kernel(const __grid_constant__ SearchParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const SpanMiSmem ss = carve_span_mi<NW>(smem, p.tile_h, p.mi_bins);
    if (threadIdx.x == 0) *ss.bounds_flag = 0;
    __syncthreads();
    for (uint32_t task = blockIdx.x; task < p.num_tasks; task += gridDim.x) run_span_mi_task<NW, CHECK>(p, task, ss);
}

// The MI span kernel's staging step, after prep_kernel: the fixed image's bins times the row
// stride B + 1 (int32, the staged fixed plane's pitch), and the quads' largest slope bound.
static __global__ void __launch_bounds__(256)
span_prep_mi_kernel(const float *__restrict__ fix, int fpitch, int fw, int fh, int B, int32_t *__restrict__ bins,
                    const float4 *__restrict__ quads, int64_t nquads, unsigned int *__restrict__ lmax) {
    const float sB = (float)B * (1.0f / 256.0f);
    const int64_t n = (int64_t)fh * fpitch;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int64_t y = i / fpitch, x = i - y * fpitch;
        bins[i] = x < fw ? mi_bin(fix[i], sB, B) * (B + 1) : 0;
    }
    // the largest slope bound 3|c10| + |c01| + 2|c11| over the quads (non-negative floats order
    // as their bits; NaN taps give NaN bits above every finite value)
    float m = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nquads; i += stride) {
        const float4 q = quads[i];
        m = fmaxf(m, fmaf(2.0f, fabsf(q.w), fmaf(3.0f, fabsf(q.y), fabsf(q.z))) * (1.0f + 0x1p-18f));
    }
    unsigned int b = __float_as_uint(m);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if ((threadIdx.x & 31) == 0) atomicMax(lmax, b);
}

}  // namespace cgs
