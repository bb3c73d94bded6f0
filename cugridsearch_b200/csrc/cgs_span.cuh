// cgs_span.cuh -- the span kernel: zero-mean NCC over fast samples, with the in/out decisions
// taken per image row instead of per sample, the moving image's taps read from shared memory,
// and the fixed image's sums read from row prefix sums.  Its staging step is span_prep_kernel
// (end of this file), after the shared staging kernel has written the span form of the quads.
//
// Decisions per row.  For one grid point the map of a fixed row y is a projective line in the
// moving image; the samples that lie inside the moving image form one interval of x.  Solving
// the four half-plane conditions of "clearly inside" (a margin of 1.5 guard bands inside the
// image's edges, the guard being map_guard's bound between the fast and the reference's
// coordinates) and of "possibly inside" (1.5 guard bands outside) gives two integer spans per
// (row, point): every pixel of the inner span is inside for the reference too and takes the
// fast path with no test; pixels of the outer span outside the inner one (a band about a
// thousandth of a pixel wide around the overlap's edge, almost never a whole pixel) take the
// reference's exact operation sequence, evaluated once per band of rows by the lane that
// computed the span; every other pixel is outside and costs nothing.  The spans are computed
// in FP32; their rounding error is below a quarter of the guard band (the constraint terms are
// those the guard's own bound is built from), which the 1.5 factor covers.
//
// Fixed-image sums.  sum f and sum f^2 over a point's overlap are the inner spans' sums, taken
// from FP64 prefix sums of each fixed row (row_prefix_kernel), plus the band pixels found
// inside; only the three sums that involve the moving image are accumulated per sample.
//
// Tiles and windows.  The fixed image is walked in tiles of TW = 32 TX columns by TH rows.  For
// every 32-column block of a tile the CTA's grid points map the block into a small region of
// the moving image (the union of the block's quadrilateral images, points of one task being
// neighbours in the locality order); the regions of a tile's blocks are copied from the staged
// tap quads into one stage of a two-stage mbarrier pipeline by bulk copies, one per region row
// (the next tile's copies overlap the current tile's sweep), and the sweep reads its 16-byte
// quads from there.  A block whose region does not fit the stage reads global memory instead
// (same values).  Blocks rather than whole tiles bound the regions of rotated maps.
//
// Sweep.  Lane l takes the tile's columns x0 + l + 32 k; each warp evaluates its G grid points
// at every pixel, two points per packed FP32x2 instruction.  Blocks inside every point's inner
// span run without any per-sample test; other blocks mask samples by the inner spans.  A
// sample's quad index comes from the floor bits of its coordinates in one FP32x2 multiply-add
// (x + pitch y, exact below 2^22), its address from one shift-add.
//
// Sums.  Per lane, per band of TH rows: three FP32 sums per point of the shifted values
// f' = f - s_f, m' = m - s_m (the images' means; sum m', sum m'^2, sum f'm'), reduced across the
// warp at the end of each band of tiles and accumulated in FP64 with the spans' fixed-image
// sums and the band pixels' sums; the cost is formed in FP64 (zncc_cost).  Which samples a lane
// sums, and in which order, depends only on the image and the tile shape, never on the points
// per warp or the warps per CTA: costs are bit-identical across those tunings.  The overlap
// count is the sum of the inner span lengths plus the band pixels found inside.
#pragma once
#include <cstddef>
#include <type_traits>

#include "cgs_kernels.cuh"

namespace cgs {

constexpr int kWinStages = 2;
// Moving images with (W + 8) H >= 2^22 are outside the span path: the quad index x + pitch y
// (pitch at most W + 7) is formed exactly in FP32 below that.
constexpr int64_t kSpanMaxQuads = (int64_t)1 << 22;
// kStatusSpanBounds (cgs_internal.h): status bit the self-checking build (CHECK = true) sets in
// the result when a fast sample's quad address fell outside its block's window or the quad
// plane (the sample is then skipped).

// Everything the span path keeps of one grid point (shared memory, one per point of the task).
struct SpanSlot {
    float A, B, PQ, C1, C2, RS, D1, D2, TU;  // fast map: w = A x + (B y + PQ), X = .., Y = ..
    float P, Q, R, S, T, U;                  // exact-path terms (with A, B, C1, C2, D1, D2)
    float gx, gy;                            // guard band (map_guard)
    int32_t ok;                              // 1: fast path valid (guard holds, point in the grid)
    int32_t valid;                           // 1: ordinal inside the grid
    uint32_t index;                          // grid index of the point
};

// Row-term coefficients of a pair of points, packed for FP32x2: {B, PQ, C2, RS, D2, TU} of
// point 2h and 2h + 1 interleaved.
struct PairRow {
    float2 B, PQ, C2, RS, D2, TU;
};

// The moving-image window of one 32-column block of a tile: quads [y0, y0 + h) x [x0, x0 + w)
// with row pitch `pitch` quads, `off` quads into the stage's window area; h == 0: no point
// samples the block on the fast path; w < 0: the window does not fit the stage and the sweep
// reads global memory.  For the sweep: rel = 16 (off - x0 - pitch y0 - kMagicBits) (mod 2^32),
// so that quad (ix, iy) lies at stage window + rel + 16 bits(fy pitch + tx); pitchf = pitch.
struct BlockWin {
    int16_t x0, y0, w, h;
    int32_t pitch, off;
    uint32_t rel;
    float pitchf;
};
static_assert(sizeof(BlockWin) == 24 && offsetof(BlockWin, rel) == 16, "the sweep reads {rel, pitchf} as 8 bytes");

// Inner span of one (point, row): [xa, xa + len).
struct InnerSpan {
    int32_t xa, len;
};

// One row of a warp's points: [ia, ib] lies in every point's inner span (empty if ia > ib),
// [ua, ub] is the hull of their inner spans (empty if ua > ub).
struct RowRun {
    int32_t ia, ib, ua, ub;
};

__host__ __device__ constexpr size_t span_head_bytes(int NW) { return 256 + 8 * (size_t)NW; }

// Shared-memory plan of the span kernel for NW warps of G points, TH-row bands, tiles of TX
// blocks, `tiles` tiles and a stage of `cap` quads.
__host__ __device__ constexpr size_t span_smem_bytes(int G, int NW, int TH, int TX, int tiles, int cap) {
    return span_head_bytes(NW) + (size_t)NW * G * sizeof(SpanSlot) + (size_t)NW * (G / 2) * sizeof(PairRow) +
           (size_t)tiles * TX * sizeof(BlockWin) + (size_t)NW * G * TH * sizeof(InnerSpan) +
           (size_t)NW * TH * sizeof(RowRun) + (size_t)NW * G * (5 * sizeof(double) + sizeof(int)) +
           (size_t)kWinStages * cap * 16 + 128;
}

struct SpanSmem {
    uint64_t *bars;   // [kWinStages]
    unsigned long long *wbest;
    int *abort_flag;
    int *bounds_flag;  // self-checking build: a sample's quad address fell outside its window
    SpanSlot *slots;   // [NW * G]
    PairRow *prow;     // [NW * G / 2]
    BlockWin *wins;    // [tiles][TX]
    InnerSpan *spans;  // [NW][G][TH]
    RowRun *runs;      // [NW][TH]
    double *dtot;      // [NW][G * 5] FP64 task totals {sum f, sum m', sum f^2, sum m'^2, sum f'm'}
    int *cnt;          // [NW][G] overlap counts of the warps' points
    float4 *win;       // [kWinStages][cap]
    int cap;
};

template <int G, int NW>
__device__ __forceinline__ SpanSmem carve_span(unsigned char *smem, int TH, int TX, int tiles, int cap) {
    SpanSmem s;
    s.bars = reinterpret_cast<uint64_t *>(smem);
    s.wbest = reinterpret_cast<unsigned long long *>(smem + 64);
    s.abort_flag = reinterpret_cast<int *>(smem + 64 + 8 * NW);
    s.bounds_flag = s.abort_flag + 1;
    unsigned char *q = smem + span_head_bytes(NW);
    s.slots = reinterpret_cast<SpanSlot *>(q);
    q += (size_t)NW * G * sizeof(SpanSlot);
    s.prow = reinterpret_cast<PairRow *>(q);
    q += (size_t)NW * (G / 2) * sizeof(PairRow);
    s.wins = reinterpret_cast<BlockWin *>(q);
    q += (size_t)tiles * TX * sizeof(BlockWin);
    s.spans = reinterpret_cast<InnerSpan *>(q);
    q += (size_t)NW * G * TH * sizeof(InnerSpan);
    s.runs = reinterpret_cast<RowRun *>(q);
    q += (size_t)NW * TH * sizeof(RowRun);
    s.dtot = reinterpret_cast<double *>(q);
    q += (size_t)NW * G * 5 * sizeof(double);
    s.cnt = reinterpret_cast<int *>(q);
    q += (size_t)NW * G * sizeof(int);
    // aligned by offset from the shared base (an integer round trip of the pointer would lose
    // its shared-memory provenance and turn every window read into a generic load)
    const size_t off = ((size_t)(q - smem) + 127) & ~(size_t)127;
    s.win = reinterpret_cast<float4 *>(smem + off);
    s.cap = cap;
    return s;
}

// Row span of one point: the integer x in [0, fw) satisfying the four half-plane conditions
// m < X/w < W - m, m < Y/w < H - m (margins mx, my; negative margins widen), w of sign s.
__device__ __forceinline__ void row_span(const SpanSlot &k, float yf, float s, int fw, float mw, float mh, float mx,
                                         float my, int &xa, int &len) {
    const float bw = fmaf(k.B, yf, k.PQ), bX = fmaf(k.C2, yf, k.RS), bY = fmaf(k.D2, yf, k.TU);
    float lo = -1.0f, hi = (float)fw;  // open interval of admissible x, clamped to the row
    bool none = false;
    auto cons = [&](float a, float b) {  // s (a x + b) > 0
        a *= s;
        b *= s;
        if (a > 0.0f) lo = fmaxf(lo, -b / a);
        else if (a < 0.0f) hi = fminf(hi, -b / a);
        else if (!(b > 0.0f)) none = true;
    };
    cons(fmaf(-mx, k.A, k.C1), fmaf(-mx, bw, bX));                    // X - m w > 0
    cons(fmaf(mw - mx, k.A, -k.C1), fmaf(mw - mx, bw, -bX));          // (W - m) w - X > 0
    cons(fmaf(-my, k.A, k.D1), fmaf(-my, bw, bY));                    // Y - m w > 0
    cons(fmaf(mh - my, k.A, -k.D1), fmaf(mh - my, bw, -bY));          // (H - m) w - Y > 0
    lo = fmaxf(lo, -1.0f);
    hi = fminf(hi, (float)fw);
    const int a0 = max(0, (int)floorf(lo) + 1), b0 = min(fw - 1, (int)ceilf(hi) - 1);
    xa = a0;
    len = (none || b0 < a0) ? 0 : b0 - a0 + 1;
}

// The corners of block [x0, x1] x [y0, y1] under a point's map: min/max of the mapped coordinates.
__device__ __forceinline__ void block_extent(const SpanSlot &k, float x0, float x1, float y0, float y1, float4 &e) {
    auto one = [&](float x, float y) {
        const float w = fmaf(k.A, x, fmaf(k.B, y, k.PQ));
        const float X = fmaf(k.C1, x, fmaf(k.C2, y, k.RS));
        const float Y = fmaf(k.D1, x, fmaf(k.D2, y, k.TU));
        const float mx = X / w, my = Y / w;
        e.x = fminf(e.x, mx);
        e.y = fminf(e.y, my);
        e.z = fmaxf(e.z, mx);
        e.w = fmaxf(e.w, my);
    };
    one(x0, y0);
    one(x1, y0);
    one(x0, y1);
    one(x1, y1);
}

// Issue (warp 0) the copies of tile t into stage `st`, completing on that stage's barrier: the
// tile's rows of the staged fixed image (TH x TW floats at the stage's start; columns past the
// image's right edge are not copied) and the windows of its blocks (quads, after the fixed tile).
template <int TX>
__device__ __forceinline__ void issue_window(const SearchParams &p, const SpanSmem &ss, int t, int st) {
    constexpr int TW = 32 * TX;
    const int lane = threadIdx.x & 31;
    const int TH = p.tile_h;
    const int x0 = (t % p.tiles_x) * TW, y0 = (t / p.tiles_x) * TH;
    const int rows = min(TH, p.fix.h - y0);
    const uint32_t row_bytes = (uint32_t)((min(TW, p.fix.w - x0) * 4 + 15) & ~15);  // within the row pitch
    const BlockWin *bw = ss.wins + t * TX;
    uint64_t *bar = &ss.bars[st];
    if (lane == 0) {
        uint32_t bytes = (uint32_t)rows * row_bytes;
#pragma unroll
        for (int c = 0; c < TX; c++)
            if (bw[c].h > 0 && bw[c].w > 0) bytes += (uint32_t)bw[c].w * (uint32_t)bw[c].h * 16u;
        fence_proxy_async_smem();  // the stage's previous reads before the async refill
        mbar_arrive_expect_tx(bar, bytes);
    }
    __syncwarp();
    fence_proxy_async_smem();
    float *fdst = reinterpret_cast<float *>(ss.win + (size_t)st * ss.cap);
    for (int j = lane; j < rows; j += 32)
        bulk_g2s(fdst + j * TW, p.fix.data + (int64_t)(y0 + j) * p.fix.pitch + x0, row_bytes, bar);
    float4 *wdst = ss.win + (size_t)st * ss.cap + TH * TW / 4;
#pragma unroll
    for (int c = 0; c < TX; c++) {
        const BlockWin b = bw[c];
        if (b.h > 0 && b.w > 0) {
            const float4 *src = p.mov_quad + (int64_t)b.y0 * p.quad_pitch + b.x0;
            for (int j = lane; j < b.h; j += 32)
                bulk_g2s(wdst + b.off + (size_t)j * b.pitch, src + (int64_t)j * p.quad_pitch, (uint32_t)b.w * 16u,
                         bar);
        }
    }
}

// One task of the span path (ZNCC, one channel, quads staged): the G grid points of each warp
// over every tile of the fixed image.  `wit` counts window stages used by this CTA (their
// barrier phases).  Returns false if a bounded wait gave up.
template <int G, int NW, int TX, bool CHECK>
__device__ __forceinline__ bool run_span_task(const SearchParams &p, uint32_t task, const SpanSmem &ss,
                                              uint32_t &wit) {
    static_assert(G % 2 == 0, "the span path pairs grid points");
    constexpr int GP = G / 2;
    constexpr int TW = 32 * TX;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int fw = p.fix.w, fh = p.fix.h;
    const int TH = p.tile_h;
    const int tiles_x = p.tiles_x, ntiles = p.tiles_x * p.tiles_y;
    const float mov_wf = p.mov_wf, mov_hf = p.mov_hf;
    const float *__restrict__ mdata = p.mov.data;
    const int mpitch = p.mov.pitch;
    const float *__restrict__ fdata = p.fix.data;
    const int fpitch = p.fix.pitch;

    // ---- the warp's points: coefficients, guard, slots
    const uint32_t ord0 = (task * NW + warp) * G;
    float2 A2[GP], C12[GP], D12[GP];
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
        const MapCoef kc = make_coef<CGS_COST_ZNCC>(q, cs, p);
        FastMap fm;
        RowTerms rt;
        float gx, gy;
        map_guard(kc, p, fm, rt, gx, gy);
        const bool ok = gvalid && fm.li_x > 0.0f;
        if (lane == 0)
            my_slots[g] = SpanSlot{kc.A, rt.B, rt.PQ, kc.C1, rt.C2, rt.RS, kc.D1, rt.D2, rt.TU, kc.P, kc.Q, kc.R,
                                   kc.S, kc.T, kc.U, gx, gy, ok ? 1 : 0, gvalid ? 1 : 0, gidx};
        if (g & 1) {
            A2[g / 2].y = kc.A; C12[g / 2].y = kc.C1; D12[g / 2].y = kc.D1;
        } else {
            A2[g / 2].x = kc.A; C12[g / 2].x = kc.C1; D12[g / 2].x = kc.D1;
        }
    }
    __syncwarp();
    if (lane < GP) {
        const SpanSlot &a = my_slots[2 * lane], &b = my_slots[2 * lane + 1];
        ss.prow[warp * GP + lane] = PairRow{make_float2(a.B, b.B), make_float2(a.PQ, b.PQ), make_float2(a.C2, b.C2),
                                            make_float2(a.RS, b.RS), make_float2(a.D2, b.D2), make_float2(a.TU, b.TU)};
    }
    // FP64 task totals and overlap counts of the warp's points (shared memory)
    double *my_dtot = ss.dtot + warp * G * 5;
    int *my_cnt = ss.cnt + warp * G;
    for (int i = lane; i < G * 5; i += 32) my_dtot[i] = 0.0;
    if (lane < G) my_cnt[lane] = 0;
    const float fshift = p.shifts[0], mshift = p.shifts[1];
    __syncthreads();  // every point's slot is written

    // ---- windows of every block of every tile: warp w takes tiles w, w + NW, ..; lanes take the
    // task's points
    {
        constexpr int P = NW * G;
        const int wcap = ss.cap - TH * TW / 4;  // quads of a stage after the fixed rows
        for (int t = warp; t < ntiles; t += NW) {
            const int x0 = (t % tiles_x) * TW, y0 = (t / tiles_x) * TH;
            const float fy0 = (float)y0, fy1 = (float)(min(y0 + TH, fh) - 1);
            float4 e[TX];
#pragma unroll
            for (int c = 0; c < TX; c++)
                e[c] = make_float4(__int_as_float(0x7f800000), __int_as_float(0x7f800000),
                                   -__int_as_float(0x7f800000), -__int_as_float(0x7f800000));
            for (int k = lane; k < P; k += 32) {
                const SpanSlot &sl = ss.slots[k];
                if (sl.ok) {
#pragma unroll
                    for (int c = 0; c < TX; c++) {
                        const int xc = x0 + 32 * c;
                        if (xc < fw) block_extent(sl, (float)xc, (float)(min(xc + 32, fw) - 1), fy0, fy1, e[c]);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < TX; c++) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    e[c].x = fminf(e[c].x, __shfl_xor_sync(0xffffffffu, e[c].x, o));
                    e[c].y = fminf(e[c].y, __shfl_xor_sync(0xffffffffu, e[c].y, o));
                    e[c].z = fmaxf(e[c].z, __shfl_xor_sync(0xffffffffu, e[c].z, o));
                    e[c].w = fmaxf(e[c].w, __shfl_xor_sync(0xffffffffu, e[c].w, o));
                }
            }
            if (lane == 0) {
                int used = 0;
#pragma unroll
                for (int c = 0; c < TX; c++) {
                    BlockWin bw{0, 0, 0, 0, 0, 0, 0u, 0.0f};
                    // cells a fast sample can use: floor of its coordinate (within the guard, < 1/8 px,
                    // of the real map, whose block image lies in the corners' hull), clipped to the image
                    const float lx = fmaxf(e[c].x - 0.25f, -1.0f), ly = fmaxf(e[c].y - 0.25f, -1.0f);
                    const float hx = fminf(e[c].z + 0.25f, mov_wf), hy = fminf(e[c].w + 0.25f, mov_hf);
                    if (lx <= hx && ly <= hy) {
                        const int cx0 = max(0, (int)floorf(lx)), cy0 = max(0, (int)floorf(ly));
                        const int cx1 = min(p.mov.w - 1, (int)floorf(hx)), cy1 = min(p.mov.h - 1, (int)floorf(hy));
                        if (cx0 <= cx1 && cy0 <= cy1) {
                            const int w = cx1 - cx0 + 1, h = cy1 - cy0 + 1;
                            const int pitch = w + ((p.win_pitch_mod - w) & 7);  // = win_pitch_mod (mod 8)
                            bw.x0 = (int16_t)cx0;
                            bw.y0 = (int16_t)cy0;
                            bw.h = (int16_t)h;
                            bw.pitch = pitch;
                            if ((int64_t)pitch * h <= wcap - used) {
                                bw.w = (int16_t)w;
                                bw.off = used;
                                bw.rel = 16u * ((uint32_t)used - (uint32_t)cx0 - (uint32_t)pitch * (uint32_t)cy0 -
                                                (uint32_t)kMagicBits);
                                bw.pitchf = (float)pitch;
                                used += pitch * h;
                            } else {
                                bw.w = -1;
                            }
                        }
                    }
                    ss.wins[t * TX + c] = bw;
                }
            }
        }
    }
    __syncthreads();
    if (warp == 0) {
        for (int t = 0; t < kWinStages && t < ntiles; t++) issue_window<TX>(p, ss, t, (int)((wit + t) % kWinStages));
    }

    // ---- sweep
    float2 part[GP][3];  // {sum m', sum m'^2, sum f'm'} of each pair of points
#pragma unroll
    for (int h = 0; h < GP; h++)
#pragma unroll
        for (int j = 0; j < 3; j++) part[h][j] = make_float2(0.0f, 0.0f);
    InnerSpan *my_spans = ss.spans + warp * G * TH;
    RowRun *my_runs = ss.runs + warp * TH;
    const float2 magic2 = make_float2(kMagic, kMagic), nmagic2 = make_float2(-kMagic, -kMagic);
    const float2 minus1 = make_float2(-1.0f, -1.0f);
    // quad index from floor bits: bits(ty + pitch fy) - kMagicBits = ix + pitch iy (exact below
    // 2^22); global quad (ix, iy) at mqbase + 16 bits
    const uint64_t mqbase = reinterpret_cast<uint64_t>(p.mov_quad) - 16ull * (uint64_t)(uint32_t)kMagicBits;
    const float2 qpitch2 = make_float2((float)p.quad_pitch, (float)p.quad_pitch);

    for (int t = 0; t < ntiles; t++, wit++) {
        const int tx = t % tiles_x, ty = t / tiles_x;
        const int x0 = tx * TW, y0 = ty * TH;
        const int x1 = min(x0 + TW, fw) - 1;
        if (tx == 0) {
            // the band's rows, every point of the warp: inner spans (their fixed-image sums from the
            // row prefix sums) and the band pixels, sampled by the reference's exact sequence;
            // entry i = g TH + r, lanes of one point reduce over its TH rows
            for (int k = 0; 32 * k < G * TH; k++) {
                const int i = lane + 32 * k;
                const bool act = i < G * TH;
                const int g = act ? i / TH : 0, r = i - g * TH;
                double s1 = 0.0, s2 = 0.0, sm = 0.0, smm = 0.0, sfm = 0.0;
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
                            if (len > 0 && plen > 0) {  // the outer span holds the inner one
                                const int lo = min(pa, xa), hi = max(pa + plen, xa + len);
                                pa = lo;
                                plen = hi - lo;
                            } else if (len > 0) {
                                pa = xa;
                                plen = len;
                            }
                        }
                        is = InnerSpan{xa, len};
                        if (len > 0) {
                            const double2 *pr = p.fix_prefix + (int64_t)y * (fw + 1);
                            const double2 a = pr[xa], b = pr[xa + len];
                            s1 = b.x - a.x;
                            s2 = b.y - a.y;
                            n = len;
                        }
                        // band pixels: the outer span outside the inner one, [pa, e0) and [e1, pa + plen)
                        const int e0 = len > 0 ? xa : pa + plen, e1 = len > 0 ? xa + len : pa + plen;
                        const MapCoef kc{sl.A, sl.B, sl.P, sl.Q, sl.C1, sl.C2, sl.R, sl.S, sl.D1, sl.D2, sl.T, sl.U};
                        const float *frow_g = fdata + (int64_t)y * fpitch;
                        auto band = [&](int xs, int xe) {
                            for (int x = xs; x < xe; x++) {
                                float ex, ey;
                                exact_map(kc, (float)x, yf, ex, ey);
                                if (in_image(ey, ex, mov_wf, mov_hf)) {
                                    const float m = bilinear_in(mdata, mpitch, ey, ex) - mshift;
                                    const float f = frow_g[x];
                                    const float fs = f - fshift;
                                    s1 += (double)f;
                                    s2 += (double)f * (double)f;
                                    sm += (double)m;
                                    smm += (double)m * (double)m;
                                    sfm += (double)fs * (double)m;
                                    n++;
                                }
                            }
                        };
                        band(pa, e0);
                        band(e1, pa + plen);
                    }
                    my_spans[g * TH + r] = is;
                }
                // sum over the TH lanes of each point (TH is 8, 16 or 32)
                for (int o = 1; o < TH && o < 32; o <<= 1) {
                    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                    sm += __shfl_xor_sync(0xffffffffu, sm, o);
                    smm += __shfl_xor_sync(0xffffffffu, smm, o);
                    sfm += __shfl_xor_sync(0xffffffffu, sfm, o);
                    n += __shfl_xor_sync(0xffffffffu, n, o);
                }
                if (act && r == 0) {
                    double *d = my_dtot + g * 5;
                    d[0] += s1;
                    d[1] += sm;
                    d[2] += s2;
                    d[3] += smm;
                    d[4] += sfm;
                    my_cnt[g] += n;
                }
            }
            __syncwarp();
            if (lane < TH) {  // the rows' common inner run and the hull of the inner spans
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
                        ib = -1;  // a point without an inner span (or outside the grid): no common run
                    }
                }
                my_runs[lane] = RowRun{ia, ib, ua, ub};
            }
            __syncwarp();
        }
        // the tile's windows
        const int st = (int)(wit % kWinStages);
        if (!mbar_wait_bounded(&ss.bars[st], (wit / kWinStages) & 1u, kWaitLimitNs)) *ss.abort_flag = 1;
        const BlockWin *twin = ss.wins + t * TX;
        const float *sfix = reinterpret_cast<const float *>(ss.win + (size_t)st * ss.cap);  // TH x TW
        const uint32_t wbase = smem_addr(ss.win + (size_t)st * ss.cap + TH * TW / 4);
        const uint32_t szero = smem_addr(ss.win);

        // one row: fast samples of G points at the lane's columns; EDGE masks by the inner spans
        auto row = [&](int r, const RowRun run) {
            const int y = y0 + r;
            const float yf = (float)y;
            const float2 yf2 = make_float2(yf, yf);
            float2 byw[GP], byx[GP], byy[GP];
#pragma unroll
            for (int h = 0; h < GP; h++) {
                const PairRow pr = ss.prow[warp * GP + h];
                byw[h] = __ffma2_rn(pr.B, yf2, pr.PQ);
                byx[h] = __ffma2_rn(pr.C2, yf2, pr.RS);
                byy[h] = __ffma2_rn(pr.D2, yf2, pr.TU);
            }
            const float *frow = sfix + r * TW;
            // one block of 32 columns; EDGE: some column may lie outside a point's inner span;
            // SMEM: the block's window is in the stage
            auto column = [&](int c, auto edge_tag, auto smem_tag) {
                constexpr bool EDGE = decltype(edge_tag)::value;
                constexpr bool SMEM = decltype(smem_tag)::value;
                // shared address of window quad (ix, iy): wbase + 16 (off + (ix - x0) + pitch (iy - y0))
                uint32_t sbase = 0u;
                float2 pitch2 = qpitch2;
                if constexpr (SMEM) {
                    const uint2 rp = *reinterpret_cast<const uint2 *>(&twin[c].rel);
                    sbase = wbase + rp.x;
                    pitch2 = make_float2(__uint_as_float(rp.y), __uint_as_float(rp.y));
                }
                InnerSpan isp[G];
                if constexpr (EDGE) {
#pragma unroll
                    for (int g = 0; g < G; g++) isp[g] = my_spans[g * TH + r];
                }
                const int x = x0 + 32 * c + lane;
                const float f = frow[32 * c + lane];  // past the image's right edge: not copied, unused
                const float fs = f - fshift;
                const float2 fs2 = make_float2(fs, fs);
                const float xf = (float)x;
                const float2 xf2 = make_float2(xf, xf);
#pragma unroll
                for (int h = 0; h < GP; h++) {
                    // both points of the pair in each FP32x2 operation: map, floor (round-down add
                    // of 1.5 * 2^23 leaves floor(m) in the mantissa), fraction, quad index
                    const float2 w = __ffma2_rn(A2[h], xf2, byw[h]);
                    const float2 X = __ffma2_rn(C12[h], xf2, byx[h]);
                    const float2 Y = __ffma2_rn(D12[h], xf2, byy[h]);
                    const float2 rw = make_float2(rcp_approx(w.x), rcp_approx(w.y));
                    const float2 mx = __fmul2_rn(X, rw), my = __fmul2_rn(Y, rw);
                    const float2 tx2 = __fadd2_rd(mx, magic2), ty2 = __fadd2_rd(my, magic2);
                    const float2 fx2 = __fadd2_rn(tx2, nmagic2), fy2 = __fadd2_rn(ty2, nmagic2);
                    const float2 ax2 = __ffma2_rn(fx2, minus1, mx), ay2 = __ffma2_rn(fy2, minus1, my);
                    const float2 qi = __ffma2_rn(fy2, pitch2, tx2);
                    bool in0 = true, in1 = true;
                    if constexpr (EDGE) {
                        const InnerSpan a = isp[2 * h], b = isp[2 * h + 1];
                        in0 = (unsigned)(x - a.xa) < (unsigned)a.len;
                        in1 = (unsigned)(x - b.xa) < (unsigned)b.len;
                    }
                    uint32_t q0b = __float_as_uint(qi.x), q1b = __float_as_uint(qi.y);
                    if constexpr (EDGE) {
                        q0b = in0 ? q0b : (uint32_t)kMagicBits;
                        q1b = in1 ? q1b : (uint32_t)kMagicBits;
                    }
                    float4 q0, q1;
                    if constexpr (SMEM) {
                        uint32_t a0 = sbase + (q0b << 4), a1 = sbase + (q1b << 4);
                        if constexpr (EDGE) {
                            a0 = in0 ? a0 : szero;
                            a1 = in1 ? a1 : szero;
                        }
                        if constexpr (CHECK) {  // inside the block's window, else recorded and skipped
                            const BlockWin bw = twin[c];
                            const int ix0 = (int)(__float_as_uint(tx2.x) - (uint32_t)kMagicBits) - bw.x0;
                            const int iy0 = (int)(__float_as_uint(ty2.x) - (uint32_t)kMagicBits) - bw.y0;
                            const int ix1 = (int)(__float_as_uint(tx2.y) - (uint32_t)kMagicBits) - bw.x0;
                            const int iy1 = (int)(__float_as_uint(ty2.y) - (uint32_t)kMagicBits) - bw.y0;
                            const bool b0 = in0 && ((unsigned)ix0 >= (unsigned)bw.w || (unsigned)iy0 >= (unsigned)bw.h);
                            const bool b1 = in1 && ((unsigned)ix1 >= (unsigned)bw.w || (unsigned)iy1 >= (unsigned)bw.h);
                            if (b0 | b1) *ss.bounds_flag = 1;
                            a0 = b0 ? szero : a0;
                            a1 = b1 ? szero : a1;
                        }
                        // the stage is ready (its barrier was waited on above); volatile keeps the
                        // loads after that wait
                        asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                                     : "=f"(q0.x), "=f"(q0.y), "=f"(q0.z), "=f"(q0.w) : "r"(a0));
                        asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                                     : "=f"(q1.x), "=f"(q1.y), "=f"(q1.z), "=f"(q1.w) : "r"(a1));
                    } else {
                        if constexpr (CHECK) {  // inside the moving image, else recorded and skipped
                            const int ix0 = (int)(__float_as_uint(tx2.x) - (uint32_t)kMagicBits);
                            const int iy0 = (int)(__float_as_uint(ty2.x) - (uint32_t)kMagicBits);
                            const int ix1 = (int)(__float_as_uint(tx2.y) - (uint32_t)kMagicBits);
                            const int iy1 = (int)(__float_as_uint(ty2.y) - (uint32_t)kMagicBits);
                            const bool b0 = in0 && ((unsigned)ix0 >= (unsigned)p.mov.w || (unsigned)iy0 >= (unsigned)p.mov.h);
                            const bool b1 = in1 && ((unsigned)ix1 >= (unsigned)p.mov.w || (unsigned)iy1 >= (unsigned)p.mov.h);
                            if (b0 | b1) *ss.bounds_flag = 1;
                            q0b = b0 ? (uint32_t)kMagicBits : q0b;
                            q1b = b1 ? (uint32_t)kMagicBits : q1b;
                        }
                        q0 = __ldg(reinterpret_cast<const float4 *>(mqbase + 16ull * q0b));
                        q1 = __ldg(reinterpret_cast<const float4 *>(mqbase + 16ull * q1b));
                    }
                    // quad = the bilinear polynomial's coefficients {c00 - s_m, c10, c01, c11}:
                    // m' = (c00 - s_m + ax c10) + ay (c01 + ax c11)
                    const float u0 = fmaf(ax2.x, q0.y, q0.x), w0 = fmaf(ax2.x, q0.w, q0.z);
                    const float u1 = fmaf(ax2.y, q1.y, q1.x), w1 = fmaf(ax2.y, q1.w, q1.z);
                    float2 ms = make_float2(fmaf(ay2.x, w0, u0), fmaf(ay2.y, w1, u1));
                    float2 fm = fs2;
                    if constexpr (EDGE) {  // by selection: a NaN outside the overlap stays out of the sums
                        ms = make_float2(in0 ? ms.x : 0.0f, in1 ? ms.y : 0.0f);
                        fm = make_float2(in0 ? fs : 0.0f, in1 ? fs : 0.0f);
                    }
                    part[h][0] = __fadd2_rn(part[h][0], ms);
                    part[h][1] = __ffma2_rn(ms, ms, part[h][1]);
                    part[h][2] = __ffma2_rn(fm, ms, part[h][2]);
                }
            };
            auto block = [&](int c, auto edge_tag) {
                if (twin[c].w > 0) column(c, edge_tag, std::true_type{});
                else column(c, edge_tag, std::false_type{});
            };
            // blocks with any inner span: [cu0, cu1]; those inside every point's inner span,
            // [cf0, cf1], run unmasked
            const int cu0 = max(0, (run.ua - x0) >> 5), cu1 = min(TX - 1, (run.ub - x0) >> 5);
            int cf0 = cu1 + 1, cf1 = cu1;
            if (run.ia <= run.ib) {
                const int a = max(cu0, (run.ia - x0 + 31) >> 5), b = min(cu1, ((run.ib - x0 + 1) >> 5) - 1);
                if (a <= b) {
                    cf0 = a;
                    cf1 = b;
                }
            }
#pragma unroll 1
            for (int c = cu0; c < cf0; c++) block(c, std::true_type{});
            int c = cf0;
#pragma unroll 1
            for (; c + 1 <= cf1; c += 2) {  // two full blocks of the same kind as straight-line code
                const bool s0 = twin[c].w > 0, s1 = twin[c + 1].w > 0;
                if (s0 && s1) {
                    column(c, std::false_type{}, std::true_type{});
                    column(c + 1, std::false_type{}, std::true_type{});
                } else if (!s0 && !s1) {
                    column(c, std::false_type{}, std::false_type{});
                    column(c + 1, std::false_type{}, std::false_type{});
                } else {
                    block(c, std::false_type{});
                    block(c + 1, std::false_type{});
                }
            }
            if (c <= cf1) block(c, std::false_type{});
#pragma unroll 1
            for (int c2 = cf1 + 1; c2 <= cu1; c2++) block(c2, std::true_type{});
        };
        for (int r = 0; r < TH; r++) {
            if (y0 + r >= fh) break;
            const RowRun run = my_runs[r];
            if (run.ua > x1 || run.ub < x0) continue;  // no point samples this row of the tile
            row(r, run);
        }
        // end of a band of tiles: the band's warp sums into the FP64 task totals
        if (tx == tiles_x - 1) {
#pragma unroll
            for (int h = 0; h < GP; h++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    const int slot = j == 0 ? 1 : (j == 1 ? 3 : 4);  // sum m', sum m'^2, sum f'm'
                    const float s0 = warp_sum(part[h][j].x), s1 = warp_sum(part[h][j].y);
                    if (lane == 0) {
                        my_dtot[(2 * h) * 5 + slot] += (double)s0;
                        my_dtot[(2 * h + 1) * 5 + slot] += (double)s1;
                    }
                    part[h][j] = make_float2(0.0f, 0.0f);
                }
        }
        __syncthreads();  // every warp is done with this stage
        if (*ss.abort_flag) {
            // a wait gave up: let this stage's copies and the next stage's (already issued) land,
            // within the same bound, before the CTA stops
            if (threadIdx.x == 0) {
                mbar_wait_bounded(&ss.bars[st], (wit / kWinStages) & 1u, kWaitLimitNs);
                if (t + 1 < ntiles)
                    mbar_wait_bounded(&ss.bars[(wit + 1) % kWinStages], ((wit + 1) / kWinStages) & 1u, kWaitLimitNs);
            }
            return false;
        }
        if (warp == 0 && t + kWinStages < ntiles) issue_window<TX>(p, ss, t + kWinStages, st);
    }

    // ---- per grid point: finalise, dump, argmin key (as the pixel-loop kernel)
    __syncwarp();
    unsigned long long kk = ~0ull;
    if (lane < G) {
        const SpanSlot &sl = my_slots[lane];
        const int n = my_cnt[lane];
        // the fixed-image sums were taken unshifted: sum f' = sum f - n s, sum f'^2 = sum f^2 -
        // 2 s sum f + n s^2 (FP64)
        const double s = (double)fshift, dn = (double)n;
        double a[5];
#pragma unroll
        for (int j = 0; j < 5; j++) a[j] = my_dtot[lane * 5 + j];
        const double f1 = a[0];
        a[0] = f1 - dn * s;
        a[2] = a[2] - 2.0 * s * f1 + dn * s * s;
        const float cost = zncc_cost(a, n, p);
        if (sl.valid) {
            if (p.costs) p.costs[sl.index] = cost;
            kk = make_key(cost, sl.index);
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
    return true;
}

// The single-pair span kernel: persistent CTAs, tasks dealt round-robin.
template <int G, int NW, int TX, bool CHECK>
__global__ void __launch_bounds__(NW * 32, 1) span_kernel(const __grid_constant__ SearchParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const SpanSmem ss = carve_span<G, NW>(smem, p.tile_h, TX, p.tiles_x * p.tiles_y, p.win_cap);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kWinStages; s++) mbar_init(&ss.bars[s], 1);
        fence_mbar_init();
        *ss.abort_flag = 0;
        *ss.bounds_flag = 0;
    }
    __syncthreads();
    const uint32_t my_tasks =
        (p.num_tasks > blockIdx.x) ? (p.num_tasks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    uint32_t wit = 0;
    for (uint32_t k = 0; k < my_tasks; k++) {
        if (!run_span_task<G, NW, TX, CHECK>(p, blockIdx.x + k * gridDim.x, ss, wit)) {
            if (threadIdx.x == 0) retire_tasks(p, ~0ull, my_tasks - k, true);
            return;
        }
    }
}

// Blocks [0, row_blocks) write the FP64 prefix sums of each staged fixed row, prefix[y (W + 1) +
// x] = {sum f, sum f^2} of pixels 0 .. x - 1 of row y (channel 0; one warp per row, a warp scan
// per 32 pixels carried in order, so the sums are the same in every run); the other blocks of
// the `nblocks` subtract the moving image's shift from every quad's constant term, so that the
// sweep's bilinear values are shifted already.
__device__ __forceinline__ void span_prep_body(const SpanPrepArgs &a, int block, int nblocks) {
    if (block >= a.row_blocks) {
        const float ms = a.shifts[1];
        const int64_t nthr = (int64_t)(nblocks - a.row_blocks) * blockDim.x;
        for (int64_t i = (int64_t)(block - a.row_blocks) * blockDim.x + threadIdx.x; i < a.nquads; i += nthr)
            a.quads[i].x -= ms;
        return;
    }
    const int row = (int)((block * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (row >= a.fh) return;
    const int fw = a.fw;
    const float *src = a.fix + (int64_t)row * a.fpitch;
    double2 *dst = a.prefix + (int64_t)row * (fw + 1);
    if (lane == 0) dst[0] = make_double2(0.0, 0.0);
    double c1 = 0.0, c2 = 0.0;
    for (int x0 = 0; x0 < fw; x0 += 32) {
        const int x = x0 + lane;
        double v = x < fw ? (double)src[x] : 0.0;
        double v2 = v * v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double t1 = __shfl_up_sync(0xffffffffu, v, o), t2 = __shfl_up_sync(0xffffffffu, v2, o);
            if (lane >= o) {
                v += t1;
                v2 += t2;
            }
        }
        if (x < fw) dst[x + 1] = make_double2(c1 + v, c2 + v2);
        c1 += __shfl_sync(0xffffffffu, v, 31);
        c2 += __shfl_sync(0xffffffffu, v2, 31);
    }
}

static __global__ void __launch_bounds__(256) span_prep_kernel(const SpanPrepArgs a) {
    span_prep_body(a, (int)blockIdx.x, (int)gridDim.x);
}

// The staging step of many pairs at once: pair blockIdx.y, its blocks blockIdx.x (gridDim.x
// exceeds every pair's row_blocks).
static __global__ void __launch_bounds__(256) span_prep_batch_kernel(const SpanPrepArgs *__restrict__ args) {
    span_prep_body(args[blockIdx.y], (int)blockIdx.x, (int)gridDim.x);
}

// ---------------------------------------------------------------- the multi-pair span kernel
//
// Batches: the tasks of many ZNCC pairs (each with its own staged planes, prefix sums, tiles
// and grid) from one counter, so that pairs too small to fill the GPU alone share it.  A
// task's pair is found in the prefix of task counts; its parameters are read from global
// memory.  Shared memory is carved once for the largest tile count of the pairs and one window
// stage size (`cap`) for all of them; each pair's results are those of span_kernel on that pair.
template <int G, int NW, int TX, bool CHECK>
__global__ void __launch_bounds__(NW * 32, 1) span_batch_kernel(const __grid_constant__ SpanBatchParams b) {
    extern __shared__ __align__(128) unsigned char smem[];
    const SpanSmem ss = carve_span<G, NW>(smem, b.tile_h, TX, b.tiles, b.cap);
    // the task word sits in the carve's head, after the flags (no static shared memory: the
    // dynamic carve may take all 227 KB)
    volatile uint32_t &s_task = *reinterpret_cast<volatile uint32_t *>(ss.bounds_flag + 1);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kWinStages; s++) mbar_init(&ss.bars[s], 1);
        fence_mbar_init();
        *ss.abort_flag = 0;
        *ss.bounds_flag = 0;
    }
    uint32_t wit = 0;
    for (;;) {
        __syncthreads();  // the previous task is done with s_task
        if (threadIdx.x == 0) s_task = atomicAdd(b.next_task, 1u);
        __syncthreads();
        const uint32_t t = s_task;
        if (t >= b.total_tasks) return;
        uint32_t lo = 0, hi = b.n_pairs;  // task_begin[lo] <= t < task_begin[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(b.task_begin + mid) <= t) lo = mid;
            else hi = mid;
        }
        const SearchParams &p = b.pairs[lo];
        const uint32_t slot = __ldg(b.slot + lo);
        if (threadIdx.x == 0 && b.t_start) atomicMin(b.t_start + slot, (unsigned long long)global_ns());
        if (!run_span_task<G, NW, TX, CHECK>(p, t - __ldg(b.task_begin + lo), ss, wit)) {
            if (threadIdx.x == 0) {
                // retire this task and every task not yet taken, with the timeout status
                retire_tasks(p, ~0ull, 1u, true);
                for (;;) {
                    const uint32_t u = atomicAdd(b.next_task, 1u);
                    if (u >= b.total_tasks) break;
                    uint32_t l2 = 0, h2 = b.n_pairs;
                    while (h2 - l2 > 1) {
                        const uint32_t mid = (l2 + h2) >> 1;
                        if (__ldg(b.task_begin + mid) <= u) l2 = mid;
                        else h2 = mid;
                    }
                    retire_tasks(b.pairs[l2], ~0ull, 1u, true);
                }
            }
            return;
        }
        if (threadIdx.x == 0 && b.t_end) atomicMax(b.t_end + slot, (unsigned long long)global_ns());
    }
}

}  // namespace cgs
