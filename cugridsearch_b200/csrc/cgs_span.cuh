// cgs_span.cuh -- the span kernel: zero-mean NCC over fast samples, with the in/out decisions
// taken per image row instead of per sample, and the moving image's taps read from shared
// memory.
//
// Decisions per row.  For one grid point the map of a fixed row y is a projective line in the
// moving image; the samples that lie inside the moving image form one interval of x.  Solving
// the four half-plane conditions of "clearly inside" (a margin of 1.5 guard bands inside the
// image's edges, the guard being map_guard's bound between the fast and the reference's
// coordinates) and of "possibly inside" (1.5 guard bands outside) gives two integer spans per
// (row, point): every pixel of the inner span is inside for the reference too and takes the
// fast path with no test; pixels of the outer span outside the inner one (a band about a
// thousandth of a pixel wide around the overlap's edge, almost never a whole pixel) take the
// reference's exact operation sequence; every other pixel is outside and costs nothing.  The
// spans are computed in FP32; their rounding error is below a quarter of the guard band (the
// constraint terms are those the guard's own bound is built from), which the 1.5 factor covers.
//
// Tiles and windows.  The fixed image is walked in tiles of TW = 32 TX columns by TH rows.  For
// every tile the CTA's grid points map the tile into a small region of the moving image (the
// union of the tile's quadrilateral images, points of one task being neighbours in the
// locality order); that region of the staged tap quads is copied into shared memory by bulk
// copies, one per region row, into a two-stage mbarrier pipeline (the next tile's copies overlap
// the current tile's sweep), and the sweep reads its 16-byte quads from there.  A region larger
// than a stage is read from global memory instead (same values).
//
// Sweep.  Lane l takes the tile's columns x0 + l + 32 k; each warp evaluates its G grid points
// at every pixel, two points per packed FP32x2 instruction.  Rows whose inner spans cover the
// tile for every point run without any per-sample test; other rows mask samples by their spans
// and send the band pixels down the exact path.
//
// Sums.  Per lane, per band of TH rows: five FP32 sums per point of the shifted values
// f' = f - s_f, m' = m - s_m (the images' means; sum f', sum m', sum f'^2, sum m'^2, sum f'm'),
// reduced across the warp at the end of each band of tiles and accumulated in FP64; the cost is
// formed in FP64 (zncc_cost).  Which samples a lane sums, and in which order, depends only on the
// image and the tile shape, never on the points per warp or the warps per CTA: costs are
// bit-identical across those tunings.  The overlap count is the sum of the inner span lengths plus the band pixels
// found inside.
#pragma once
#include <type_traits>

#include "cgs_kernels.cuh"

namespace cgs {

constexpr int kWinStages = 2;
// kStatusSpanBounds (cgs_internal.h): status bit the self-checking build (CHECK = true) sets in
// the result when a fast sample's quad address fell outside the tile's window or the quad plane
// (the sample is then skipped).

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

// The moving-image window of one tile: quads [y0, y0 + h) x [x0, x0 + w) with row pitch `pitch`
// quads in the stage, after the tile's fixed rows; h == 0: no point samples the tile on the fast
// path; w < 0: the window does not fit a stage and the sweep reads global memory.
struct TileWin {
    int16_t x0, y0, w, h;
    int32_t pitch, pad;
};

// Spans of one (point, row): inner [xa, xa + len), outer [pa, pa + plen).
struct RowSpan {
    int16_t xa, len, pa, plen;
};

// One row of a warp's points: [ia, ib] lies in every point's inner span (empty if ia > ib),
// [ua, ub] holds every point's outer span (empty if ua > ub).
struct RowRun {
    int32_t ia, ib, ua, ub;
};

__host__ __device__ constexpr size_t span_head_bytes(int NW) { return 256 + 8 * (size_t)NW; }

// Shared-memory plan of the span kernel for NW warps of G points, TH-row bands, `tiles` tiles and
// a stage of `cap` quads.
__host__ __device__ constexpr size_t span_smem_bytes(int G, int NW, int TH, int tiles, int cap) {
    return span_head_bytes(NW) + (size_t)NW * G * sizeof(SpanSlot) + (size_t)NW * (G / 2) * sizeof(PairRow) +
           (size_t)tiles * sizeof(TileWin) + (size_t)NW * G * TH * sizeof(RowSpan) +
           (size_t)NW * TH * sizeof(RowRun) + (size_t)NW * G * (5 * sizeof(double) + sizeof(int)) +
           (size_t)kWinStages * cap * 16 + 128;
}

struct SpanSmem {
    uint64_t *bars;   // [kWinStages]
    unsigned long long *wbest;
    int *abort_flag;
    int *bounds_flag;  // self-checking build: a sample's quad address fell outside its window
    SpanSlot *slots;  // [NW * G]
    PairRow *prow;    // [NW * G / 2]
    TileWin *tiles;   // [tiles]
    RowSpan *spans;   // [NW][G][TH]
    RowRun *runs;     // [NW][TH]
    double *dtot;     // [NW][G * 5] FP64 task totals of the warps' points
    int *cnt;         // [NW][G] overlap counts of the warps' points
    float4 *win;      // [kWinStages][cap]
    int cap;
};

template <int G, int NW>
__device__ __forceinline__ SpanSmem carve_span(unsigned char *smem, int TH, int tiles, int cap) {
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
    s.tiles = reinterpret_cast<TileWin *>(q);
    q += (size_t)tiles * sizeof(TileWin);
    s.spans = reinterpret_cast<RowSpan *>(q);
    q += (size_t)NW * G * TH * sizeof(RowSpan);
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

// The corners of tile [x0, x1] x [y0, y1] under a point's map: min/max of the mapped coordinates.
__device__ __forceinline__ void tile_extent(const SpanSlot &k, float x0, float x1, float y0, float y1, float4 &e) {
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
// image's right edge are not copied) and the moving-image window (quads, after the fixed tile).
template <int TW>
__device__ __forceinline__ void issue_window(const SearchParams &p, const SpanSmem &ss, int t, int st) {
    const int lane = threadIdx.x & 31;
    const int TH = p.tile_h;
    const int x0 = (t % p.tiles_x) * TW, y0 = (t / p.tiles_x) * TH;
    const int rows = min(TH, p.fix.h - y0);
    const uint32_t row_bytes = (uint32_t)((min(TW, p.fix.w - x0) * 4 + 15) & ~15);  // within the row pitch
    const TileWin tw = ss.tiles[t];
    uint64_t *bar = &ss.bars[st];
    const bool copy = tw.h > 0 && tw.w > 0;
    if (lane == 0) {
        fence_proxy_async_smem();  // the stage's previous reads before the async refill
        mbar_arrive_expect_tx(bar, (uint32_t)rows * row_bytes + (copy ? (uint32_t)tw.w * (uint32_t)tw.h * 16u : 0u));
    }
    __syncwarp();
    fence_proxy_async_smem();
    float *fdst = reinterpret_cast<float *>(ss.win + (size_t)st * ss.cap);
    for (int j = lane; j < rows; j += 32)
        bulk_g2s(fdst + j * TW, p.fix.data + (int64_t)(y0 + j) * p.fix.pitch + x0, row_bytes, bar);
    if (copy) {
        float4 *dst = ss.win + (size_t)st * ss.cap + TH * TW / 4;
        const float4 *src = p.mov_quad + (int64_t)tw.y0 * p.quad_pitch + tw.x0;
        for (int j = lane; j < tw.h; j += 32)
            bulk_g2s(dst + (size_t)j * tw.pitch, src + (int64_t)j * p.quad_pitch, (uint32_t)tw.w * 16u, bar);
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
    const int qpitch = p.quad_pitch;
    const float4 *__restrict__ mquad = p.mov_quad;

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

    // ---- windows of every tile: warp w takes tiles w, w + NW, ..; lanes take the task's points
    {
        constexpr int P = NW * G;
        for (int t = warp; t < ntiles; t += NW) {
            const int x0 = (t % tiles_x) * TW, y0 = (t / tiles_x) * TH;
            const float fx0 = (float)x0, fx1 = (float)(min(x0 + TW, fw) - 1);
            const float fy0 = (float)y0, fy1 = (float)(min(y0 + TH, fh) - 1);
            float4 e = make_float4(__int_as_float(0x7f800000), __int_as_float(0x7f800000),
                                   -__int_as_float(0x7f800000), -__int_as_float(0x7f800000));
            for (int k = lane; k < P; k += 32) {
                const SpanSlot &sl = ss.slots[k];
                if (sl.ok) tile_extent(sl, fx0, fx1, fy0, fy1, e);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                e.x = fminf(e.x, __shfl_xor_sync(0xffffffffu, e.x, o));
                e.y = fminf(e.y, __shfl_xor_sync(0xffffffffu, e.y, o));
                e.z = fmaxf(e.z, __shfl_xor_sync(0xffffffffu, e.z, o));
                e.w = fmaxf(e.w, __shfl_xor_sync(0xffffffffu, e.w, o));
            }
            if (lane == 0) {
                TileWin tw{0, 0, 0, 0, 0, 0};
                // cells a fast sample can use: floor of its coordinate (within the guard, < 1/8 px,
                // of the real map, whose tile image lies in the corners' hull), clipped to the image
                const float lx = fmaxf(e.x - 0.25f, -1.0f), ly = fmaxf(e.y - 0.25f, -1.0f);
                const float hx = fminf(e.z + 0.25f, mov_wf), hy = fminf(e.w + 0.25f, mov_hf);
                if (lx <= hx && ly <= hy) {
                    const int cx0 = max(0, (int)floorf(lx)), cy0 = max(0, (int)floorf(ly));
                    const int cx1 = min(p.mov.w - 1, (int)floorf(hx)), cy1 = min(p.mov.h - 1, (int)floorf(hy));
                    if (cx0 <= cx1 && cy0 <= cy1) {
                        const int w = cx1 - cx0 + 1, h = cy1 - cy0 + 1;
                        const int pitch = w + ((p.win_pitch_mod - w) & 7);  // = win_pitch_mod (mod 8)
                        tw.x0 = (int16_t)cx0;
                        tw.y0 = (int16_t)cy0;
                        tw.h = (int16_t)h;
                        tw.w = (int16_t)((int64_t)pitch * h <= ss.cap - TH * TW / 4 ? w : -1);
                        tw.pitch = pitch;
                    }
                }
                ss.tiles[t] = tw;
            }
        }
    }
    __syncthreads();
    if (warp == 0) {
        for (int t = 0; t < kWinStages && t < ntiles; t++) issue_window<TW>(p, ss, t, (int)((wit + t) % kWinStages));
    }

    // ---- sweep
    float2 part[GP][5];
#pragma unroll
    for (int h = 0; h < GP; h++)
#pragma unroll
        for (int j = 0; j < 5; j++) part[h][j] = make_float2(0.0f, 0.0f);
    RowSpan *my_spans = ss.spans + warp * G * TH;
    RowRun *my_runs = ss.runs + warp * TH;
    const float2 magic2 = make_float2(kMagic, kMagic), nmagic2 = make_float2(-kMagic, -kMagic);
    const float2 minus1 = make_float2(-1.0f, -1.0f);
    const float2 shift2 = make_float2(-mshift, -mshift);

    for (int t = 0; t < ntiles; t++, wit++) {
        const int tx = t % tiles_x, ty = t / tiles_x;
        const int x0 = tx * TW, y0 = ty * TH;
        const int x1 = min(x0 + TW, fw) - 1;
        if (tx == 0) {
            // spans of the band's rows, every point of the warp; inner lengths count the overlap
            for (int i = lane; i < G * TH; i += 32) {
                const int g = i / TH, r = i - g * TH;
                const SpanSlot &sl = my_slots[g];
                const int y = y0 + r;
                RowSpan rs{0, 0, 0, 0};
                if (y < fh && sl.valid) {
                    if (sl.ok) {
                        const float yf = (float)y;
                        const float wm = fmaf(sl.A, 0.5f * (float)(fw - 1), fmaf(sl.B, yf, sl.PQ));
                        const float s = wm > 0.0f ? 1.0f : -1.0f;
                        int xa, len, pa, plen;
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
                        rs = RowSpan{(int16_t)xa, (int16_t)len, (int16_t)pa, (int16_t)plen};
                        if (len > 0) atomicAdd(&my_cnt[g], len);
                    } else {
                        rs = RowSpan{0, 0, 0, (int16_t)fw};  // ill-conditioned: every pixel exact
                    }
                }
                my_spans[g * TH + r] = rs;
            }
            __syncwarp();
            if (lane < TH) {  // the rows' common inner run and outer hull over the warp's points
                int ia = 0, ib = fw - 1, ua = 1 << 15, ub = -1;
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const RowSpan rs = my_spans[g * TH + lane];
                    if (my_slots[g].valid && rs.len > 0) {
                        ia = max(ia, (int)rs.xa);
                        ib = min(ib, rs.xa + rs.len - 1);
                    } else {
                        ib = -1;  // a point without an inner span (or outside the grid): no common run
                    }
                    if (rs.plen > 0) {
                        ua = min(ua, (int)rs.pa);
                        ub = max(ub, rs.pa + rs.plen - 1);
                    }
                }
                my_runs[lane] = RowRun{ia, ib, ua, ub};
            }
            __syncwarp();
        }
        // the tile's window
        const int st = (int)(wit % kWinStages);
        if (!mbar_wait_bounded(&ss.bars[st], (wit / kWinStages) & 1u, kWaitLimitNs)) *ss.abort_flag = 1;
        const TileWin tw = ss.tiles[t];
        const bool in_smem = tw.w > 0;
        // index of quad (ix, iy) from the bits of tx = ix + 1.5 * 2^23, ty = iy + 1.5 * 2^23: in the
        // window, bx + pitch * by - wK = (ix - x0) + pitch * (iy - y0); in the plane, bx + qpitch *
        // by - gK = ix + qpitch * iy (both mod 2^32, exact for in-image cells)
        const float *sfix = reinterpret_cast<const float *>(ss.win + (size_t)st * ss.cap);  // TH x TW
        // shared address of window quad (ix, iy): sbase + 16 bx + 16 pitch by (mod 2^32)
        const uint32_t wpitch = (uint32_t)tw.pitch;
        const uint32_t spitch16 = 16u * wpitch;
        const uint32_t sbase = smem_addr(ss.win + (size_t)st * ss.cap + TH * TW / 4) -
                               16u * ((uint32_t)tw.x0 + wpitch * (uint32_t)tw.y0 + (uint32_t)kMagicBits * (1u + wpitch));
        const uint32_t szero = smem_addr(ss.win);
        const uint32_t gK = (uint32_t)kMagicBits * (1u + (uint32_t)qpitch);

        // one row: fast samples of G points at the lane's columns; EDGE masks by the spans
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
            // one block of 32 columns; EDGE: some column may lie outside a point's inner span
            auto column = [&](int c, auto edge_tag) {
                constexpr bool EDGE = decltype(edge_tag)::value;
                RowSpan rsp[G];
                if constexpr (EDGE) {
#pragma unroll
                    for (int g = 0; g < G; g++) rsp[g] = my_spans[g * TH + r];
                }
                const int x = x0 + 32 * c + lane;
                const float f = frow[32 * c + lane];  // past the image's right edge: not copied, unused
                const float fs = f - fshift;
                const float xf = (float)x;
                const float2 xf2 = make_float2(xf, xf);
                bool amb_any = false;
                bool amb[G];
#pragma unroll
                for (int h = 0; h < GP; h++) {
                    // both points of the pair in each FP32x2 operation: map, floor (round-down add
                    // of 1.5 * 2^23 leaves floor(m) in the mantissa), fraction
                    const float2 w = __ffma2_rn(A2[h], xf2, byw[h]);
                    const float2 X = __ffma2_rn(C12[h], xf2, byx[h]);
                    const float2 Y = __ffma2_rn(D12[h], xf2, byy[h]);
                    const float2 rw = make_float2(rcp_approx(w.x), rcp_approx(w.y));
                    const float2 mx = __fmul2_rn(X, rw), my = __fmul2_rn(Y, rw);
                    const float2 tx2 = __fadd2_rd(mx, magic2), ty2 = __fadd2_rd(my, magic2);
                    const float2 fx2 = __fadd2_rn(tx2, nmagic2), fy2 = __fadd2_rn(ty2, nmagic2);
                    const float2 ax2 = __ffma2_rn(fx2, minus1, mx), ay2 = __ffma2_rn(fy2, minus1, my);
                    const float2 axy0 = make_float2(ax2.x, ay2.x), axy1 = make_float2(ax2.y, ay2.y);
                    const float2 txy0 = make_float2(tx2.x, ty2.x), txy1 = make_float2(tx2.y, ty2.y);
                    bool in0 = true, in1 = true;
                    if constexpr (EDGE) {
                        const RowSpan a = rsp[2 * h], b = rsp[2 * h + 1];
                        in0 = (unsigned)(x - a.xa) < (unsigned)a.len;
                        in1 = (unsigned)(x - b.xa) < (unsigned)b.len;
                        amb[2 * h] = !in0 && (unsigned)(x - a.pa) < (unsigned)a.plen;
                        amb[2 * h + 1] = !in1 && (unsigned)(x - b.pa) < (unsigned)b.plen;
                        amb_any |= amb[2 * h] | amb[2 * h + 1];
                    }
                    float v0, v1;
                    {
                        const uint32_t bx0 = __float_as_uint(txy0.x), by0 = __float_as_uint(txy0.y);
                        const uint32_t bx1 = __float_as_uint(txy1.x), by1 = __float_as_uint(txy1.y);
                        float4 q0, q1;
                        if (in_smem) {
                            uint32_t a0 = sbase + by0 * spitch16 + bx0 * 16u;
                            uint32_t a1 = sbase + by1 * spitch16 + bx1 * 16u;
                            if constexpr (EDGE) {
                                a0 = in0 ? a0 : szero;
                                a1 = in1 ? a1 : szero;
                            }
                            if constexpr (CHECK) {  // inside the tile's window, else recorded and skipped
                                const bool b0 = in0 && ((unsigned)((int)(bx0 - (uint32_t)kMagicBits) - tw.x0) >= (unsigned)tw.w ||
                                                        (unsigned)((int)(by0 - (uint32_t)kMagicBits) - tw.y0) >= (unsigned)tw.h);
                                const bool b1 = in1 && ((unsigned)((int)(bx1 - (uint32_t)kMagicBits) - tw.x0) >= (unsigned)tw.w ||
                                                        (unsigned)((int)(by1 - (uint32_t)kMagicBits) - tw.y0) >= (unsigned)tw.h);
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
                            uint32_t o0 = bx0 + by0 * (uint32_t)qpitch - gK;
                            uint32_t o1 = bx1 + by1 * (uint32_t)qpitch - gK;
                            if constexpr (EDGE) {
                                o0 = in0 ? o0 : 0u;
                                o1 = in1 ? o1 : 0u;
                            }
                            if constexpr (CHECK) {  // inside the moving image, else recorded and skipped
                                const bool b0 = (unsigned)((int)(bx0 - (uint32_t)kMagicBits)) >= (unsigned)p.mov.w ||
                                                (unsigned)((int)(by0 - (uint32_t)kMagicBits)) >= (unsigned)p.mov.h;
                                const bool b1 = (unsigned)((int)(bx1 - (uint32_t)kMagicBits)) >= (unsigned)p.mov.w ||
                                                (unsigned)((int)(by1 - (uint32_t)kMagicBits)) >= (unsigned)p.mov.h;
                                if ((in0 && b0) | (in1 && b1)) *ss.bounds_flag = 1;
                                o0 = (in0 && b0) ? 0u : o0;
                                o1 = (in1 && b1) ? 0u : o1;
                            }
                            q0 = __ldg(mquad + o0);
                            q1 = __ldg(mquad + o1);
                        }
                        // quad = {left column, its differences to the right column}: the row lerps
                        const float t0 = fmaf(axy0.x, q0.z, q0.x), b0 = fmaf(axy0.x, q0.w, q0.y);
                        const float t1 = fmaf(axy1.x, q1.z, q1.x), b1 = fmaf(axy1.x, q1.w, q1.y);
                        v0 = fmaf(axy0.y, b0 - t0, t0);
                        v1 = fmaf(axy1.y, b1 - t1, t1);
                    }
                    float2 ms = __fadd2_rn(make_float2(v0, v1), shift2);
                    float2 fm2 = make_float2(fs, fs);
                    if constexpr (EDGE) {
                        ms = make_float2(in0 ? ms.x : 0.0f, in1 ? ms.y : 0.0f);
                        fm2 = make_float2(in0 ? fs : 0.0f, in1 ? fs : 0.0f);
                    }
                    part[h][0] = __fadd2_rn(part[h][0], fm2);
                    part[h][1] = __fadd2_rn(part[h][1], ms);
                    part[h][2] = __ffma2_rn(fm2, fm2, part[h][2]);
                    part[h][3] = __ffma2_rn(ms, ms, part[h][3]);
                    part[h][4] = __ffma2_rn(fm2, ms, part[h][4]);
                }
                if constexpr (EDGE) {
                    // band pixels: the reference's exact operation sequence decides and samples
                    if (__any_sync(0xffffffffu, amb_any)) {
#pragma unroll
                        for (int g = 0; g < G; g++) {
                            if (amb[g]) {
                                const SpanSlot &sl = my_slots[g];
                                const MapCoef kc{sl.A, sl.B, sl.P, sl.Q, sl.C1, sl.C2, sl.R, sl.S,
                                                 sl.D1, sl.D2, sl.T, sl.U};
                                float ex, ey;
                                exact_map(kc, xf, yf, ex, ey);
                                if (in_image(ey, ex, mov_wf, mov_hf)) {
                                    const float m = bilinear_in(mdata, mpitch, ey, ex) - mshift;
                                    if (g & 1) {
                                        part[g / 2][0].y += fs;
                                        part[g / 2][1].y += m;
                                        part[g / 2][2].y = fmaf(fs, fs, part[g / 2][2].y);
                                        part[g / 2][3].y = fmaf(m, m, part[g / 2][3].y);
                                        part[g / 2][4].y = fmaf(fs, m, part[g / 2][4].y);
                                    } else {
                                        part[g / 2][0].x += fs;
                                        part[g / 2][1].x += m;
                                        part[g / 2][2].x = fmaf(fs, fs, part[g / 2][2].x);
                                        part[g / 2][3].x = fmaf(m, m, part[g / 2][3].x);
                                        part[g / 2][4].x = fmaf(fs, m, part[g / 2][4].x);
                                    }
                                    atomicAdd(&my_cnt[g], 1);
                                }
                            }
                        }
                    }
                }
            };
            // blocks of 32 columns inside every point's inner span run unmasked
#pragma unroll 1
            for (int c = 0; c < TX; c++) {
                const int xc = x0 + 32 * c;
                if (xc > run.ub || xc + 31 < run.ua) continue;  // no point samples these columns
                if (xc >= run.ia && xc + 31 <= run.ib) column(c, std::false_type{});
                else column(c, std::true_type{});
            }
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
                for (int j = 0; j < 5; j++) {
                    const float s0 = warp_sum(part[h][j].x), s1 = warp_sum(part[h][j].y);
                    const int i0 = (2 * h) * 5 + j, i1 = (2 * h + 1) * 5 + j;
                    if (lane == 0) {
                        my_dtot[i0] += (double)s0;
                        my_dtot[i1] += (double)s1;
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
        if (warp == 0 && t + kWinStages < ntiles) issue_window<TW>(p, ss, t + kWinStages, st);
    }

    // ---- per grid point: finalise, dump, argmin key (as the pixel-loop kernel)
    __syncwarp();
    unsigned long long kk = ~0ull;
    if (lane < G) {
        const SpanSlot &sl = my_slots[lane];
        double a[5];
#pragma unroll
        for (int j = 0; j < 5; j++) a[j] = my_dtot[lane * 5 + j];
        const float cost = zncc_cost(a, my_cnt[lane], p);
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
    const SpanSmem ss = carve_span<G, NW>(smem, p.tile_h, p.tiles_x * p.tiles_y, p.win_cap);
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

}  // namespace cgs
