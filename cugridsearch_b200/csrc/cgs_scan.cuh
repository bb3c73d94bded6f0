// cgs_scan.cuh -- the scanline functors calcNCCAlt, calcSQDAlt and calcMIAlt on sm_100a.
//
// These reference functors (src/gpu/cudaErrorFunctions.cuh:226-376,
// src/gpu/cudaErrorFunction_mi.cuh:117-255) do not loop over fixed pixels: for each fixed row
// they intersect the row's image under the homography with the moving image
// (parametricAssignValues[Norm], cudaImageFunctions.cuh:315-441), then step a float lambda
// along the row by repeated addition, sampling the moving image at lambda * v + p0 and the
// fixed image at (row, lambda).  Which samples exist, where they lie and the overlap gates
// all follow float recurrences; cgs_seq.cuh reproduces those recurrences exactly, so each
// lane can jump straight to its own lambda.
//
// Work layout: one warp per grid point (persistent over grid points in the locality order of
// the pixel kernel).  For each block of 32 rows every lane sets up one row (the exact
// intersection, ~100 correctly rounded operations), the warp then walks the rows, lanes
// taking every 32nd lambda.  Both images are read through L1 from the staged planes, whose
// extra column and zero row make the reference's flat-index neighbours explicit.
#pragma once
#include "cgs_kernels.cuh"
#include "cgs_seq.cuh"

namespace cgs {

// parametersToHomographyNorm (src/gpu/cudaImageFunctions.cuh:181-214): integer size ratios,
// rounded integer centres (cmy from the moving WIDTH, :201), scale divided by the ratios.
__device__ __forceinline__ Homog h_norm(const float *q, float c, float s, int mw, int mh, int fw, int fh) {
    const float x_ratio = (float)(fw / mw), y_ratio = (float)(fh / mh);
    const float cfx = (float)(fw / 2), cfy = (float)(fh / 2), cmx = (float)(mw / 2), cmy = (float)(mw / 2);
    const float sx = xd(q[1], x_ratio), sy = xd(q[2], y_ratio), sh = q[3], tx = q[4], ty = q[5];
    Homog h;
    h.h11 = xm(sx, c);
    h.h12 = xs(xm(xm(sy, sh), c), xm(sy, s));
    h.h13 = xd(xa(xs(tx, cfx), cmx), (float)fw);
    h.h21 = xm(sx, s);
    h.h22 = xa(xm(xm(sy, sh), s), xm(sy, c));
    h.h23 = xd(xa(xs(ty, cfy), cmy), (float)fh);
    h.h31 = q[6];
    h.h32 = q[7];
    return h;
}

struct RowInfo {
    float ls, le;        // first lambda, exclusive lambda limit (min of the reference's two bounds)
    float vx, vy, p0x, p0y;
    float mag;           // |v| (calcNCCAlt/calcSQDAlt mov_area increment)
    float rowv;          // fixed-image row coordinate of the samples
    uint32_t n;          // number of lambda samples (0 when the row misses the moving image)
    int nseg;            // lambda segments; -1: more than kMaxSegs (lanes step explicitly)
};

constexpr int kMaxSegs = 24;

// parametricAssignValues (cudaImageFunctions.cuh:315-376) in the reference's operation order.
__device__ inline void assign_values(const Homog &H, int m_width, int m_height, int f_width, int f_height, int row_i,
                                     float &ls, float &le, float &v_x, float &v_y, float &p0_x, float &p0_y,
                                     bool &in) {
    const float h11 = H.h11, h12 = H.h12, h13 = H.h13, h21 = H.h21, h22 = H.h22, h23 = H.h23, h31 = H.h31,
                h32 = H.h32;
    const float row = (float)row_i, fw = (float)f_width, mh = (float)m_height, mw = (float)m_width;
    const float D = xs(xa(xa(xs(xs(xm(h11, h22), xm(h12, h21)), xm(xm(h11, h23), h32)), xm(xm(h12, h23), h31)),
                          xm(xm(h13, h21), h32)),
                       xm(xm(h13, h22), h31));
    const float den1 = xa(xs(xs(xm(h11, h22), xm(h12, h21)), xm(xm(h11, h32), row)), xm(xm(h12, h31), row));
    const float den2 = xa(xs(xs(xa(xs(xm(h11, h22), xm(h12, h21)), xm(xm(fw, h21), h32)), xm(xm(fw, h22), h31)),
                             xm(xm(h11, h32), row)),
                          xm(xm(h12, h31), row));
    const float dd = xm(den1, den2);
    v_x = xd(xm(xs(h22, xm(h32, row)), D), dd);
    v_y = xd(-xm(xs(h21, xm(h31, row)), D), dd);
    const float pden = xa(xs(xm(h12, h21), xm(h11, h22)), xm(row, xs(xm(h11, h32), xm(h12, h31))));
    p0_x = xd(xa(xs(xm(h13, h22), xm(h12, h23)), xm(row, xs(h12, xm(h13, h32)))), pden);
    p0_y = xd(-xa(xs(xm(h13, h21), xm(h11, h23)), xm(row, xs(h11, xm(h13, h31)))), pden);
    const float a21 = xs(h21, xm(h31, row)), a22 = xs(h22, xm(h32, row));
    const float inner1 = xa(xs(xs(xm(h11, h23), xm(h13, h21)), xm(h11, row)), xm(xm(h13, h31), row));
    const float lambda_top = xd(-xm(inner1, den2), xm(a21, D));
    const float x_top_ipt = xd(-xs(h23, row), a21);
    const float inner2 =
        xa(xs(xa(xs(xa(xs(xs(xm(h11, h23), xm(h13, h21)), xm(h11, row)), xm(xm(h11, h22), mh)), xm(xm(h12, h21), mh)),
                 xm(xm(h13, h31), row)),
              xm(xm(xm(h11, h32), mh), row)),
           xm(xm(xm(h12, h31), mh), row));
    const float lambda_bottom = xd(-xm(den2, inner2), xm(a21, D));
    const float x_bottom_ipt = xd(-xs(xa(xs(h23, row), xm(h22, mh)), xm(xm(h32, mh), row)), a21);
    const float inner3 = xa(xs(xs(xm(h12, h23), xm(h13, h22)), xm(h12, row)), xm(xm(h13, h32), row));
    const float lambda_left = xd(-xm(inner3, den2), xm(a22, D));
    const float y_left_ipt = xd(-xs(h23, row), a22);
    const float inner4 =
        xs(xa(xa(xa(xs(xs(xs(xm(h12, h23), xm(h13, h22)), xm(h12, row)), xm(xm(h11, h22), mw)), xm(xm(h12, h21), mw)),
                 xm(xm(h13, h32), row)),
              xm(xm(xm(h11, h32), mw), row)),
           xm(xm(xm(h12, h31), mw), row));
    const float lambda_right = xd(-xm(den2, inner4), xm(a22, D));
    const float y_right_ipt = xd(-xs(xa(xs(h23, row), xm(h21, mw)), xm(xm(h31, mw), row)), a22);
    if (x_top_ipt >= 0 && x_top_ipt < m_width && lambda_top >= 0 && lambda_top < f_width) {
        if (v_y > 0) ls = lambda_top; else le = lambda_top;
        in = true;
    }
    if (x_bottom_ipt >= 0 && x_bottom_ipt < m_width && lambda_bottom >= 0 && lambda_bottom < f_width) {
        if (v_y < 0) ls = lambda_bottom; else le = lambda_bottom;
        in = true;
    }
    if (y_left_ipt >= 0 && y_left_ipt < m_height && lambda_left >= 0 && lambda_left < f_height) {
        if (v_x > 0) ls = lambda_left; else le = lambda_left;
        in = true;
    }
    if (y_right_ipt >= 0 && y_right_ipt < m_height && lambda_right >= 0 && lambda_right < f_height) {
        if (v_x < 0) ls = lambda_right; else le = lambda_right;
        in = true;
    }
}

// parametricAssignValuesNorm (cudaImageFunctions.cuh:378-441) in the reference's order.
__device__ inline void assign_values_norm(const Homog &H, float row, float &ls, float &le, float &v_x, float &v_y,
                                          float &p0_x, float &p0_y, bool &in) {
    const float h11 = H.h11, h12 = H.h12, h13 = H.h13, h21 = H.h21, h22 = H.h22, h23 = H.h23, h31 = H.h31,
                h32 = H.h32;
    const float col = -0.5f;
    const float D = xs(xa(xa(xs(xs(xm(h11, h22), xm(h12, h21)), xm(xm(h11, h23), h32)), xm(xm(h12, h23), h31)),
                          xm(xm(h13, h21), h32)),
                       xm(xm(h13, h22), h31));
    const float a21 = xs(h21, xm(h31, row)), a22 = xs(h22, xm(h32, row));
    v_y = xd(-a21, D);
    v_x = xd(a22, D);
    const float den = xs(xa(xs(xm(h11, h22), xm(h12, h21)), xm(col, xs(xm(h21, h32), xm(h22, h31)))),
                         xm(row, xs(xm(h11, h32), xm(h12, h31))));
    const float numx = xs(xa(xs(xm(h12, h23), xm(h13, h22)), xm(col, xs(h22, xm(h23, h32)))),
                          xm(row, xs(h12, xm(h13, h32))));
    const float numy = xs(xa(xs(xm(h11, h23), xm(h13, h21)), xm(col, xs(h21, xm(h23, h31)))),
                          xm(row, xs(h11, xm(h13, h31))));
    p0_x = xd(numx, den);
    p0_y = xd(-numy, den);
    const float qy = xd(numy, den), qx = xd(numx, den);
    const float two_h23 = xm(2.0f, h23), two_row = xm(2.0f, row);
    const float lambda_top = xd(-xm(xs(qy, 0.5f), D), a21);
    const float x_top_ipt = xd(xs(xa(xs(h22, two_h23), two_row), xm(h32, row)), xm(2.0f, a21));
    const float lambda_bottom = xd(-xm(xa(qy, 0.5f), D), a21);
    const float x_bottom_ipt = xd(-xs(xs(xa(h22, two_h23), two_row), xm(h32, row)), xm(2.0f, a21));
    const float lambda_left = xd(-xm(xa(qx, 0.5f), D), a22);
    const float y_left_ipt = xd(xs(xa(xs(h21, two_h23), two_row), xm(h31, row)), xm(2.0f, a22));
    const float lambda_right = xd(-xm(xs(qx, 0.5f), D), a22);
    const float y_right_ipt = xd(-xs(xs(xa(h21, two_h23), two_row), xm(h31, row)), xm(2.0f, a22));
    if (x_top_ipt > -0.5f && x_top_ipt < 0.5f && lambda_top >= 0 && lambda_top < 1) {
        if (v_y > 0) ls = lambda_top; else le = lambda_top;
        in = true;
    }
    if (x_bottom_ipt > -0.5f && x_bottom_ipt < 0.5f && lambda_bottom > 0 && lambda_bottom < 1) {
        if (v_y < 0) ls = lambda_bottom; else le = lambda_bottom;
        in = true;
    }
    if (y_left_ipt > -0.5f && y_left_ipt < 0.5f && lambda_left > 0 && lambda_left < 1) {
        if (v_x > 0) ls = lambda_left; else le = lambda_left;
        in = true;
    }
    if (y_right_ipt > -0.5f && y_right_ipt < 0.5f && lambda_right > 0 && lambda_right < 1) {
        if (v_x < 0) ls = lambda_right; else le = lambda_right;
        in = true;
    }
}

// CudaImage::valueAt_bilinear including its inImage test (0 outside), reference order.
__device__ __forceinline__ float value_exact(const float *pl, int pitch, float wf, float hf, float y, float x) {
    return in_image(y, x, wf, hf) ? bilinear_in(pl, pitch, y, x) : 0.0f;
}

// The same value with fused interpolation (for sums, where only FP32 accuracy matters).
__device__ __forceinline__ float value_fast(const float *pl, int pitch, float wf, float hf, float y, float x) {
    if (!in_image(y, x, wf, hf)) return 0.0f;
    const float fy = floorf(y), fx = floorf(x);
    const float *q = pl + (int)fx + pitch * (int)fy;
    const float v00 = __ldg(q), v01 = __ldg(q + 1), v10 = __ldg(q + pitch), v11 = __ldg(q + pitch + 1);
    const float ax = x - fx, ay = y - fy;
    const float top = fmaf(ax, v01 - v00, v00), bot = fmaf(ax, v11 - v10, v10);
    return fmaf(ay, bot - top, top);
}

constexpr int kScanRows = 32;  // rows set up per block (one per lane)
constexpr int kScanWarps = 8;  // warps per CTA (one grid point each)

template <int COST, int C, int NW>
__global__ void __launch_bounds__(NW * 32, 1) scan_kernel(const __grid_constant__ SearchParams p) {
    constexpr bool kMI = (COST == CGS_COST_MI_ALT);
    constexpr bool kNCC = (COST == CGS_COST_NCC_ALT);
    constexpr int BN = 64;                 // calcMIAlt's bins
    constexpr int HS = BN + 1;             // padded row stride; row / column BN hold the marginals
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned long long *wbest = reinterpret_cast<unsigned long long *>(smem);
    RowInfo *rows_all = reinterpret_cast<RowInfo *>(smem + 8 * NW);
    Seg *segs_all = reinterpret_cast<Seg *>(rows_all + NW * kScanRows);
    uint32_t *hist_all = reinterpret_cast<uint32_t *>(segs_all + NW * kScanRows * kMaxSegs);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    RowInfo *rows = rows_all + warp * kScanRows;
    Seg *segs = segs_all + warp * kScanRows * kMaxSegs;
    uint32_t *hist = hist_all + (size_t)warp * HS * HS;
    const int fw = p.fix.w, fh = p.fix.h, mw = p.mov.w, mh = p.mov.h;
    const float fwf = (float)fw, fhf = (float)fh, mwf = p.mov_wf, mhf = p.mov_hf;
    const int nrows = kMI ? p.n_rows : fh;
    const double lam_inc = kMI ? (double)(1.0f / (float)(fw - 1)) : 1.0;
    const float lam_cap = kMI ? 1.0f : fwf;

    unsigned long long best = ~0ull;
    const uint32_t total_warps = gridDim.x * NW;
    for (uint32_t o = blockIdx.x * NW + warp; o < p.n; o += total_warps) {
        int32_t ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const uint32_t gidx = ordinal_to_index(p, o, ax);
        float q[8];
        grid_values(p, ax, q);
        const float2 cs = p.trig[min(ax[0], kMaxTrig - 1)];
        const Homog H = kMI ? h_norm(q, cs.x, cs.y, mw, mh, fw, fh) : h_centred(q, cs.x, cs.y, p.cx, p.cy);

        float out = 0.0f, i1 = 0.0f, i2 = 0.0f;  // lane partial sums (NCC/SQD)
        double mov_area_d = 0.0;                 // sum n_r * mag_r (lane 0)
        uint32_t steps = 0;                      // lambda steps over all rows (uniform)
        bool stalled = false;
        if constexpr (kMI) {
            for (int i = lane; i < HS * HS; i += 32) hist[i] = 0u;
        }
        __syncwarp();

        for (int rb = 0; rb < nrows; rb += kScanRows) {
            const int nb = min(kScanRows, nrows - rb);
            if (lane < nb) {
                RowInfo ri;
                ri.ls = 0.0f;
                ri.le = kMI ? 1.0f : fwf;
                ri.vx = ri.vy = ri.p0x = ri.p0y = 0.0f;
                bool in = false;
                if constexpr (kMI) {
                    const float rv = p.row_table[rb + lane];
                    assign_values_norm(H, rv, ri.ls, ri.le, ri.vx, ri.vy, ri.p0x, ri.p0y, in);
                    ri.rowv = __double2float_rn(((double)rv + 0.5) * (double)(fh - 1));
                    ri.mag = 0.0f;
                } else {
                    assign_values(H, mw, mh, fw, fh, rb + lane, ri.ls, ri.le, ri.vx, ri.vy, ri.p0x, ri.p0y, in);
                    ri.rowv = (float)(rb + lane);
                    ri.mag = __fsqrt_rn(xa(xm(ri.vx, ri.vx), xm(ri.vy, ri.vy)));
                }
                bool st = false, ovf = false;
                ri.nseg = 0;
                ri.n = in ? seq_segments(ri.ls, lam_inc, fminf(ri.le, lam_cap), segs + lane * kMaxSegs, kMaxSegs,
                                         ri.nseg, ovf, st)
                          : 0u;
                if (ovf) ri.nseg = -1;
                // a row has at most about W_f / step samples; anything else is a stalled
                // recurrence the reference would never leave
                const double max_n = (double)(kMI ? fw : fw) / fmin(lam_inc, 1.0) + 8.0;
                if ((double)ri.n > max_n) st = true;
                if (st) ri.n = 0u;
                rows[lane] = ri;
                stalled |= st;
            }
            __syncwarp();
            for (int rr = 0; rr < nb; rr++) {
                const RowInfo ri = rows[rr];
                if (ri.n == 0) continue;
                steps += ri.n;
                if (lane == 0 && !kMI) mov_area_d += (double)ri.n * (double)ri.mag;
                const Seg *rs = segs + rr * kMaxSegs;
                int cur = 0;
                float lam = ri.ls;
                bool ok = true;
                if (ri.nseg < 0 && lane < (int)ri.n) ok = seq_advance(lam, lam_inc, (uint32_t)lane);
                for (uint32_t k = lane; k < ri.n; k += 32) {
                    if (ri.nseg >= 0) lam = seq_value(rs, ri.nseg, cur, k);
                    const float nx0 = xa(xm(lam, ri.vx), ri.p0x);
                    const float ny0 = xa(xm(lam, ri.vy), ri.p0y);
#pragma unroll
                    for (int c = 0; c < C; c++) {
                        const float *mpl = p.mov.data + c * p.mov.plane;
                        const float *fpl = p.fix.data + c * p.fix.plane;
                        if constexpr (kMI) {
                            const float nx = __double2float_rn(((double)nx0 + 0.5) * (double)mw);
                            const float ny = __double2float_rn(((double)ny0 + 0.5) * (double)mh);
                            const float lamIdx = xm(lam, (float)(fw - 1));
                            const float vf = value_exact(fpl, p.fix.pitch, fwf, fhf, ri.rowv, lamIdx);
                            const float vm = value_exact(mpl, p.mov.pitch, mwf, mhf, ny, nx);
                            int bf = (int)floorf(xm(64.0f, xd(vf, 256.0f)));
                            int bm = (int)floorf(xm(64.0f, xd(vm, 256.0f)));
                            bf = min(max(bf, 0), BN - 1);
                            bm = min(max(bm, 0), BN - 1);
                            atomicAdd(&hist[bf * HS + bm], 1u);
                        } else {
                            const float vm = value_fast(mpl, p.mov.pitch, mwf, mhf, ny0, nx0) * (1.0f / 255.0f);
                            const float vf = value_fast(fpl, p.fix.pitch, fwf, fhf, ri.rowv, lam) * (1.0f / 255.0f);
                            if constexpr (kNCC) {
                                out = fmaf(vm, vf, out);
                            } else {
                                const float d = vm - vf;
                                out = fmaf(d, d, out);
                            }
                            i1 = fmaf(vm, vm, i1);
                            i2 = fmaf(vf, vf, i2);
                        }
                    }
                    if (ri.nseg < 0 && k + 32 < ri.n) ok &= seq_advance(lam, lam_inc, 32);
                }
                stalled |= !ok;
            }
            __syncwarp();
        }

        // ---- cost of this grid point
        float cost;
        if constexpr (kMI) {
            __syncwarp();
            // marginals: fixed (rows) into column BN, moving (columns) into row BN
            for (int i = lane; i < BN; i += 32) {
                uint32_t rs = 0, csum = 0;
                for (int j = 0; j < BN; j++) {
                    rs += hist[i * HS + j];
                    csum += hist[j * HS + i];
                }
                hist[i * HS + BN] = rs;
                hist[BN * HS + i] = csum;
            }
            __syncwarp();
            uint32_t cnt = 0;
            for (int i = lane; i < BN; i += 32) cnt += hist[i * HS + BN];
            cnt = (uint32_t)warp_sum_i((int)cnt);
            // the reference's float formula: P = n_xy / count, sum P (log2 P - (log2 Px + log2 Py))
            const float countf = (float)cnt;
            float s = 0.0f;
            for (int b = lane; b < BN * BN; b += 32) {
                const int i = b / BN, j = b - i * BN;
                const uint32_t v = hist[i * HS + j];
                if (v) {
                    const float P = (float)v / countf;
                    const float Px = (float)hist[i * HS + BN] / countf;
                    const float Py = (float)hist[BN * HS + j] / countf;
                    s += P * (log2f(P) - (log2f(Px) + log2f(Py)));
                }
            }
            s = warp_sum(s);
            // fix_area: one 1/(W_f H_f) per lambda step, accumulated as the reference does
            float fix_area = 0.0f;
            seq_advance(fix_area, 1.0 / (double)((int64_t)fw * fh), steps);
            cost = (-1.0f * s) * fix_area;
        } else {
            out = warp_sum(out);
            i1 = warp_sum(i1);
            i2 = warp_sum(i2);
            // gates (cudaErrorFunctions.cuh:296, 372): fix_area counts lambda steps exactly;
            // mov_area is a float running sum, decided from its double value unless that is
            // within the float sum's error bound of the threshold, then replayed exactly
            const float fix_area = (float)steps;
            const float den_m = xm((float)(p.mov.w * p.mov.h), q[2]);
            bool gate_fix = (double)xd(fix_area, (float)(fw * fh)) > 0.35;
            bool gate_mov = false;
            if (lane == 0) {
                const double ratio = mov_area_d / (double)den_m;
                const double margin = ((double)steps + 4.0) * 5.9604644775390625e-8 * fabs(ratio) + 1e-12;
                if (fabs(ratio - 0.25) > margin) {
                    gate_mov = ratio > 0.25;
                } else {
                    // exact replay of the reference's sequential float sum
                    float mov_area = 0.0f;
                    for (int r = 0; r < fh; r++) {
                        float ls = 0.0f, le = fwf, vx = 0, vy = 0, p0x = 0, p0y = 0;
                        bool in = false;
                        assign_values(H, mw, mh, fw, fh, r, ls, le, vx, vy, p0x, p0y, in);
                        if (!in) continue;
                        bool st;
                        const uint32_t n = seq_count_below(ls, 1.0, fminf(le, fwf), st);
                        const float mag = __fsqrt_rn(xa(xm(vx, vx), xm(vy, vy)));
                        seq_advance(mov_area, (double)mag, n);
                    }
                    gate_mov = (double)xd(mov_area, den_m) > 0.25;
                }
            }
            gate_mov = __shfl_sync(0xffffffffu, gate_mov, 0);
            if (gate_mov && gate_fix) {
                cost = kNCC ? xd(-out, __fsqrt_rn(xm(i1, i2))) : xd(out, __fsqrt_rn(xm(i1, i2)));
            } else {
                cost = 123123.0f;
            }
        }
        stalled = __any_sync(0xffffffffu, stalled);
        if (lane == 0) {
            if (stalled) atomicOr(p.status, (unsigned)CGS_ERROR_UNSUPPORTED);
            if (p.costs) p.costs[gidx] = cost;
            const unsigned long long kk = make_key(cost, gidx);
            best = kk < best ? kk : best;
        }
        __syncwarp();
    }

    if (lane == 0) wbest[warp] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long b = ~0ull;
        for (int w = 0; w < NW; w++) b = wbest[w] < b ? wbest[w] : b;
        if (b != ~0ull) atomicMin(p.key, b);
        __threadfence();
        const unsigned int ticket = atomicAdd(p.done, 1u);
        if (ticket == gridDim.x - 1) {
            __threadfence();
            write_result(p);
        }
    }
}

}  // namespace cgs
