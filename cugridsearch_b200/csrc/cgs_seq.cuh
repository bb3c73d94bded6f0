// cgs_seq.cuh -- closed forms of the reference's float recurrences x_{k+1} = fl(x_k + inc).
//
// The scanline functors step their sample positions and areas by repeated float addition
// (calcNCCAlt/calcSQDAlt: lambda += 1, mov_area += mag_norm, cudaErrorFunctions.cuh:272,289;
// calcMIAlt: lambda += 1/(colsf-1), fix_area += 1.0/(colsf*rowsf), cudaErrorFunction_mi.cuh:179,201).
// Each step rounds, so x_k is not x_0 + k*inc.  It is, however, piecewise arithmetic: while x
// stays in one binade [2^e, 2^(e+1)) every value is a multiple of that binade's ulp u, and
// fl(x + inc) = x + d with d = inc rounded to a multiple of u -- unless inc lies exactly half
// way between two multiples, when round-to-even makes the step depend on x's last bit.  So
// x_k is found by walking binades: whole runs of d inside a binade, one explicitly rounded
// step across each boundary, and explicit steps on ties.  Every value involved is exact in
// double.  Non-negative x only (all uses start at x_0 >= 0 and add inc > 0).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#define CGS_HD __host__ __device__

namespace cgs {

// One reference step: the exact sum rounded to float once (float + float, or float + double
// followed by the conversion back to float -- both round the exact sum once).
CGS_HD __forceinline__ float seq_step(float x, double inc) {
#ifdef __CUDA_ARCH__
    return __double2float_rn((double)x + inc);
#else
    return (float)((double)x + inc);
#endif
}

// ulp of a positive float, and the end of its binade.
CGS_HD __forceinline__ void binade(float x, double &u, double &top) {
#ifdef __CUDA_ARCH__
    const int bits = __float_as_int(x);
#else
    int bits;
    memcpy(&bits, &x, 4);
#endif
    const int ef = (bits >> 23) & 0xff;
    if (ef == 0) {  // subnormal: fixed spacing 2^-149 up to 2^-126
        u = ldexp(1.0, -149);
        top = ldexp(1.0, -126);
        return;
    }
    const int e = ef - 127;
    u = ldexp(1.0, e - 23);
    top = ldexp(1.0, e + 1);
}

// inc rounded to a multiple of u (nearest); tie = inc exactly half way.
CGS_HD __forceinline__ double round_to(double inc, double u, bool &tie) {
    const double q = inc / u;  // exact: u is a power of two
    const double f = floor(q);
    const double r = q - f;
    tie = (r == 0.5);
    return (r < 0.5 ? f : f + 1.0) * u;
}

// Largest j >= 0 with x + j*d <= lim (lim >= x); the quotient is corrected in exact arithmetic.
CGS_HD __forceinline__ double steps_upto(double x, double d, double lim) {
    double j = floor((lim - x) / d);
    if (j < 0.0) j = 0.0;
    while (x + (j + 1.0) * d <= lim) j += 1.0;
    while (j > 0.0 && x + j * d > lim) j -= 1.0;
    return j;
}

// Largest j >= 0 with x + j*d < lim (lim > x).
CGS_HD __forceinline__ double steps_below(double x, double d, double lim) {
    double j = ceil((lim - x) / d) - 1.0;
    if (j < 0.0) j = 0.0;
    while (x + (j + 1.0) * d < lim) j += 1.0;
    while (j > 0.0 && x + j * d >= lim) j -= 1.0;
    return j;
}

// x_k of the recurrence from x_0 = x.  Returns false if the sequence stalls (an increment
// rounds to zero: the reference would loop forever) before k steps.
CGS_HD inline bool seq_advance(float &x, double inc, uint32_t k) {
    while (k > 0) {
        if (x == 0.0f) {
            x = seq_step(x, inc);
            k--;
            continue;
        }
        double u, top;
        binade(x, u, top);
        bool tie;
        const double d = round_to(inc, u, tie);
        if (tie) {
            const float x1 = seq_step(x, inc);
            if (x1 == x) return false;
            x = x1;
            k--;
            continue;
        }
        if (d == 0.0) return false;
        const double n_in = steps_upto((double)x, d, top - u);  // steps that stay in this binade
        if (n_in >= 1.0) {
            const uint32_t m = (double)k < n_in ? k : (uint32_t)n_in;
            x = (float)((double)x + (double)m * d);  // exact: a multiple of u inside the binade
            k -= m;
            if (k == 0) return true;
        }
        x = seq_step(x, inc);  // the step across the boundary
        k--;
    }
    return true;
}

// Number of k >= 0 with x_k < limit (the sequence is non-decreasing).  stalled is set when
// the reference's loop would not terminate.
CGS_HD inline uint32_t seq_count_below(float x, double inc, float limit, bool &stalled) {
    stalled = false;
    if (!(x < limit)) return 0;
    uint32_t count = 1;  // x_0
    for (int guard = 0; guard < 4096; guard++) {
        // here x = x_{count-1} < limit
        if (x == 0.0f) {
            x = seq_step(x, inc);
            if (!(x < limit)) return count;
            count++;
            continue;
        }
        double u, top;
        binade(x, u, top);
        bool tie;
        const double d = round_to(inc, u, tie);
        if (tie) {
            const float x1 = seq_step(x, inc);
            if (x1 == x) { stalled = true; return count; }
            if (!(x1 < limit)) return count;
            count++;
            x = x1;
            continue;
        }
        if (d == 0.0) { stalled = true; return count; }
        const double n_in = steps_upto((double)x, d, top - u);
        const double n_lim = steps_below((double)x, d, (double)limit);
        if (n_lim < n_in) return count + (uint32_t)n_lim;  // the limit comes inside this binade
        count += (uint32_t)n_in;
        x = (float)((double)x + n_in * d);
        const float x1 = seq_step(x, inc);  // across the boundary
        if (!(x1 < limit)) return count;
        count++;
        x = x1;
    }
    stalled = true;
    return count;
}

// The sequence as arithmetic segments: x_k = x0 + (k - k0) * d for k0 <= k < next segment's
// k0, each result exactly representable, so one fused multiply-add evaluates it exactly.
struct Seg {
    uint32_t k0;
    float x0, d;
};

// Builds the segments of x_0 = x, ..., x_{n-1} (the values below limit) into segs (at most
// max_segs) and returns n.  overflow is set if more segments were needed (segs then covers a
// prefix); stalled if the reference's loop would not terminate.
CGS_HD inline uint32_t seq_segments(float x, double inc, float limit, Seg *segs, int max_segs, int &nseg,
                                    bool &overflow, bool &stalled) {
    nseg = 0;
    overflow = false;
    stalled = false;
    if (!(x < limit)) return 0;
    uint32_t k = 0;  // index of x
    for (int guard = 0; guard < 4096; guard++) {
        if (nseg == max_segs) overflow = true;
        if (x == 0.0f) {
            if (!overflow) segs[nseg++] = Seg{k, 0.0f, 0.0f};
            const float x1 = seq_step(x, inc);
            k++;
            if (!(x1 < limit)) return k;
            x = x1;
            continue;
        }
        double u, top;
        binade(x, u, top);
        bool tie;
        double d = round_to(inc, u, tie);
        if (tie) {
            // round-half-even: from an even multiple of u every step adds the even one of the
            // two neighbouring multiples; an odd start takes one explicit step first
            const double m = floor(inc / u);
            const double xu = (double)x / u;
            if (fmod(xu, 2.0) != 0.0) {
                if (!overflow) segs[nseg++] = Seg{k, x, 0.0f};
                const float x1 = seq_step(x, inc);
                if (x1 == x) { stalled = true; return k + 1; }
                k++;
                if (!(x1 < limit)) return k;
                x = x1;
                continue;
            }
            d = (fmod(m, 2.0) == 0.0 ? m : m + 1.0) * u;
        }
        if (d == 0.0) { stalled = true; return k + 1; }
        const double n_in = steps_upto((double)x, d, top - u);
        const double n_lim = steps_below((double)x, d, (double)limit);
        const double run = fmin(n_in, n_lim);
        if (!overflow) segs[nseg++] = Seg{k, x, (float)d};
        if (n_lim < n_in) return k + (uint32_t)run + 1;
        k += (uint32_t)run;
        x = (float)((double)x + run * d);
        const float x1 = seq_step(x, inc);  // across the binade boundary
        k++;
        if (!(x1 < limit)) return k;
        x = x1;
    }
    stalled = true;
    return k;
}

// x_k from the segments (k below the count returned by seq_segments); seg is the caller's
// cursor, advanced monotonically as k grows.
CGS_HD __forceinline__ float seq_value(const Seg *segs, int nseg, int &seg, uint32_t k) {
    while (seg + 1 < nseg && segs[seg + 1].k0 <= k) seg++;
    const Seg s = segs[seg];
    return fmaf((float)(k - s.k0), s.d, s.x0);
}

}  // namespace cgs
