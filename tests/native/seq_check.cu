// Host check of the closed-form float recurrences (cgs_seq.cuh) against plain sequential
// loops, over random starts and increments, including the reference's own increments
// (1.0, 1/(W-1) for every W in [2, 2048], 1/(W*H)).  Prints "ok" or the first mismatch.
#include <cstdio>
#include <random>
#include "cgs_seq.cuh"

using namespace cgs;

static int check(float x0, double inc, uint32_t maxk, float limit) {
    // sequential reference
    float x = x0;
    uint32_t count = (x < limit) ? 1 : 0;
    bool below = x < limit;
    for (uint32_t k = 1; k <= maxk; k++) {
        const float y = (float)((double)x + inc);
        if (y == x) break;
        x = y;
        float z = x0;
        if (k % 37 == 0 || k == maxk || k < 5) {
            if (!seq_advance(z, inc, k) || z != x) {
                printf("advance mismatch x0=%a inc=%a k=%u got %a want %a\n", x0, inc, k, z, x);
                return 1;
            }
        }
        if (below && x < limit) count++;
        else below = false;
    }
    if (below) return 0;  // limit not reached within maxk: count not comparable
    {
        Seg segs[64];
        int nseg;
        bool ovf, st;
        const uint32_t n = seq_segments(x0, inc, limit, segs, 64, nseg, ovf, st);
        if (n != count || ovf || st) {
            printf("segments count mismatch x0=%a inc=%a limit=%a got %u want %u ovf=%d\n", x0, inc, limit, n, count, ovf);
            return 1;
        }
        float y = x0;
        int cur = 0;
        for (uint32_t k = 0; k < n; k++) {
            const float v = seq_value(segs, nseg, cur, k);
            if (v != y) {
                printf("segment value mismatch x0=%a inc=%a k=%u got %a want %a\n", x0, inc, k, v, y);
                return 1;
            }
            y = (float)((double)y + inc);
        }
    }
    bool stalled;
    const uint32_t c = seq_count_below(x0, inc, limit, stalled);
    if (c != count || stalled) {
        printf("count mismatch x0=%a inc=%a limit=%a got %u want %u\n", x0, inc, limit, c, count);
        return 1;
    }
    return 0;
}

int main() {
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    int bad = 0;
    for (int t = 0; t < 3000 && !bad; t++) {
        const float x0 = (float)(U(rng) * (t % 3 == 0 ? 300.0 : 1.0));
        bad |= check(x0, 1.0, 700, (float)(x0 + 1.0 + U(rng) * 600.0));
    }
    for (int w = 2; w <= 2048 && !bad; w++) {
        const double inc = (double)(1.0f / (float)(w - 1));
        const float x0 = (float)U(rng);
        bad |= check(x0, inc, 2 * w + 8, 1.0f);
        bad |= check(0.0f, inc, 2 * w + 8, 1.0f);
    }
    for (int t = 0; t < 200 && !bad; t++) {
        const int w = 2 + (int)(U(rng) * 1000), h = 2 + (int)(U(rng) * 1000);
        bad |= check(0.0f, 1.0 / (double)(w * h), 300000, 2.0f);
    }
    for (int t = 0; t < 2000 && !bad; t++) {  // mag_norm-like increments
        const float inc = (float)(0.5 + U(rng) * 2.0);
        bad |= check((float)(U(rng) * 1e4), (double)inc, 5000, 3e4f);
    }
    // ties: increments exactly half an ulp of some binade, odd and even starts
    for (int t = 0; t < 3000 && !bad; t++) {
        const int e = -(int)(U(rng) * 20) - 1;
        const double u = ldexp(1.0, e - 23);
        const double inc = (floor(U(rng) * 64) + 0.5) * u;
        float x0 = (float)ldexp(1.0 + floor(U(rng) * 1000) * ldexp(1.0, -23), e);
        bad |= check(x0, inc, 3000, (float)ldexp(1.0, e + 2));
    }
    if (!bad) printf("ok\n");
    return bad;
}
