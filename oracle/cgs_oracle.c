/*
 * cgs_oracle.c -- CPU oracle for the homography grid search (TEST INFRASTRUCTURE ONLY).
 *
 * Restates, in plain C, the reference functors of uncc-visionlab/cuGridSearch on the
 * hot path.  FP32 functions keep the reference's operation order term by term (each
 * C expression below is parenthesised the way C parses the reference expression) and
 * must be compiled with -ffp-contract=off, so the results are bit-identical to the
 * reference source built for the host.  FP64 functions take exactly the same samples
 * (coordinates, bilinear values and the reference's discrete in/out decisions, all
 * in FP32) and accumulate in double.
 *
 * The reference reads one row (plus one element) past the end of the moving image when
 * a sample lands in (H-1, H) (cudaTensor.cuh:561-566 with ceil); that read is undefined
 * behaviour in the reference.  The oracle defines it as zero, which is what a zero-padded
 * buffer gives; the parity harness pads its buffers the same way.
 */
#include "cgs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* Image access: CudaImage<T,C> (include/cudaTensor.cuh:507-575)              */
/* ------------------------------------------------------------------------- */

static inline float og_at(const og_image *im, int64_t flat) {
    int64_t total = (int64_t)im->height * im->width * im->channels;
    if (flat < 0 || flat >= total) return 0.0f; /* past-the-end read: zero pad */
    switch (im->pix) {
        case OG_PIX_U8: return (float)((const uint8_t *)im->data)[flat];
        case OG_PIX_F64: return (float)((const double *)im->data)[flat];
        case OG_PIX_U16: return (float)((const uint16_t *)im->data)[flat];
        default: return ((const float *)im->data)[flat];
    }
}

/* CudaImage::inImage (cudaTensor.cuh:548-550): float coordinates against int sizes. */
static inline int og_in_image(const og_image *im, float y, float x) {
    return x >= 0 && y >= 0 && x < (float)im->width && y < (float)im->height;
}

/* CudaTensor::toIndex1d with float axis indices (cudaTensor.cuh:171-180, 531-534):
 * int accumulator, each step an int*float product added in float, then truncated. */
static inline int64_t og_flat(const og_image *im, float y, float x, float c) {
    int32_t e = (int32_t)c;
    e = (int32_t)((float)e + (float)im->channels * x);
    e = (int32_t)((float)e + (float)(im->channels * im->width) * y);
    return e;
}

/* CudaImage::valueAt_bilinear (cudaTensor.cuh:561-575). */
static inline float og_bilinear(const og_image *im, float y, float x, float c) {
    if (!og_in_image(im, y, x)) return 0.0f;
    float fy = floorf(y), fx = floorf(x), cy = ceilf(y), cx = ceilf(x);
    float tlc = og_at(im, og_flat(im, fy, fx, c));
    float trc = og_at(im, og_flat(im, fy, cx, c));
    float blc = og_at(im, og_flat(im, cy, fx, c));
    float brc = og_at(im, og_flat(im, cy, cx, c));
    float alpha_x = x - fx;
    float alpha_y = y - fy;
    float top = ((1.0f - alpha_x) * tlc) + (alpha_x * trc);
    float bottom = ((1.0f - alpha_x) * blc) + (alpha_x * brc);
    return ((1.0f - alpha_y) * top) + (alpha_y * bottom);
}

void og_bilinear_probe(const og_image *img, float y, float x, int c, float *out) {
    *out = og_bilinear(img, y, x, (float)c);
}

/* ------------------------------------------------------------------------- */
/* Grid (src/gpu/cudaGridSearch.cuh:74-272)                                   */
/* ------------------------------------------------------------------------- */

void og_grid_update(og_grid *g, int changed_axis) {
    int D = g->dims;
    if (changed_axis >= 0 && changed_axis < D) { /* cudaGridSearch.cuh:241-255 */
        int a = changed_axis;
        if ((double)fabsf(g->end[a] - g->start[a]) < 1.0e-7 * (double)g->count[a]) g->count[a] = 1;
        if (g->count[a] == 1) {
            g->resolution[a] = 2 * (g->end[a] - g->start[a]);
        } else {
            /* (int)(end - start) / (count - 1): the int is converted back to float */
            g->resolution[a] = (float)(int32_t)(g->end[a] - g->start[a]) / (g->count[a] - 1);
        }
        return;
    }
    for (int a = 0; a < D; a++) { /* cudaGridSearch.cuh:257-270 */
        if ((double)fabsf(g->end[a] - g->start[a]) < 1.0e-7 * (double)g->count[a]) g->count[a] = 1;
        if (g->count[a] == 1) {
            /* The reference indexes the end/start rows with changed_axis = -1 here
             * (cudaGridSearch.cuh:266); the value is never used because a count-1 axis
             * always decodes index 0.  The oracle stores the evident intent. */
            g->resolution[a] = 2 * (g->end[a] - g->start[a]);
        } else {
            g->resolution[a] = (g->end[a] - g->start[a]) / (g->count[a] - 1);
        }
    }
}

void og_grid_increments(const og_grid *g, int32_t inc[8]) {
    /* indexToGridPoint: dimensional_increments[a] = count[a-1] * inc[a-1] (float
     * product stored in an int32_t), cudaGridSearch.cuh:168-172. */
    inc[0] = 1;
    for (int a = 1; a < g->dims; a++) inc[a] = (int32_t)(g->count[a - 1] * (float)inc[a - 1]);
    for (int a = g->dims; a < 8; a++) inc[a] = 0;
}

int64_t og_grid_num_elements(const og_grid *g) {
    /* numElements (cudaGridSearch.cuh:89-98): int32 total * float count, truncated. */
    int32_t total = 1;
    for (int a = 0; a < g->dims; a++) total = (int32_t)((float)total * g->count[a]);
    return (int64_t)total;
}

void og_grid_point(const og_grid *g, int64_t index, int use_fma, float out[8]) {
    int32_t inc[8];
    int32_t idx[8];
    og_grid_increments(g, inc);
    int32_t rem = (int32_t)index;
    for (int a = g->dims - 1; a >= 0; a--) {
        idx[a] = rem / inc[a];
        rem -= idx[a] * inc[a];
    }
    for (int a = 0; a < 8; a++) out[a] = 0.0f;
    for (int a = 0; a < g->dims; a++) {
        if (use_fma) out[a] = fmaf((float)idx[a], g->resolution[a], g->start[a]);
        else out[a] = g->start[a] + ((float)idx[a] * g->resolution[a]);
    }
}

/* ------------------------------------------------------------------------- */
/* Homographies (src/gpu/cudaImageFunctions.cuh, cudaErrorFunctions.cuh)       */
/* ------------------------------------------------------------------------- */

/* parametersToHomography, centred on (cx, cy) (cudaImageFunctions.cuh:216-252).
 * Parameter order [theta, sx, sy, shear, tx, ty, kx, ky]; h33 divides everything. */
void og_params_to_h(const float *p, float cx, float cy, float h[8]) {
    const float th = p[0], sx = p[1], sy = p[2], sh = p[3], tx = p[4], ty = p[5], kx = p[6], ky = p[7];
    const float c = cosf(th), s = sinf(th);
    float a2 = (cx * kx) + 1;                 /* (cx*keystoneX + 1) */
    float a4 = cx * ky;                       /* cx*keystoneY */
    float a6 = (c * a2) + (a4 * s);           /* cos*(..) + cx*ky*sin */
    float h11 = sx * a6;
    float t5 = ((sh * a6) - (s * a2)) + (a4 * c);
    float h12 = sy * t5;
    float u3 = cx * sx, u6 = cy * sy;
    float h13 = (((cx + (tx * a2)) - (u3 * a6)) - (u6 * t5)) + (a4 * ty);
    float b2 = (cy * ky) + 1;
    float b4 = cy * kx;
    float b6 = (s * b2) + (b4 * c);
    float h21 = sx * b6;
    float v5 = ((sh * b6) + (c * b2)) - (b4 * s);
    float h22 = sy * v5;
    float h23 = (((cy + (ty * b2)) - (u3 * b6)) - (u6 * v5)) + (b4 * tx);
    float d3 = (kx * c) + (ky * s);
    float h31 = sx * d3;
    float e5 = ((sh * d3) + (ky * c)) - (kx * s);
    float h32 = sy * e5;
    float h33 = ((((kx * tx) + (ky * ty)) - (u6 * e5)) - (u3 * d3)) + 1;
    h[0] = h11 / h33; h[1] = h12 / h33; h[2] = h13 / h33;
    h[3] = h21 / h33; h[4] = h22 / h33; h[5] = h23 / h33;
    h[6] = h31 / h33; h[7] = h32 / h33;
}

/* Uncentred parametrisation inlined in averageAbsoluteDifference
 * (cudaErrorFunctions.cuh:42-57). */
void og_params_to_h_uncentred(const float *p, float h[8]) {
    const float th = p[0], sx = p[1], sy = p[2], sh = p[3], tx = p[4], ty = p[5], kx = p[6], ky = p[7];
    const float c = cosf(th), s = sinf(th);
    h[0] = sx * c;
    h[1] = ((sy * sh) * c) - (sy * s);
    h[2] = sx * tx;
    h[3] = sx * s;
    h[4] = ((sy * sh) * s) + (sy * c);
    h[5] = sy * ty;
    h[6] = kx;
    h[7] = ky;
}

/* parametersToHomographyNorm (cudaImageFunctions.cuh:181-214): integer ratios, the
 * rounded centres (cmy uses the moving WIDTH, :201) and the scale mutation. */
void og_params_to_h_norm(const float *p, int mw, int mh, int fw, int fh, float h[8]) {
    const float th = p[0], sh = p[3], tx = p[4], ty = p[5], kx = p[6], ky = p[7];
    float x_ratio = (float)(fw / mw);
    float y_ratio = (float)(fh / mh);
    float cfx = (float)round((double)(fw / 2));
    float cfy = (float)round((double)(fh / 2));
    float cmx = (float)round((double)(mw / 2));
    float cmy = (float)round((double)(mw / 2));
    float sx = p[1] / x_ratio;
    float sy = p[2] / y_ratio;
    const float c = cosf(th), s = sinf(th);
    h[0] = sx * c;
    h[1] = ((sy * sh) * c) - (sy * s);
    h[2] = ((tx - cfx) + cmx) / (float)fw;
    h[3] = sx * s;
    h[4] = ((sy * sh) * s) + (sy * c);
    h[5] = ((ty - cfy) + cmy) / (float)fh;
    h[6] = kx;
    h[7] = ky;
}

/* calcNewCoordH (cudaImageFunctions.cuh:277-285): applies the adjugate of H, i.e. maps a
 * fixed-image pixel to moving-image coordinates. */
void og_new_coord(const float h[8], int x, int y, float *nx, float *ny) {
    const float h11 = h[0], h12 = h[1], h13 = h[2], h21 = h[3], h22 = h[4], h23 = h[5], h31 = h[6], h32 = h[7];
    const float fx = (float)x, fy = (float)y;
    float w = ((((h21 * h32) - (h22 * h31)) * fx + ((h12 * h31) - (h11 * h32)) * fy) + (h11 * h22)) - (h12 * h21);
    float X = ((((h22 - (h23 * h32)) * fx) + ((h13 * h32) - h12) * fy) + (h12 * h23)) - (h13 * h22);
    float Y = ((((h23 * h31) - h21) * fx + (h11 - (h13 * h31)) * fy) + (h13 * h21)) - (h11 * h23);
    *nx = X / w;
    *ny = Y / w;
}

/* parametricAssignValues (cudaImageFunctions.cuh:315-376). */
static void og_assign_values(const float h[8], int m_width, int m_height, int f_width, int f_height, int row_i,
                             float *ls, float *le, float *v_x, float *v_y, float *p0_x, float *p0_y, int *in) {
    (void)f_height;
    const float h11 = h[0], h12 = h[1], h13 = h[2], h21 = h[3], h22 = h[4], h23 = h[5], h31 = h[6], h32 = h[7];
    const float row = (float)row_i, fw = (float)f_width, mh = (float)m_height, mw = (float)m_width;
    float D = (((((h11 * h22) - (h12 * h21)) - ((h11 * h23) * h32)) + ((h12 * h23) * h31)) + ((h13 * h21) * h32)) -
              ((h13 * h22) * h31);
    float den1 = (((h11 * h22) - (h12 * h21)) - ((h11 * h32) * row)) + ((h12 * h31) * row);
    float den2 = (((((h11 * h22) - (h12 * h21)) + ((fw * h21) * h32)) - ((fw * h22) * h31)) - ((h11 * h32) * row)) +
                 ((h12 * h31) * row);
    *v_x = ((h22 - (h32 * row)) * D) / (den1 * den2);
    *v_y = (-((h21 - (h31 * row)) * D)) / (den1 * den2);
    float pden = ((h12 * h21) - (h11 * h22)) + (row * ((h11 * h32) - (h12 * h31)));
    *p0_x = (((h13 * h22) - (h12 * h23)) + (row * (h12 - (h13 * h32)))) / pden;
    *p0_y = (-(((h13 * h21) - (h11 * h23)) + (row * (h11 - (h13 * h31))))) / pden;

    float inner1 = (((h11 * h23) - (h13 * h21)) - (h11 * row)) + ((h13 * h31) * row);
    float lambda_top = (-(inner1 * den2)) / ((h21 - (h31 * row)) * D);
    float x_top_ipt = (-(h23 - row)) / (h21 - (h31 * row));
    float inner2 = (((((((h11 * h23) - (h13 * h21)) - (h11 * row)) + ((h11 * h22) * mh)) - ((h12 * h21) * mh)) +
                     ((h13 * h31) * row)) - (((h11 * h32) * mh) * row)) + (((h12 * h31) * mh) * row);
    float lambda_bottom = (-(den2 * inner2)) / ((h21 - (h31 * row)) * D);
    float x_bottom_ipt = (-(((h23 - row) + (h22 * mh)) - ((h32 * mh) * row))) / (h21 - (h31 * row));
    float inner3 = (((h12 * h23) - (h13 * h22)) - (h12 * row)) + ((h13 * h32) * row);
    float lambda_left = (-(inner3 * den2)) / ((h22 - (h32 * row)) * D);
    float y_left_ipt = (-(h23 - row)) / (h22 - (h32 * row));
    float inner4 = (((((((h12 * h23) - (h13 * h22)) - (h12 * row)) - ((h11 * h22) * mw)) + ((h12 * h21) * mw)) +
                     ((h13 * h32) * row)) + (((h11 * h32) * mw) * row)) - (((h12 * h31) * mw) * row);
    float lambda_right = (-(den2 * inner4)) / ((h22 - (h32 * row)) * D);
    float y_right_ipt = (-(((h23 - row) + (h21 * mw)) - ((h31 * mw) * row))) / (h22 - (h32 * row));

    if (x_top_ipt >= 0 && x_top_ipt < m_width && lambda_top >= 0 && lambda_top < f_width) {
        if (*v_y > 0) *ls = lambda_top; else *le = lambda_top;
        *in = 1;
    }
    if (x_bottom_ipt >= 0 && x_bottom_ipt < m_width && lambda_bottom >= 0 && lambda_bottom < f_width) {
        if (*v_y < 0) *ls = lambda_bottom; else *le = lambda_bottom;
        *in = 1;
    }
    if (y_left_ipt >= 0 && y_left_ipt < m_height && lambda_left >= 0 && lambda_left < f_height) {
        if (*v_x > 0) *ls = lambda_left; else *le = lambda_left;
        *in = 1;
    }
    if (y_right_ipt >= 0 && y_right_ipt < m_height && lambda_right >= 0 && lambda_right < f_height) {
        if (*v_x < 0) *ls = lambda_right; else *le = lambda_right;
        *in = 1;
    }
}

/* parametricAssignValuesNorm (cudaImageFunctions.cuh:378-441), normalised coordinates. */
static void og_assign_values_norm(const float h[8], float row, float *ls, float *le, float *v_x, float *v_y,
                                  float *p0_x, float *p0_y, int *in) {
    const float h11 = h[0], h12 = h[1], h13 = h[2], h21 = h[3], h22 = h[4], h23 = h[5], h31 = h[6], h32 = h[7];
    const float col = -0.5f;
    float D = (((((h11 * h22) - (h12 * h21)) - ((h11 * h23) * h32)) + ((h12 * h23) * h31)) + ((h13 * h21) * h32)) -
              ((h13 * h22) * h31);
    *v_y = (-(h21 - (h31 * row))) / D;
    *v_x = (h22 - (h32 * row)) / D;
    float den = (((h11 * h22) - (h12 * h21)) + (col * ((h21 * h32) - (h22 * h31)))) - (row * ((h11 * h32) - (h12 * h31)));
    float numx = (((h12 * h23) - (h13 * h22)) + (col * (h22 - (h23 * h32)))) - (row * (h12 - (h13 * h32)));
    float numy = (((h11 * h23) - (h13 * h21)) + (col * (h21 - (h23 * h31)))) - (row * (h11 - (h13 * h31)));
    *p0_x = numx / den;
    *p0_y = (-numy) / den;
    float lambda_top = (-(((numy / den) - 0.5f) * D)) / (h21 - (h31 * row));
    float x_top_ipt = (((h22 - (2 * h23)) + (2 * row)) - (h32 * row)) / (2 * (h21 - (h31 * row)));
    float lambda_bottom = (-(((numy / den) + 0.5f) * D)) / (h21 - (h31 * row));
    float x_bottom_ipt = (-(((h22 + (2 * h23)) - (2 * row)) - (h32 * row))) / (2 * (h21 - (h31 * row)));
    float lambda_left = (-(((numx / den) + 0.5f) * D)) / (h22 - (h32 * row));
    float y_left_ipt = (((h21 - (2 * h23)) + (2 * row)) - (h31 * row)) / (2 * (h22 - (h32 * row)));
    float lambda_right = (-(((numx / den) - 0.5f) * D)) / (h22 - (h32 * row));
    float y_right_ipt = (-(((h21 + (2 * h23)) - (2 * row)) - (h31 * row))) / (2 * (h22 - (h32 * row)));

    if (x_top_ipt > -0.5 && x_top_ipt < 0.5 && lambda_top >= 0 && lambda_top < 1) {
        if (*v_y > 0) *ls = lambda_top; else *le = lambda_top;
        *in = 1;
    }
    if (x_bottom_ipt > -0.5 && x_bottom_ipt < 0.5 && lambda_bottom > 0 && lambda_bottom < 1) {
        if (*v_y < 0) *ls = lambda_bottom; else *le = lambda_bottom;
        *in = 1;
    }
    if (y_left_ipt > -0.5 && y_left_ipt < 0.5 && lambda_left > 0 && lambda_left < 1) {
        if (*v_x > 0) *ls = lambda_left; else *le = lambda_left;
        *in = 1;
    }
    if (y_right_ipt > -0.5 && y_right_ipt < 0.5 && lambda_right > 0 && lambda_right < 1) {
        if (*v_x < 0) *ls = lambda_right; else *le = lambda_right;
        *in = 1;
    }
}

/* ------------------------------------------------------------------------- */
/* Cost bodies, instantiated for float and double accumulators                 */
/* ------------------------------------------------------------------------- */

static inline uint32_t og_bin(float v, int bins) {
    float b = floorf((float)bins * (v / 256.0f));
    if (!(b >= 0.0f)) return 0; /* reference: negative -> huge unsigned index (UB); clamped */
    if (b > (float)(bins - 1)) return (uint32_t)(bins - 1);
    return (uint32_t)b;
}

/* The shifts of the zero-mean NCC moments: an image's mean over a fixed subsample -- at most
 * 4096 evenly strided elements of the HWC array (stride total / 4096), summed in double and
 * rounded to float.  The library's staging kernel takes the same elements; a cost does not depend
 * on its shifts beyond rounding, but the degenerate-overlap rule below is stated with them. */
static float og_subsample_mean(const og_image *im) {
    const int64_t total = (int64_t)im->height * im->width * im->channels;
    const int64_t stride = total > 4096 ? total / 4096 : 1;
    const int64_t count = total > 4096 ? 4096 : total;
    double s = 0.0;
    for (int64_t i = 0; i < count; i++) s += (double)og_at(im, i * stride);
    return (float)(s / (double)count);
}

#define OG_ACC float
#define OG_SQRT sqrtf
#define OG_SFX _f32
#include "cgs_oracle_body.inc"
#undef OG_ACC
#undef OG_SQRT
#undef OG_SFX

#define OG_ACC double
#define OG_SQRT sqrt
#define OG_SFX _f64
#include "cgs_oracle_body.inc"
#undef OG_ACC
#undef OG_SQRT
#undef OG_SFX

float og_cost_f32(int cost, const float *params, const og_image *mov, const og_image *fix, const og_opts *opts,
                  int64_t *n_out) {
    return og_cost_body_f32(cost, params, mov, fix, opts, n_out, NULL);
}

double og_cost_f64(int cost, const float *params, const og_image *mov, const og_image *fix, const og_opts *opts,
                   int64_t *n_out) {
    return og_cost_body_f64(cost, params, mov, fix, opts, n_out, NULL);
}

int64_t og_histogram(int cost, const float *params, const og_image *mov, const og_image *fix, const og_opts *opts,
                     uint32_t *hist) {
    int64_t n = 0;
    if (cost != OG_MI && cost != OG_MI_ALT) return -1;
    og_cost_body_f64(cost, params, mov, fix, opts, &n, hist);
    return n;
}

int og_search(int cost, const og_grid *g, int use_fma, const og_image *mov, const og_image *fix, const og_opts *opts,
              int64_t first, int64_t count, int64_t stride, float *costs32, double *costs64, int threads) {
    if (cost < 0 || cost >= OG_NUM_COSTS || count < 0 || stride <= 0) return 1;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
#endif
    for (int64_t k = 0; k < count; k++) {
        float pt[8];
        og_grid_point(g, first + k * stride, use_fma, pt);
        if (costs32) costs32[k] = og_cost_f32(cost, pt, mov, fix, opts, NULL);
        if (costs64) costs64[k] = og_cost_f64(cost, pt, mov, fix, opts, NULL);
    }
    (void)threads;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Covariance around the grid minimum (src/gpu/cudaGridSearch.cuh:316-419)     */
/* ------------------------------------------------------------------------- */

void og_covariance(const og_grid *g, const float *costs, int64_t n, double *out_f64, float *out_ref) {
    const int D = g->dims;
    for (int i = 0; i < D * D; i++) {
        if (out_f64) out_f64[i] = 0.0;
        if (out_ref) out_ref[i] = 0.0f;
    }
    float fmin = 0.0f;
    int64_t imin = 0;
    for (int64_t t = 0; t < n; t++) /* func_precision min_val = 0; strict '<' */
        if (costs[t] < fmin) {
            fmin = costs[t];
            imin = t;
        }
    float xm[8], x[8];
    og_grid_point(g, imin, 1, xm);
    const float lmin = logf(fabsf(fmin));
    for (int64_t t = 0; t < n; t++) {
        if (t == imin) continue;
        og_grid_point(g, t, 1, x);
        float f = costs[t];
        if (f == 0.0f) f = -1e-9f;
        float d[8], gv[8], len = 0.0f;
        for (int a = 0; a < D; a++) {
            d[a] = x[a] - xm[a];
            len = fmaf(d[a], d[a], len); /* length += d * d, fused by the device build */
        }
        len = sqrtf(len);
        const float slope = (lmin - logf(fabsf(f))) * (1.0f / len);
        if (slope < 0.0f) continue;
        for (int a = 0; a < D; a++) gv[a] = (d[a] * slope) / len;
        for (int r = 0; r < D; r++)
            for (int c = 0; c < D; c++) {
                if (out_f64) out_f64[r * D + c] += (double)gv[r] * (double)gv[c];
                if (out_ref) out_ref[r * D + c] = fmaf(gv[r], gv[c], out_ref[r * D + c]);
            }
    }
}
