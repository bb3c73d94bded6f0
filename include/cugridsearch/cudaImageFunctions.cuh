/*
 * cudaImageFunctions.cuh -- homography helpers of the grid search (reference:
 * src/gpu/cudaImageFunctions.cuh:181-441), as __host__ __device__ templates.
 *
 * Parameter order everywhere: [theta, scaleX, scaleY, shearXY, translateX, translateY,
 * keystoneX, keystoneY].  Each expression is evaluated in the reference's order (the
 * parenthesisation below is how C++ parses the reference's expressions), so host builds
 * give the reference's FP32 results bit for bit; on the device the compiler's FMA
 * contraction applies to both alike.
 */
#ifndef CUGRIDSEARCH_CUDAIMAGEFUNCTIONS_CUH
#define CUGRIDSEARCH_CUDAIMAGEFUNCTIONS_CUH

#ifndef CUDAFUNCTION
#define CUDAFUNCTION __host__ __device__
#endif

#include <cmath>
#include <cstdint>

#include "nvVectorNd.h"

// Homography centred on (cx, cy) (the moving image's centre in the functors), normalised
// by h33 (cudaImageFunctions.cuh:216-252).
template <typename Tp, uint8_t D>
CUDAFUNCTION void parametersToHomography(nv_ext::Vec<Tp, D> &parameters, float &cx, float &cy, float &h11, float &h12,
                                         float &h13, float &h21, float &h22, float &h23, float &h31, float &h32) {
    const float th = parameters[0], sx = parameters[1], sy = parameters[2], sh = parameters[3];
    const float tx = parameters[4], ty = parameters[5], kx = parameters[6], ky = parameters[7];
    const float c = cos(th), s = sin(th);
    const float a2 = (cx * kx) + 1;  // cx*keystoneX + 1
    const float a4 = cx * ky;
    const float a6 = (c * a2) + (a4 * s);
    const float t5 = ((sh * a6) - (s * a2)) + (a4 * c);
    const float u3 = cx * sx, u6 = cy * sy;
    const float b2 = (cy * ky) + 1;
    const float b4 = cy * kx;
    const float b6 = (s * b2) + (b4 * c);
    const float v5 = ((sh * b6) + (c * b2)) - (b4 * s);
    const float d3 = (kx * c) + (ky * s);
    const float e5 = ((sh * d3) + (ky * c)) - (kx * s);
    h11 = sx * a6;
    h12 = sy * t5;
    h13 = (((cx + (tx * a2)) - (u3 * a6)) - (u6 * t5)) + (a4 * ty);
    h21 = sx * b6;
    h22 = sy * v5;
    h23 = (((cy + (ty * b2)) - (u3 * b6)) - (u6 * v5)) + (b4 * tx);
    h31 = sx * d3;
    h32 = sy * e5;
    const float h33 = ((((kx * tx) + (ky * ty)) - (u6 * e5)) - (u3 * d3)) + 1;
    h11 /= h33;
    h12 /= h33;
    h13 /= h33;
    h21 /= h33;
    h22 /= h33;
    h23 /= h33;
    h31 /= h33;
    h32 /= h33;
}

// Normalised-coordinate homography of calcMIAlt (cudaImageFunctions.cuh:181-214).  As in the
// reference, parameters[1] and parameters[2] are divided by the integer size ratios IN PLACE,
// and the moving centre's y uses the moving WIDTH.
template <typename Tp, uint8_t D>
CUDAFUNCTION void parametersToHomographyNorm(nv_ext::Vec<Tp, D> &parameters, int &m_width, int &m_height, int &f_width,
                                             int &f_height, float &h11, float &h12, float &h13, float &h21, float &h22,
                                             float &h23, float &h31, float &h32) {
    const float x_ratio = (float)(f_width / m_width);
    const float y_ratio = (float)(f_height / m_height);
    const float cfx = (float)round((double)(f_width / 2));
    const float cfy = (float)round((double)(f_height / 2));
    const float cmx = (float)round((double)(m_width / 2));
    const float cmy = (float)round((double)(m_width / 2));
    parameters[1] = parameters[1] / x_ratio;
    parameters[2] = parameters[2] / y_ratio;
    const float th = parameters[0], sx = parameters[1], sy = parameters[2], sh = parameters[3];
    const float tx = parameters[4], ty = parameters[5];
    const float c = cos(th), s = sin(th);
    h11 = sx * c;
    h12 = ((sy * sh) * c) - (sy * s);
    h13 = ((tx - cfx) + cmx) / (float)f_width;
    h21 = sx * s;
    h22 = ((sy * sh) * s) + (sy * c);
    h23 = ((ty - cfy) + cmy) / (float)f_height;
    h31 = parameters[6];
    h32 = parameters[7];
}

// Moves the centring of a homography (cudaImageFunctions.cuh:254-275).
template <typename Tp, uint8_t D>
CUDAFUNCTION void uncenterHomography(float &cx, float &cy, float &h11, float &h12, float &h13, float &h21, float &h22,
                                     float &h23, float &h31, float &h32) {
    h11 = h11 - (cx * h31);
    h12 = h12 - (cx * h32);
    h13 = ((h13 - cx) + (cx * (h11 - (cx * h31)))) + (cy * (h12 - (cx * h32)));
    h21 = h21 - (cy * h31);
    h22 = h22 - (cy * h32);
    h23 = ((h23 - cy) + (cx * (h21 - (cy * h31)))) + (cy * (h22 - (cy * h32)));
    const float h33 = ((cx * h31) + (cy * h32)) + 1;
    h11 /= h33;
    h12 /= h33;
    h13 /= h33;
    h21 /= h33;
    h22 /= h33;
    h23 /= h33;
    h31 /= h33;
    h32 /= h33;
}

// Fixed-image pixel (x, y) -> moving-image coordinates through the adjugate of H
// (cudaImageFunctions.cuh:277-285).
CUDAFUNCTION inline void calcNewCoordH(float &h11, float &h12, float &h13, float &h21, float &h22, float &h23,
                                       float &h31, float &h32, int &x, int &y, float &new_x, float &new_y) {
    const float fx = (float)x, fy = (float)y;
    const float w = ((((h21 * h32) - (h22 * h31)) * fx + ((h12 * h31) - (h11 * h32)) * fy) + (h11 * h22)) - (h12 * h21);
    const float X = ((((h22 - (h23 * h32)) * fx) + ((h13 * h32) - h12) * fy) + (h12 * h23)) - (h13 * h22);
    const float Y = ((((h23 * h31) - h21) * fx + (h11 - (h13 * h31)) * fy) + (h13 * h21)) - (h11 * h23);
    new_x = X / w;
    new_y = Y / w;
}

// Inverse of the uncentred parametrisation (cudaImageFunctions.cuh:287-313).
template <typename Tp, uint8_t D>
void homographyToParameters(float &h11, float &h12, float &h13, float &h21, float &h22, float &h23, float &h31,
                            float &h32, nv_ext::Vec<Tp, D> &parameters) {
    const float theta = atan2(h21, h11);
    const float scaleX = sqrt((h11 * h11) + (h21 * h21));
    const float shy = (h12 * cos(theta)) + (h22 * sin(theta));
    float scaleY;
    if (std::abs(sin(theta)) > 1.0e-6)
        scaleY = ((shy * cos(theta)) - h12) / sin(theta);
    else
        scaleY = (h22 - (shy * sin(theta))) / cos(theta);
    parameters[0] = theta;
    parameters[1] = scaleX;
    parameters[2] = scaleY;
    parameters[3] = shy / scaleY;
    parameters[4] = h13;
    parameters[5] = h23;
    parameters[6] = h31;
    parameters[7] = h32;
}

// Scanline of fixed-image row `row` mapped into the moving image: moving point =
// lambda * (v_x, v_y) + (p0_x, p0_y) for lambda in [lambda_start, lambda_end), and whether
// the line crosses the moving image at all (cudaImageFunctions.cuh:315-376).  The four edge
// tests run in the reference's order; a later crossing overrides an earlier one.
inline CUDAFUNCTION void parametricAssignValues(float &h11, float &h12, float &h13, float &h21, float &h22, float &h23,
                                                float &h31, float &h32, int &m_width, int &m_height, int &f_width,
                                                int &f_height, int &row_i, float &lambda_start, float &lambda_end,
                                                float &v_x, float &v_y, float &p0_x, float &p0_y, bool &inImage) {
    const float row = (float)row_i, fw = (float)f_width, mh = (float)m_height, mw = (float)m_width;
    const float D = (((((h11 * h22) - (h12 * h21)) - ((h11 * h23) * h32)) + ((h12 * h23) * h31)) + ((h13 * h21) * h32)) -
                    ((h13 * h22) * h31);
    const float den1 = (((h11 * h22) - (h12 * h21)) - ((h11 * h32) * row)) + ((h12 * h31) * row);
    const float den2 =
        (((((h11 * h22) - (h12 * h21)) + ((fw * h21) * h32)) - ((fw * h22) * h31)) - ((h11 * h32) * row)) +
        ((h12 * h31) * row);
    v_x = ((h22 - (h32 * row)) * D) / (den1 * den2);
    v_y = (-((h21 - (h31 * row)) * D)) / (den1 * den2);
    const float pden = ((h12 * h21) - (h11 * h22)) + (row * ((h11 * h32) - (h12 * h31)));
    p0_x = (((h13 * h22) - (h12 * h23)) + (row * (h12 - (h13 * h32)))) / pden;
    p0_y = (-(((h13 * h21) - (h11 * h23)) + (row * (h11 - (h13 * h31))))) / pden;

    const float top_in = (((h11 * h23) - (h13 * h21)) - (h11 * row)) + ((h13 * h31) * row);
    const float lambda_top = (-(top_in * den2)) / ((h21 - (h31 * row)) * D);
    const float x_top = (-(h23 - row)) / (h21 - (h31 * row));
    const float bot_in = (((((((h11 * h23) - (h13 * h21)) - (h11 * row)) + ((h11 * h22) * mh)) - ((h12 * h21) * mh)) +
                           ((h13 * h31) * row)) - (((h11 * h32) * mh) * row)) + (((h12 * h31) * mh) * row);
    const float lambda_bottom = (-(den2 * bot_in)) / ((h21 - (h31 * row)) * D);
    const float x_bottom = (-(((h23 - row) + (h22 * mh)) - ((h32 * mh) * row))) / (h21 - (h31 * row));
    const float left_in = (((h12 * h23) - (h13 * h22)) - (h12 * row)) + ((h13 * h32) * row);
    const float lambda_left = (-(left_in * den2)) / ((h22 - (h32 * row)) * D);
    const float y_left = (-(h23 - row)) / (h22 - (h32 * row));
    const float right_in = (((((((h12 * h23) - (h13 * h22)) - (h12 * row)) - ((h11 * h22) * mw)) + ((h12 * h21) * mw)) +
                             ((h13 * h32) * row)) + (((h11 * h32) * mw) * row)) - (((h12 * h31) * mw) * row);
    const float lambda_right = (-(den2 * right_in)) / ((h22 - (h32 * row)) * D);
    const float y_right = (-(((h23 - row) + (h21 * mw)) - ((h31 * mw) * row))) / (h22 - (h32 * row));

    if (x_top >= 0 && x_top < m_width && lambda_top >= 0 && lambda_top < f_width) {
        if (v_y > 0) lambda_start = lambda_top; else lambda_end = lambda_top;
        inImage = true;
    }
    if (x_bottom >= 0 && x_bottom < m_width && lambda_bottom >= 0 && lambda_bottom < f_width) {
        if (v_y < 0) lambda_start = lambda_bottom; else lambda_end = lambda_bottom;
        inImage = true;
    }
    if (y_left >= 0 && y_left < m_height && lambda_left >= 0 && lambda_left < f_height) {
        if (v_x > 0) lambda_start = lambda_left; else lambda_end = lambda_left;
        inImage = true;
    }
    if (y_right >= 0 && y_right < m_height && lambda_right >= 0 && lambda_right < f_height) {
        if (v_x < 0) lambda_start = lambda_right; else lambda_end = lambda_right;
        inImage = true;
    }
}

// The same in normalised coordinates (image spans [-0.5, 0.5]) for calcMIAlt
// (cudaImageFunctions.cuh:378-441).
inline CUDAFUNCTION void parametricAssignValuesNorm(float &h11, float &h12, float &h13, float &h21, float &h22,
                                                    float &h23, float &h31, float &h32, int &m_width, int &m_height,
                                                    int &f_width, int &f_height, float &row, float &lambda_start,
                                                    float &lambda_end, float &v_x, float &v_y, float &p0_x,
                                                    float &p0_y, bool &inImage) {
    (void)m_width;
    (void)m_height;
    (void)f_width;
    (void)f_height;
    const float col = -0.5f;
    const float D = (((((h11 * h22) - (h12 * h21)) - ((h11 * h23) * h32)) + ((h12 * h23) * h31)) + ((h13 * h21) * h32)) -
                    ((h13 * h22) * h31);
    v_y = (-(h21 - (h31 * row))) / D;
    v_x = (h22 - (h32 * row)) / D;
    const float den =
        (((h11 * h22) - (h12 * h21)) + (col * ((h21 * h32) - (h22 * h31)))) - (row * ((h11 * h32) - (h12 * h31)));
    const float numx = (((h12 * h23) - (h13 * h22)) + (col * (h22 - (h23 * h32)))) - (row * (h12 - (h13 * h32)));
    const float numy = (((h11 * h23) - (h13 * h21)) + (col * (h21 - (h23 * h31)))) - (row * (h11 - (h13 * h31)));
    p0_x = numx / den;
    p0_y = (-numy) / den;
    const float lambda_top = (-(((numy / den) - 0.5f) * D)) / (h21 - (h31 * row));
    const float x_top = (((h22 - (2 * h23)) + (2 * row)) - (h32 * row)) / (2 * (h21 - (h31 * row)));
    const float lambda_bottom = (-(((numy / den) + 0.5f) * D)) / (h21 - (h31 * row));
    const float x_bottom = (-(((h22 + (2 * h23)) - (2 * row)) - (h32 * row))) / (2 * (h21 - (h31 * row)));
    const float lambda_left = (-(((numx / den) + 0.5f) * D)) / (h22 - (h32 * row));
    const float y_left = (((h21 - (2 * h23)) + (2 * row)) - (h31 * row)) / (2 * (h22 - (h32 * row)));
    const float lambda_right = (-(((numx / den) - 0.5f) * D)) / (h22 - (h32 * row));
    const float y_right = (-(((h21 + (2 * h23)) - (2 * row)) - (h31 * row))) / (2 * (h22 - (h32 * row)));

    if (x_top > -0.5 && x_top < 0.5 && lambda_top >= 0 && lambda_top < 1) {
        if (v_y > 0) lambda_start = lambda_top; else lambda_end = lambda_top;
        inImage = true;
    }
    if (x_bottom > -0.5 && x_bottom < 0.5 && lambda_bottom > 0 && lambda_bottom < 1) {
        if (v_y < 0) lambda_start = lambda_bottom; else lambda_end = lambda_bottom;
        inImage = true;
    }
    if (y_left > -0.5 && y_left < 0.5 && lambda_left > 0 && lambda_left < 1) {
        if (v_x > 0) lambda_start = lambda_left; else lambda_end = lambda_left;
        inImage = true;
    }
    if (y_right > -0.5 && y_right < 0.5 && lambda_right > 0 && lambda_right < 1) {
        if (v_x < 0) lambda_start = lambda_right; else lambda_end = lambda_right;
        inImage = true;
    }
}

#endif  // CUGRIDSEARCH_CUDAIMAGEFUNCTIONS_CUH
