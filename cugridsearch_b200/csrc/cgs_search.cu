// cgs_search.cu -- C ABI of the sm_100a grid search: argument checks, the reference's
// grid arithmetic on the host, image staging, launch configuration and the argmin.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cgs_internal.h"
#include "cgs_scan.cuh"

namespace cgs {

// ---------------------------------------------------------------- error reporting

static thread_local std::string g_last_error;

cgs_status fail(cgs_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

cgs_status cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(CGS_ERROR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    return fail(CGS_ERROR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------- device memory pool

// One pool per device; scratch is taken and returned on the caller's stream, so
// concurrent calls on different streams never share it.
struct DevicePool {
    std::mutex mu;
    cudaMemPool_t pool[64] = {};
};
static DevicePool g_pools;

cgs_status get_pool(int dev, cudaMemPool_t *out) {
    std::lock_guard<std::mutex> lock(g_pools.mu);
    if (dev < 0 || dev >= 64) return fail(CGS_ERROR_NO_DEVICE, "device ordinal out of range");
    if (!g_pools.pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p;
        CGS_CUDA(cudaMemPoolCreate(&p, &props), "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;  // keep freed blocks for reuse by later calls
        CGS_CUDA(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
        g_pools.pool[dev] = p;
    }
    *out = g_pools.pool[dev];
    return CGS_SUCCESS;
}

cgs_status device_info(DeviceInfo *d) {
    CGS_CUDA(cudaGetDevice(&d->dev), "cudaGetDevice");
    CGS_CUDA(cudaDeviceGetAttribute(&d->sms, cudaDevAttrMultiProcessorCount, d->dev), "cudaDeviceGetAttribute");
    CGS_CUDA(cudaDeviceGetAttribute(&d->major, cudaDevAttrComputeCapabilityMajor, d->dev), "cudaDeviceGetAttribute");
    if (d->major != 10) return fail(CGS_ERROR_NO_DEVICE, "this build runs on sm_100 (B200) devices only");
    CGS_CUDA(cudaDeviceGetAttribute(&d->tex_align, cudaDevAttrTextureAlignment, d->dev), "cudaDeviceGetAttribute");
    CGS_CUDA(cudaDeviceGetAttribute(&d->tex_pitch_align, cudaDevAttrTexturePitchAlignment, d->dev),
             "cudaDeviceGetAttribute");
    return CGS_SUCCESS;
}

// ---------------------------------------------------------------- grid arithmetic

// CudaGrid dimensional increments and element count exactly as the reference computes
// them: float count times int increment, truncated to int32 (cudaGridSearch.cuh:89-98, 168-172).
void grid_increments(const cgs_grid &g, int32_t inc[8], int64_t *num) {
    inc[0] = 1;
    for (int a = 1; a < 8; a++) inc[a] = (a < g.dims) ? (int32_t)(g.count[a - 1] * (float)inc[a - 1]) : 0;
    int32_t total = 1;
    for (int a = 0; a < g.dims; a++) total = (int32_t)((float)total * g.count[a]);
    *num = total;
}

// The locality order needs the grid to be an exact product of integer counts: then
// index = sum(i_a * inc[a]) is a bijection onto [0, n).  Fractional counts (the reference
// allows them, cudaGridSearch_main_mi.cu:304-305) or float products that round make the
// reference's own decode non-bijective; such grids run in the reference order.
static bool integral_counts(const cgs_grid &g) {
    int32_t inc[8];
    int64_t n;
    grid_increments(g, inc, &n);
    int64_t exact = 1;
    for (int a = 0; a < g.dims; a++) {
        if (!(g.count[a] >= 1.0f) || g.count[a] != std::floor(g.count[a]) || g.count[a] > 1.0e7f) return false;
        if (inc[a] != exact) return false;
        exact *= (int64_t)g.count[a];
        if (exact > INT32_MAX) return false;
    }
    return exact == n;
}

static bool cost_uses_theta(int cost) {
    return cost == CGS_COST_SAD_AVG || cost == CGS_COST_SQD_REF || cost == CGS_COST_NCC_REF ||
           cost == CGS_COST_ZNCC || cost == CGS_COST_MI || cost == CGS_COST_SQD_ALT || cost == CGS_COST_NCC_ALT ||
           cost == CGS_COST_MI_ALT;
}

// Host model (double precision) of the sample position of fixed pixel (x, y) for a grid
// point; used only to choose the evaluation order, never for a cost.
static void model_map(int cost, const double *q, double cx, double cy, double x, double y, double *mx, double *my) {
    double h[9];
    const double th = q[0], sx = q[1], sy = q[2], sh = q[3], tx = q[4], ty = q[5], kx = q[6], ky = q[7];
    const double c = std::cos(th), s = std::sin(th);
    if (cost == CGS_COST_SAD_SUM_T || cost == CGS_COST_SAD_SUM_T_REF) {
        *mx = x + q[0];
        *my = y + q[1];
        return;
    }
    if (cost == CGS_COST_SAD_AVG_H) {
        const double z = q[6] * x + q[7] * y + 1.0;
        *mx = (q[0] * x + q[1] * y + q[2]) / z;
        *my = (q[3] * x + q[4] * y + q[5]) / z;
        return;
    }
    if (cost == CGS_COST_SAD_AVG) {
        h[0] = sx * c; h[1] = sy * sh * c - sy * s; h[2] = sx * tx;
        h[3] = sx * s; h[4] = sy * sh * s + sy * c; h[5] = sy * ty;
        h[6] = kx; h[7] = ky; h[8] = 1.0;
    } else {
        const double a2 = cx * kx + 1, a4 = cx * ky, a6 = c * a2 + a4 * s;
        const double t5 = sh * a6 - s * a2 + a4 * c;
        const double b2 = cy * ky + 1, b4 = cy * kx, b6 = s * b2 + b4 * c;
        const double v5 = sh * b6 + c * b2 - b4 * s;
        const double d3 = kx * c + ky * s, e5 = sh * d3 + ky * c - kx * s;
        h[0] = sx * a6; h[1] = sy * t5;
        h[2] = cx + tx * a2 - cx * sx * a6 - cy * sy * t5 + a4 * ty;
        h[3] = sx * b6; h[4] = sy * v5;
        h[5] = cy + ty * b2 - cx * sx * b6 - cy * sy * v5 + b4 * tx;
        h[6] = sx * d3; h[7] = sy * e5;
        h[8] = kx * tx + ky * ty - cy * sy * e5 - cx * sx * d3 + 1;
    }
    // inverse map through the adjugate (calcNewCoordH)
    const double w = (h[3] * h[7] - h[4] * h[6]) * x + (h[1] * h[6] - h[0] * h[7]) * y + h[0] * h[4] - h[1] * h[3];
    const double X = (h[4] * h[8] - h[5] * h[7]) * x + (h[2] * h[7] - h[1] * h[8]) * y + h[1] * h[5] - h[2] * h[4];
    const double Y = (h[5] * h[6] - h[3] * h[8]) * x + (h[0] * h[8] - h[2] * h[6]) * y + h[2] * h[3] - h[0] * h[5];
    *mx = X / w;
    *my = Y / w;
}

// Evaluation order: axes sorted by how far one step moves the sampled footprint (the
// largest displacement over the fixed image's corners and centre), smallest first.
static void locality_order(int cost, const cgs_grid &g, int fw, int fh, int mw, int mh, int32_t perm[8]) {
    double mid[8] = {0, 1, 1, 0, 0, 0, 0, 0};
    for (int a = 0; a < g.dims; a++) mid[a] = g.start[a] + 0.5 * (g.count[a] - 1) * g.resolution[a];
    const double cx = mw * 0.5, cy = mh * 0.5;
    const double px[5] = {0, (double)fw - 1, 0, (double)fw - 1, 0.5 * fw};
    const double py[5] = {0, 0, (double)fh - 1, (double)fh - 1, 0.5 * fh};
    std::vector<std::pair<double, int>> disp;
    for (int a = 0; a < g.dims; a++) {
        double d = 0;
        if (g.count[a] > 1) {
            double q2[8];
            memcpy(q2, mid, sizeof(q2));
            q2[a] += g.resolution[a];
            for (int k = 0; k < 5; k++) {
                double x0, y0, x1, y1;
                model_map(cost, mid, cx, cy, px[k], py[k], &x0, &y0);
                model_map(cost, q2, cx, cy, px[k], py[k], &x1, &y1);
                double dd = std::hypot(x1 - x0, y1 - y0);
                if (!(dd == dd)) dd = 1e30;
                d = std::max(d, dd);
            }
        }
        disp.push_back({d, a});
    }
    std::stable_sort(disp.begin(), disp.end());
    for (int j = 0; j < 8; j++) perm[j] = j < g.dims ? disp[j].second : j;
}

// ---------------------------------------------------------------- kernels: staging, argmin


__device__ __forceinline__ float load_pix(const void *src, int pix, int64_t i) {
    switch (pix) {
        case CGS_PIXEL_U8: return (float)static_cast<const uint8_t *>(src)[i];
        case CGS_PIXEL_F64: return (float)static_cast<const double *>(src)[i];  // rounded to nearest
        case CGS_PIXEL_U16: return (float)static_cast<const uint16_t *>(src)[i];
        default: return static_cast<const float *>(src)[i];
    }
}

// HWC images -> one zero-padded FP32 plane per channel.  Moving planes are (H + 1) rows of
// `mpitch` floats: pixels in columns 0..W-1, pixel (0, y + 1) in column W (the reference's
// flat-index neighbour of (W - 1, y)), zeros elsewhere, a zero row H.  Fixed planes use a
// 16-byte row pitch so rows can be bulk-copied.
__device__ __forceinline__ void prep_body(const PrepParams &q, int64_t tid, int64_t nthr) {
    if (tid == 0) {
        *q.key = ~0ull;
        *q.done = 0u;
        *q.status = 0u;
    }
    const int64_t mtot = q.mplane * q.c;
    unsigned int vmax_bits = 0u;  // max |v| as float bits (non-negative floats order as integers)
    for (int64_t i = tid; i < mtot; i += nthr) {
        const int c = (int)(i / q.mplane);
        const int64_t e = i - (int64_t)c * q.mplane;
        const int64_t y = e / q.mpitch, x = e - y * q.mpitch;
        float v = 0.0f;
        if (y < q.mh && x < q.mw) v = load_pix(q.mov_src, q.mov_pix, (y * q.mw + x) * q.c + c);
        else if (y + 1 < q.mh && x == q.mw) v = load_pix(q.mov_src, q.mov_pix, ((y + 1) * q.mw) * q.c + c);
        q.mov_dst[i] = v;
        const float av = fabsf(v);
        const unsigned int b = (av == av) ? __float_as_uint(av) : 0x7f800000u;
        vmax_bits = b > vmax_bits ? b : vmax_bits;
    }
    vmax_bits = __reduce_max_sync(0xffffffffu, vmax_bits);
    if ((threadIdx.x & 31) == 0 && vmax_bits) atomicMax(reinterpret_cast<unsigned int *>(q.vmax), vmax_bits);
    const int64_t ftot = q.fplane * q.c;
    for (int64_t i = tid; i < ftot; i += nthr) {
        const int c = (int)(i / q.fplane);
        const int64_t e = i - (int64_t)c * q.fplane;
        const int64_t y = e / q.fpitch, x = e - y * q.fpitch;
        float v = 0.0f;
        if (y < q.fh && x < q.fw) v = load_pix(q.fix_src, q.fix_pix, (y * q.fw + x) * q.c + c);
        else if (q.fix_alias && y + 1 < q.fh && x == q.fw)
            v = load_pix(q.fix_src, q.fix_pix, ((y + 1) * q.fw) * q.c + c);
        q.fix_dst[i] = v;
    }
    if (q.quad_dst) {
        // tap quads of the staged moving plane, the left column and the FP32 differences to the
        // right column: {P(y, x), P(y + 1, x), P(y, x + 1) - P(y, x), P(y + 1, x + 1) - P(y + 1, x)}
        // with P the padded plane (column W = the next row's pixel 0, row H = 0); the search
        // kernel's bilinear step takes the differences as they are.  The span kernel's form holds
        // the bilinear polynomial's coefficients instead (quad_form 1)
        const int64_t qtot = q.qplane * q.c;
        auto P = [&](int c, int64_t y, int64_t x) -> float {
            if (y >= q.mh) return 0.0f;
            if (x < q.mw) return load_pix(q.mov_src, q.mov_pix, (y * q.mw + x) * q.c + c);
            return (y + 1 < q.mh) ? load_pix(q.mov_src, q.mov_pix, ((y + 1) * q.mw) * q.c + c) : 0.0f;
        };
        for (int64_t i = tid; i < qtot; i += nthr) {
            const int c = (int)(i / q.qplane);
            const int64_t e = i - (int64_t)c * q.qplane;
            const int64_t y = e / q.mw, x = e - y * q.mw;
            const float v00 = P(c, y, x), v10 = P(c, y + 1, x);
            const float d0 = P(c, y, x + 1) - v00, d1 = P(c, y + 1, x + 1) - v10;
            q.quad_dst[i] = q.quad_form ? make_float4(v00, d0, v10 - v00, d1 - d0) : make_float4(v00, v10, d0, d1);
        }
    }
    if (q.row_table && tid == 0) {
        // calcMIAlt's rows: row = -0.5; while (row < 0.5) row += 1 / (float)(rowsf - 1)
        // (cudaErrorFunction_mi.cuh:164), the same float additions as the reference
        float row = -0.5f;
        int n = 0;
        const float inc = 1.0f / (float)(q.rowsf - 1);
        while ((double)row < 0.5 && n < q.rowsf + 2) {
            q.row_table[n++] = row;
            row = __fadd_rn(row, inc);
        }
    }
}

// The images' means for the ZNCC shifts, over a fixed subsample (at most kShiftSamples evenly
// strided elements of each HWC image), summed in FP64 in a fixed order by one block of 256
// threads: the same bits on every call.  shifts = {fixed mean, moving mean}.
constexpr int64_t kShiftSamples = 4096;

__device__ void staging_means(const PrepParams &q) {
    __shared__ double part[2][8];
    const int t = threadIdx.x;
    double acc[2] = {0.0, 0.0};
    for (int k = 0; k < 2; k++) {
        const void *src = k == 0 ? q.fix_src : q.mov_src;
        const int pix = k == 0 ? q.fix_pix : q.mov_pix;
        const int64_t total = k == 0 ? (int64_t)q.fh * q.fw * q.c : (int64_t)q.mh * q.mw * q.c;
        const int64_t stride = total > kShiftSamples ? total / kShiftSamples : 1;
        const int64_t count = total > kShiftSamples ? kShiftSamples : total;
        double s = 0.0;
        for (int64_t i = t; i < count; i += 256) s += (double)load_pix(src, pix, i * stride);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((t & 31) == 0) part[k][t >> 5] = s;
        acc[k] = (double)count;
    }
    __syncthreads();
    if (t == 0) {
        for (int k = 0; k < 2; k++) {
            double s = 0.0;
            for (int w = 0; w < 8; w++) s += part[k][w];
            q.shifts[k] = (float)(s / acc[k]);
        }
    }
}

__global__ void __launch_bounds__(256) prep_kernel(const PrepParams q) {
    if (blockIdx.x == 0 && q.shifts) staging_means(q);
    prep_body(q, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// Staging of a batch: blockIdx.y selects the pair, the x blocks stride over its elements.
__global__ void __launch_bounds__(256) batch_prep_kernel(const PrepParams *__restrict__ qs) {
    const PrepParams &q = qs[blockIdx.y];
    if (blockIdx.x == 0 && q.shifts) staging_means(q);
    prep_body(q, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

const void *batch_prep_kernel_fn() { return (const void *)batch_prep_kernel; }

__global__ void empty_result_kernel(cgs_argmin *r) {
    cgs_argmin e;
    e.cost = __int_as_float(0x7f800000);
    e.valid = 0;
    e.index = -1;
    for (int a = 0; a < 8; a++) e.params[a] = 0.0f;
    e.status = 0;
    clear_verify_fields(e);
    *r = e;
}

// Argmin of n floats: grid-stride key min, warp and block reduction, one atomicMin per
// block; the last block writes the result.  scratch = {key, ticket} preset to all ones.
__global__ void __launch_bounds__(256) argmin_kernel(const float *__restrict__ v, uint64_t n,
                                                     unsigned long long *key, unsigned int *ticket,
                                                     cgs_argmin *out) {
    __shared__ unsigned long long wk[8];
    unsigned long long best = ~0ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = make_key(__ldg(v + i), (uint32_t)i);
        best = k < best ? k : best;
    }
    best = warp_min_u64(best);
    if ((threadIdx.x & 31) == 0) wk[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) best = wk[w] < best ? wk[w] : best;
        if (best != ~0ull) atomicMin(key, best);
        __threadfence();
        // the ticket starts at 0xffffffff: the first add returns it, the last returns gridDim - 2
        const unsigned int t = atomicAdd(ticket, 1u) + 1u;
        if (t == gridDim.x - 1) {
            __threadfence();
            const unsigned long long k = atomicAdd(key, 0ull);
            cgs_argmin r;
            r.status = 0;
            clear_verify_fields(r);
            for (int a = 0; a < 8; a++) r.params[a] = 0.0f;
            if (k == ~0ull) {
                r.valid = 0;
                r.index = -1;
                r.cost = __int_as_float(0x7f800000);
            } else {
                r.valid = 1;
                r.index = (int64_t)(k & 0xffffffffull);
                r.cost = key_cost(k);
            }
            *out = r;
        }
    }
}

// Joint B x B histogram (row = fixed bin, column = moving bin) of the MI sampling at one
// parameter vector, every sample on the exact path.  hist must be zeroed.
struct HistParams {
    Plane mov, fix;
    float mov_wf, mov_hf;
    float q[8];
    float c, s;
    int bins;
    uint32_t *hist;
};

__global__ void hist_kernel(const HistParams hp) {
    const Plane mov = hp.mov, fix = hp.fix;
    const float mov_wf = hp.mov_wf, mov_hf = hp.mov_hf;
    const int bins = hp.bins;
    uint32_t *hist = hp.hist;
    const MapCoef k = coef_from_h(h_centred(hp.q, hp.c, hp.s, mov_wf / 2, mov_hf / 2));
    const float sB = (float)bins * (1.0f / 256.0f);
    const int64_t npix = (int64_t)fix.w * fix.h;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix; i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / fix.w), x = (int)(i - (int64_t)y * fix.w);
        float ex, ey;
        exact_map(k, (float)x, (float)y, ex, ey);
        if (!in_image(ey, ex, mov_wf, mov_hf)) continue;
        for (int c = 0; c < fix.c; c++) {
            const float f = fix.data[c * fix.plane + (int64_t)y * fix.pitch + x];
            const float v = bilinear_in(mov.data + c * mov.plane, mov.pitch, ey, ex);
            const int bf = min(max((int)floorf(f * sB), 0), bins - 1);
            const int bm = min(max((int)floorf(v * sB), 0), bins - 1);
            atomicAdd(&hist[bf * bins + bm], 1u);
        }
    }
}

// ---------------------------------------------------------------- launch planning

static int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }


// Sampling mode of a request (see CGS_FLAG_EXACT_SAMPLES / CGS_FLAG_FAST_SAMPLES).
bool exact_samples(int cost, int flags) {
    if (flags & CGS_FLAG_EXACT_SAMPLES) return true;
    if (flags & CGS_FLAG_FAST_SAMPLES) return false;
    return !(cost == CGS_COST_ZNCC || cost == CGS_COST_MI);
}

static bool is_scanline(int cost) {
    return cost == CGS_COST_SQD_ALT || cost == CGS_COST_NCC_ALT || cost == CGS_COST_MI_ALT;
}

// Number of rows calcMIAlt visits (the float recurrence of its row loop, on the host).
static int32_t mi_alt_rows(int rowsf) {
    float row = -0.5f;
    int n = 0;
    const float inc = 1.0f / (float)(rowsf - 1);
    while ((double)row < 0.5 && n < rowsf + 2) {
        n++;
        row = row + inc;
    }
    return n;
}

Staging staging_layout(const cgs_image &mov, const cgs_image &fix, int tex_align, int tex_pitch_align,
                              bool fix_alias, bool row_table, bool quads) {
    Staging st;
    const int C = fix.channels;
    st.mpitch = (int32_t)round_up(mov.width + 1, std::max(1, tex_pitch_align / 4));
    st.mplane = (int64_t)(mov.height + 1) * st.mpitch;
    st.fpitch = (int32_t)round_up(fix.width + (fix_alias ? 1 : 0), 4);
    st.fplane = round_up((int64_t)(fix.height + (fix_alias ? 1 : 0)) * st.fpitch, 64);
    // offsets from a tex_align-aligned origin; the allocation carries tex_align bytes of slack
    st.mov_off = (size_t)round_up(256, tex_align);
    st.fix_off = st.mov_off + (size_t)round_up(st.mplane * C * 4, 256);
    st.rows_off = st.fix_off + (size_t)round_up(st.fplane * C * 4, 256);
    st.quad_off = st.rows_off + (row_table ? (size_t)round_up((int64_t)(fix.height + 2) * 4, 256) : 0);
    st.qplane = quads ? (int64_t)mov.width * mov.height : 0;
    st.bytes = st.quad_off + (size_t)round_up(st.qplane * C * 16, 256) + (size_t)tex_align;
    return st;
}

// Origin of a staging block: the first tex_align boundary at or after the allocation.
char *staging_origin(void *scratch, int tex_align) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(scratch);
    return reinterpret_cast<char *>((a + (uintptr_t)tex_align - 1) / (uintptr_t)tex_align * (uintptr_t)tex_align);
}

// Texture objects over staged moving images, cached by (device, address, geometry): scratch
// comes from the library's pool, so steady workloads reuse the same few blocks.  Each entry
// records an event after every kernel that reads it; an entry is destroyed only after its
// event completes.  The mutex is held from lookup through launch and event record.
struct TexEntry {
    int dev;
    const void *ptr;
    int w, h;
    size_t pitch;
    cudaTextureObject_t tex;
    cudaEvent_t last;
};
static std::mutex g_tex_mu;
static std::vector<TexEntry> g_tex;
constexpr size_t kTexCacheMax = 64;

static cgs_status texture_for(int dev, const float *ptr, int w, int h, size_t pitch_bytes, TexEntry **out) {
    for (auto &e : g_tex)
        if (e.dev == dev && e.ptr == ptr && e.w == w && e.h == h && e.pitch == pitch_bytes) {
            *out = &e;
            return CGS_SUCCESS;
        }
    if (g_tex.size() >= kTexCacheMax) {
        TexEntry &old = g_tex.front();
        cudaEventSynchronize(old.last);
        cudaDestroyTextureObject(old.tex);
        cudaEventDestroy(old.last);
        g_tex.erase(g_tex.begin());
    }
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = const_cast<float *>(ptr);
    rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
    rd.res.pitch2D.width = (size_t)w;
    rd.res.pitch2D.height = (size_t)h;
    rd.res.pitch2D.pitchInBytes = pitch_bytes;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;  // outside reads 0
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    TexEntry e{dev, ptr, w, h, pitch_bytes, 0, nullptr};
    CGS_CUDA(cudaCreateTextureObject(&e.tex, &rd, &td, nullptr), "cudaCreateTextureObject");
    cudaError_t err = cudaEventCreateWithFlags(&e.last, cudaEventDisableTiming);
    if (err != cudaSuccess) {
        cudaDestroyTextureObject(e.tex);
        return cuda_fail(err, "cudaEventCreateWithFlags");
    }
    g_tex.push_back(e);
    *out = &g_tex.back();
    return CGS_SUCCESS;
}

static KernelGetter getter_for(int cost) {
    switch (cost) {
        case CGS_COST_SAD_AVG: return kernel_sad_avg;
        case CGS_COST_SAD_AVG_H: return kernel_sad_avg_h;
        case CGS_COST_SAD_SUM_T: return kernel_sad_sum_t;
        case CGS_COST_SAD_SUM_T_REF: return kernel_sad_sum_t_ref;
        case CGS_COST_SQD_REF: return kernel_sqd_ref;
        case CGS_COST_NCC_REF: return kernel_ncc_ref;
        case CGS_COST_ZNCC: return kernel_zncc;
        case CGS_COST_MI: return kernel_mi;
        default: return nullptr;
    }
}

static cgs_status check_image(const cgs_image *im, const char *name) {
    if (!im) return fail(CGS_ERROR_INVALID_VALUE, std::string(name) + " is null");
    if (!im->data) return fail(CGS_ERROR_INVALID_VALUE, std::string(name) + "->data is null");
    if (im->height < 1 || im->width < 1)
        return fail(CGS_ERROR_INVALID_VALUE, std::string(name) + " has an empty size");
    if (im->pixel < CGS_PIXEL_F32 || im->pixel > CGS_PIXEL_U16)
        return fail(CGS_ERROR_INVALID_VALUE, std::string(name) + " has an unknown pixel type");
    if (im->channels < 1 || im->channels > 4)
        return fail(CGS_ERROR_INVALID_VALUE, std::string(name) + " must have 1..4 channels");
    if ((int64_t)(im->height + 1) * im->channels > 65000 || im->width + 1 > 131000)
        return fail(CGS_ERROR_UNSUPPORTED, std::string(name) + " exceeds the 2-D texture limits");
    // flat indices are formed in FP32 by the reference; keep them exact
    if ((int64_t)(im->height + 1) * im->width * im->channels >= (int64_t)1 << 24)
        return fail(CGS_ERROR_UNSUPPORTED, std::string(name) + " exceeds 2^24 elements");
    return CGS_SUCCESS;
}

cgs_status check_grid(const cgs_grid *g) {
    if (!g) return fail(CGS_ERROR_INVALID_VALUE, "grid is null");
    if (g->dims < 1 || g->dims > 8) return fail(CGS_ERROR_INVALID_VALUE, "grid dims must be 1..8");
    for (int a = 0; a < g->dims; a++) {
        if (!std::isfinite(g->start[a]) || !std::isfinite(g->end[a]) || !std::isfinite(g->count[a]))
            return fail(CGS_ERROR_INVALID_VALUE, "grid has a non-finite start, end or count");
        if (!(g->count[a] >= 1.0f)) return fail(CGS_ERROR_INVALID_VALUE, "grid counts must be >= 1");
        if (!std::isfinite(g->resolution[a]))
            return fail(CGS_ERROR_INVALID_VALUE, "grid resolution is not finite (call cgs_grid_update)");
    }
    return CGS_SUCCESS;
}

// Validates a search request (images, grid, options) as cgs_search does; *mi_bins gets the
// MI bin count in use.
cgs_status check_request(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid, const cgs_options *options,
                         int *mi_bins) {
    cgs_status s;
    if ((s = check_image(mov, "moving")) != CGS_SUCCESS) return s;
    if ((s = check_image(fix, "fixed")) != CGS_SUCCESS) return s;
    if ((s = check_grid(grid)) != CGS_SUCCESS) return s;
    if (!options) return fail(CGS_ERROR_INVALID_VALUE, "options is null");
    const int cost = options->cost;
    if (cost < 0 || cost >= CGS_COST_COUNT) return fail(CGS_ERROR_INVALID_VALUE, "unknown cost");
    if (mov->channels != fix->channels)
        return fail(CGS_ERROR_INVALID_VALUE, "moving and fixed images must have the same channel count");
    const bool eight = !(cost == CGS_COST_SAD_SUM_T || cost == CGS_COST_SAD_SUM_T_REF);
    if (eight && grid->dims != 8) return fail(CGS_ERROR_INVALID_VALUE, "this cost needs an 8-parameter grid");
    if (!eight && grid->dims < 2) return fail(CGS_ERROR_INVALID_VALUE, "this cost needs a grid of >= 2 axes");
    if ((cost == CGS_COST_SAD_AVG_H || cost == CGS_COST_SAD_SUM_T || cost == CGS_COST_SAD_SUM_T_REF) &&
        fix->channels != 1)
        return fail(CGS_ERROR_INVALID_VALUE, "this reference functor is single-channel (CudaImage<T>)");
    *mi_bins = 32;
    if (cost == CGS_COST_MI) {
        *mi_bins = options->mi_bins == 0 ? 32 : options->mi_bins;
        if (*mi_bins < 2 || *mi_bins > 64 || (*mi_bins & (*mi_bins - 1)))
            return fail(CGS_ERROR_INVALID_VALUE, "mi_bins must be a power of two in [2, 64]");
    }
    return CGS_SUCCESS;
}

// Kernel parameters of a validated pixel-loop request, except the staged planes, scratch
// words, outputs and texture: the reference's grid tables, the evaluation order, cos/sin of
// the rotation axis, image geometry and cost options.  *n64 = grid points.
cgs_status fill_params(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid, const cgs_options &o,
                       int mi_bins, SearchParams *pp, int64_t *n64) {
    const int cost = o.cost;
    const int C = fix->channels;
    int32_t inc[8];
    grid_increments(*grid, inc, n64);
    if (*n64 > INT32_MAX) return fail(CGS_ERROR_GRID_TOO_LARGE, "grid has more than 2^31-1 points");
    SearchParams &p = *pp;
    memset(&p, 0, sizeof(p));
    if (*n64 <= 0) return CGS_SUCCESS;
    for (int a = 0; a < 8; a++) {
        p.start[a] = a < grid->dims ? grid->start[a] : 0.0f;
        p.res[a] = a < grid->dims ? grid->resolution[a] : 0.0f;
        p.inc[a] = inc[a];
    }
    p.dims = grid->dims;
    p.cost = cost;
    p.n = (uint32_t)*n64;
    p.natural = ((o.flags & CGS_FLAG_NATURAL_ORDER) || !integral_counts(*grid)) ? 1 : 0;
    p.exact_only = exact_samples(cost, o.flags) ? 1 : 0;
    if (!p.natural) {
        locality_order(cost, *grid, fix->width, fix->height, mov->width, mov->height, p.perm);
        for (int j = 0; j < grid->dims; j++) p.ocount[j] = (int32_t)grid->count[p.perm[j]];
    }
    if (cost_uses_theta(cost)) {
        // cos/sin of every axis-0 grid value, with the host libm the reference's CPU path uses
        const int32_t n0 = grid->dims > 1 ? inc[1] : (int32_t)*n64;
        if (n0 > kMaxTrig) return fail(CGS_ERROR_UNSUPPORTED, "more than 256 values on the rotation axis");
        for (int32_t i = 0; i < n0; i++) {
            const float th = std::fmaf((float)i, grid->resolution[0], grid->start[0]);
            p.trig[i] = make_float2(std::cos(th), std::sin(th));
        }
    }
    p.mov_wf = (float)mov->width;
    p.mov_hf = (float)mov->height;
    p.cx = (float)mov->width / 2;
    p.cy = (float)mov->height / 2;
    p.mi_bins = mi_bins;
    p.total_terms = (float)((double)fix->width * fix->height * C);
    p.gate_n = (float)((double)o.overlap_gate * fix->width * fix->height * C);
    return CGS_SUCCESS;
}

// Fixed-image chunking: about 16 KB of rows per chunk (at least one row).  Returns the bytes
// of one stage.
int64_t set_chunks(SearchParams *p, const Staging &st, int C, int fix_h) {
    const int64_t row_bytes = (int64_t)st.fpitch * 4 * C;
    int R = (int)std::max<int64_t>(1, 16384 / row_bytes);
    R = std::min(R, fix_h);
    p->chunk_rows = R;
    p->num_chunks = (fix_h + R - 1) / R;
    return (int64_t)R * row_bytes;
}

// Staging-kernel parameters of a pair whose scratch words start at sb (key, done, status,
// max |moving pixel|) and whose staged planes are at mstage / fstage.
PrepParams make_prep(const cgs_image *mov, const cgs_image *fix, const Staging &st, char *sb, float *mstage,
                     float *fstage) {
    PrepParams q{};  // every field zero unless set below
    q.mov_src = mov->data;
    q.fix_src = fix->data;
    q.mov_pix = mov->pixel;
    q.fix_pix = fix->pixel;
    q.mh = mov->height; q.mw = mov->width; q.fh = fix->height; q.fw = fix->width; q.c = fix->channels;
    q.mov_dst = mstage;
    q.fix_dst = fstage;
    q.mplane = st.mplane;
    q.fplane = st.fplane;
    q.mpitch = st.mpitch;
    q.fpitch = st.fpitch;
    q.key = reinterpret_cast<unsigned long long *>(sb);
    q.done = reinterpret_cast<unsigned int *>(sb + 8);
    q.status = reinterpret_cast<unsigned int *>(sb + 12);
    q.vmax = reinterpret_cast<float *>(sb + 16);
    q.shifts = reinterpret_cast<float *>(sb + 24);
    return q;
}

struct Plan {
    int G = 2, NW = 16;
};

static int accumulators(int cost) {
    switch (cost) {
        case CGS_COST_SQD_REF:
        case CGS_COST_NCC_REF: return AccN<CGS_COST_NCC_REF>::value;
        case CGS_COST_ZNCC: return AccN<CGS_COST_ZNCC>::value;
        default: return 1;
    }
}

// Bytes of a CTA's sums or MI histograms region (CtaSmem::acc).
size_t acc_bytes(int cost, int G, int NW, bool block_split, int mi_bins) {
    if (cost == CGS_COST_MI) return (size_t)(block_split ? 1 : NW) * G * (mi_bins + 1) * (mi_bins + 1) * 4;
    return (size_t)NW * G * accumulators(cost) * 32 * 4;
}

static Plan choose_plan(int cost, const cgs_options &o, int mi_bins) {
    Plan pl;
    if (cost == CGS_COST_MI) {
        pl.NW = mi_bins > 32 ? 8 : 16;
        pl.G = mi_bins > 32 ? 1 : 2;
    } else {
        pl.G = 4;
    }
    if (o.points_per_warp == 1 || o.points_per_warp == 2 || o.points_per_warp == 4) pl.G = o.points_per_warp;
    if (o.warps_per_block > 0) pl.NW = o.warps_per_block;
    return pl;
}

// Launch plan of the span kernel: points per warp (the request's 2, else 4), 16 warps, tiles of
// 32 TX columns by TH rows (256 x 16 unless the tuning variables CGS_SPAN_TX = 2 | 4 | 8 and
// CGS_SPAN_TH = 8 | 16 | 32 say otherwise), the window stage filling the shared memory that is
// left (at most CGS_SPAN_CAP 16-byte units when that is set; a stage holds the tile's fixed rows
// and its blocks' windows) and window rows padded to CGS_SPAN_PITCH (mod 8) quads.
// CGS_SPAN_CHECK=1 selects the self-checking build (every fast sample's quad address is checked
// against its window; a miss sets status bit 0x100 and skips the sample).  False where the span
// kernel does not apply: several channels, images of 32768 or more pixels a side, moving images
// with (W + 8) H of 2^22 or more, or too many tiles for shared memory.
static int env_int(const char *name, int dflt) {
    const char *v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : dflt;
}

bool span_plan(const cgs_image &mov, const cgs_image &fix, const cgs_options &o, SpanPlan *sp) {
    if (fix.channels != 1 || mov.width >= 32768 || mov.height >= 32768 || fix.width >= 32768 || fix.height >= 32768 ||
        (int64_t)(mov.width + 8) * mov.height >= span_max_quads())
        return false;
    sp->G = o.points_per_warp == 2 ? 2 : 4;
    sp->NW = 16;
    sp->TX = env_int("CGS_SPAN_TX", 8);
    sp->TH = env_int("CGS_SPAN_TH", 16);
    if (!(sp->TX == 2 || sp->TX == 4 || sp->TX == 8) || !(sp->TH == 8 || sp->TH == 16 || sp->TH == 32)) return false;
    sp->check = env_int("CGS_SPAN_CHECK", 0) != 0;
    sp->kfn = kernel_span_zncc(sp->G, sp->NW, sp->TX, sp->check);
    if (!sp->kfn) return false;
    sp->tiles_x = (fix.width + 32 * sp->TX - 1) / (32 * sp->TX);
    sp->tiles_y = (fix.height + sp->TH - 1) / sp->TH;
    const int tiles = sp->tiles_x * sp->tiles_y;
    const size_t budget = 227 * 1024, fixed = span_kernel_smem(sp->G, sp->NW, sp->TH, sp->TX, tiles, 0);
    if (fixed + (size_t)kMinSpanCap * 32 > budget) return false;
    sp->cap = (int)((budget - fixed) / 32);
    // CGS_SPAN_CAP (quads) lowers the stage size, e.g. to exercise the global-memory path
    sp->cap = std::max(kMinSpanCap, std::min(sp->cap, env_int("CGS_SPAN_CAP", sp->cap)));
    sp->cap = std::max(sp->cap, kMinSpanCap + sp->TH * 32 * sp->TX / 4);  // room for the fixed rows
    sp->pitch_mod = env_int("CGS_SPAN_PITCH", 0) & 7;
    sp->smem = span_kernel_smem(sp->G, sp->NW, sp->TH, sp->TX, tiles, sp->cap);
    return sp->smem <= budget;
}

// Launch plan of the MI span kernel: 16 warps of 2 points, bands of TH = 16 rows (CGS_SPAN_TH
// = 8 | 16 | 32), self-checking with CGS_SPAN_CHECK=1.  False where it does not apply: several
// channels, more than 32 bins (the histograms of 32 points must fit shared memory), images of
// 32768 or more pixels a side or moving images with (W + 8) H of 2^22 or more.
bool span_mi_plan(const cgs_image &mov, const cgs_image &fix, const cgs_options &o, int mi_bins, SpanPlan *sp) {
    if (fix.channels != 1 || mi_bins > 32 || mov.width >= 32768 || mov.height >= 32768 || fix.width >= 32768 ||
        fix.height >= 32768 || (int64_t)(mov.width + 8) * mov.height >= span_max_quads())
        return false;
    (void)o;
    sp->G = 2;
    sp->NW = 16;
    sp->TX = 1;
    sp->TH = env_int("CGS_SPAN_TH", 16);
    if (!(sp->TH == 8 || sp->TH == 16 || sp->TH == 32)) return false;
    sp->check = env_int("CGS_SPAN_CHECK", 0) != 0;
    sp->kfn = kernel_span_mi(sp->NW, sp->check);
    if (!sp->kfn) return false;
    sp->tiles_x = 1;
    sp->tiles_y = (fix.height + sp->TH - 1) / sp->TH;
    sp->cap = 0;
    sp->pitch_mod = 0;
    sp->smem = span_mi_kernel_smem(sp->NW, sp->TH, mi_bins);
    return sp->smem <= 227 * 1024;
}

// The scanline functors: staging with both images aliased, the calcMIAlt row table, one warp
// per grid point.  Arguments are validated by cgs_search.
static cgs_status search_scanline(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid,
                                  const cgs_options &o, float *costs, cgs_argmin *result, cudaStream_t stream,
                                  const DeviceInfo &di) {
    const int cost = o.cost;
    const int C = fix->channels;
    const void *kfn = kernel_scan(cost, C);
    if (!kfn) return fail(CGS_ERROR_UNSUPPORTED, "no scanline kernel for this channel count");
    int32_t inc[8];
    int64_t n64;
    grid_increments(*grid, inc, &n64);
    if (n64 > INT32_MAX) return fail(CGS_ERROR_GRID_TOO_LARGE, "grid has more than 2^31-1 points");
    if (n64 <= 0) {
        empty_result_kernel<<<1, 1, 0, stream>>>(result);
        CGS_CUDA(cudaGetLastError(), "empty_result_kernel");
        return CGS_SUCCESS;
    }
    SearchParams p;
    memset(&p, 0, sizeof(p));
    for (int a = 0; a < 8; a++) {
        p.start[a] = a < grid->dims ? grid->start[a] : 0.0f;
        p.res[a] = a < grid->dims ? grid->resolution[a] : 0.0f;
        p.inc[a] = inc[a];
    }
    p.dims = grid->dims;
    p.cost = cost;
    p.n = (uint32_t)n64;
    p.natural = ((o.flags & CGS_FLAG_NATURAL_ORDER) || !integral_counts(*grid)) ? 1 : 0;
    if (!p.natural) {
        locality_order(cost == CGS_COST_MI_ALT ? CGS_COST_SAD_AVG : cost, *grid, fix->width, fix->height, mov->width,
                       mov->height, p.perm);
        for (int j = 0; j < grid->dims; j++) p.ocount[j] = (int32_t)grid->count[p.perm[j]];
    }
    const int32_t n0 = grid->dims > 1 ? inc[1] : (int32_t)n64;
    if (n0 > kMaxTrig) return fail(CGS_ERROR_UNSUPPORTED, "more than 256 values on the rotation axis");
    for (int32_t i = 0; i < n0; i++) {
        const float th = std::fmaf((float)i, grid->resolution[0], grid->start[0]);
        p.trig[i] = make_float2(std::cos(th), std::sin(th));
    }
    p.mov_wf = (float)mov->width;
    p.mov_hf = (float)mov->height;
    p.cx = (float)mov->width / 2;
    p.cy = (float)mov->height / 2;
    const bool mi = cost == CGS_COST_MI_ALT;
    p.n_rows = mi ? mi_alt_rows(fix->height) : fix->height;

    const Staging st = staging_layout(*mov, *fix, di.tex_align, di.tex_pitch_align, true, mi);
    cgs_status s;
    cudaMemPool_t pool;
    if ((s = get_pool(di.dev, &pool)) != CGS_SUCCESS) return s;
    void *scratch = nullptr;
    CGS_CUDA(cudaMallocFromPoolAsync(&scratch, st.bytes, pool, stream), "cudaMallocFromPoolAsync");
    char *sb = staging_origin(scratch, di.tex_align);
    p.key = reinterpret_cast<unsigned long long *>(sb);
    p.done = reinterpret_cast<unsigned int *>(sb + 8);
    p.status = reinterpret_cast<unsigned int *>(sb + 12);
    p.vmax = reinterpret_cast<float *>(sb + 16);
    p.shifts = reinterpret_cast<const float *>(sb + 24);
    float *mstage = reinterpret_cast<float *>(sb + st.mov_off);
    float *fstage = reinterpret_cast<float *>(sb + st.fix_off);
    float *rtab = mi ? reinterpret_cast<float *>(sb + st.rows_off) : nullptr;
    p.mov = Plane{mstage, mov->height, mov->width, C, st.mpitch, st.mplane};
    p.fix = Plane{fstage, fix->height, fix->width, C, st.fpitch, st.fplane};
    p.row_table = rtab;
    p.costs = costs;
    p.result = result;

    PrepParams q{};  // every field zero unless set below

    q.mov_src = mov->data;
    q.fix_src = fix->data;
    q.mov_pix = mov->pixel;
    q.fix_pix = fix->pixel;
    q.mh = mov->height; q.mw = mov->width; q.fh = fix->height; q.fw = fix->width; q.c = C;
    q.mov_dst = mstage;
    q.fix_dst = fstage;
    q.mplane = st.mplane;
    q.fplane = st.fplane;
    q.mpitch = st.mpitch;
    q.fpitch = st.fpitch;
    q.key = p.key;
    q.done = p.done;
    q.status = p.status;
    q.vmax = reinterpret_cast<float *>(sb + 16);
    q.fix_alias = 1;
    q.row_table = rtab;
    q.rowsf = fix->height;
    cudaError_t e = cudaMemsetAsync(sb, 0, 256, stream);
    if (e == cudaSuccess) {
        const int64_t prep_elems = (st.mplane + st.fplane) * C;
        prep_kernel<<<(int)std::min<int64_t>((prep_elems + 255) / 256, (int64_t)di.sms * 8), 256, 0, stream>>>(q);
        e = cudaGetLastError();
    }
    const size_t smem = scan_smem_bytes(cost);
    const int threads = kScanWarps * 32;
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
    if (e == cudaSuccess && per_sm >= 1) {
        const uint32_t blocks = std::min<uint32_t>((p.n + kScanWarps - 1) / kScanWarps, (uint32_t)(di.sms * per_sm));
        void *args[] = {&p};
        e = cudaLaunchKernel(kfn, dim3(blocks), dim3(threads), args, smem, stream);
    }
    cudaFreeAsync(scratch, stream);
    if (e != cudaSuccess) return cuda_fail(e, "scanline kernel");
    if (per_sm < 1) return fail(CGS_ERROR_UNSUPPORTED, "scanline kernel does not fit on an SM");
    return CGS_SUCCESS;
}

}  // namespace cgs

using namespace cgs;

// ================================================================= C ABI

extern "C" {

int32_t cgs_version(void) { return 100; }

const char *cgs_status_string(cgs_status s) {
    switch (s) {
        case CGS_SUCCESS: return "success";
        case CGS_ERROR_INVALID_VALUE: return "invalid value";
        case CGS_ERROR_UNSUPPORTED: return "unsupported";
        case CGS_ERROR_GRID_TOO_LARGE: return "grid too large";
        case CGS_ERROR_OUT_OF_MEMORY: return "out of memory";
        case CGS_ERROR_CUDA: return "CUDA error";
        case CGS_ERROR_NO_DEVICE: return "no usable device";
        case CGS_ERROR_DEVICE_TIMEOUT: return "device wait timed out";
    }
    return "unknown status";
}

const char *cgs_last_error(void) { return g_last_error.c_str(); }

cgs_status cgs_grid_update(cgs_grid *g, int32_t changed_axis) {
    if (!g || g->dims < 1 || g->dims > 8) return fail(CGS_ERROR_INVALID_VALUE, "grid is null or dims not in 1..8");
    const int D = g->dims;
    auto one = [&](int a, bool changed) {
        // updateProcess (cudaGridSearch.cuh:241-270): a step below 1e-7 * count collapses
        // the axis to one sample; the comparison is done in double, as there.
        if ((double)std::fabs(g->end[a] - g->start[a]) < 1.0e-7 * (double)g->count[a]) g->count[a] = 1;
        if (g->count[a] == 1) {
            g->resolution[a] = 2 * (g->end[a] - g->start[a]);
        } else if (changed) {
            g->resolution[a] = (float)(int32_t)(g->end[a] - g->start[a]) / (g->count[a] - 1);
        } else {
            g->resolution[a] = (g->end[a] - g->start[a]) / (g->count[a] - 1);
        }
    };
    if (changed_axis >= 0 && changed_axis < D) {
        one(changed_axis, true);
    } else {
        for (int a = 0; a < D; a++) one(a, false);
    }
    return CGS_SUCCESS;
}

cgs_status cgs_grid_num_elements(const cgs_grid *g, uint64_t *num) {
    if (!num) return fail(CGS_ERROR_INVALID_VALUE, "num is null");
    cgs_status s = check_grid(g);
    if (s != CGS_SUCCESS) return s;
    int32_t inc[8];
    int64_t n;
    grid_increments(*g, inc, &n);
    *num = n < 0 ? 0 : (uint64_t)n;
    return CGS_SUCCESS;
}

cgs_status cgs_grid_point(const cgs_grid *g, int64_t index, float out[8]) {
    if (!out) return fail(CGS_ERROR_INVALID_VALUE, "out is null");
    cgs_status s = check_grid(g);
    if (s != CGS_SUCCESS) return s;
    int32_t inc[8];
    int64_t n;
    grid_increments(*g, inc, &n);
    if (index < 0 || index > INT32_MAX) return fail(CGS_ERROR_INVALID_VALUE, "index out of range");
    int32_t rem = (int32_t)index, ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int a = g->dims - 1; a >= 0; a--) {
        ax[a] = rem / inc[a];
        rem -= ax[a] * inc[a];
    }
    for (int a = 0; a < 8; a++)
        out[a] = a < g->dims ? std::fmaf((float)ax[a], g->resolution[a], g->start[a]) : 0.0f;
    return CGS_SUCCESS;
}

}  // extern "C"

namespace cgs {

// The body of cgs_search.  ext = nullptr: scratch from the stream-ordered pool.  ext != nullptr
// (span searches only, else CGS_ERROR_UNSUPPORTED): the caller's scratch block ext->ptr of
// ext->bytes bytes holds the staging block, the span tables and the verification header; with
// ext->query set only the block's size is computed into ext->bytes and nothing is enqueued.
static cgs_status search_core(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid,
                              const cgs_options *options, float *costs, cgs_argmin *result, cudaStream_t stream,
                              ExtScratch *ext) {
    cgs_status s;
    int mi_bins = 32;
    if ((s = check_request(mov, fix, grid, options, &mi_bins)) != CGS_SUCCESS) return s;
    const bool query = ext && ext->query;
    if (!result && !query) return fail(CGS_ERROR_INVALID_VALUE, "result is null");
    const cgs_options o = *options;
    const int cost = o.cost;
    if (is_scanline(cost) && ext) return fail(CGS_ERROR_UNSUPPORTED, "caller scratch: span searches only");
    if (is_scanline(cost)) {
        DeviceInfo dsi;
        if ((s = device_info(&dsi)) != CGS_SUCCESS) return s;
        return search_scanline(mov, fix, grid, o, costs, result, stream, dsi);
    }
    KernelGetter getter = getter_for(cost);
    if (!getter) return fail(CGS_ERROR_UNSUPPORTED, "cost not implemented by this build");
    const int C = fix->channels;
    const Plan pl = choose_plan(cost, o, mi_bins);
    // taps: pre-gathered quads where the fast sampling path runs (measured faster than texture
    // gathers there); texture gathers (MI: scalar loads) for exact sampling and for MI
    const bool fast_path = !exact_samples(cost, o.flags) && cost != CGS_COST_MI;
    // zero-mean NCC and MI on the fast path: the span kernels (row decisions; ZNCC with
    // shared-memory windows, MI with shared-memory histograms); both read span-form quads
    SpanPlan sp;
    const bool per_sample = (o.flags & CGS_FLAG_PER_SAMPLE_DECISIONS) != 0;
    const bool span = cost == CGS_COST_ZNCC && fast_path && !(o.flags & CGS_FLAG_TEXTURE_TAPS) && !per_sample &&
                      span_plan(*mov, *fix, o, &sp);
    const bool span_mi = cost == CGS_COST_MI && !exact_samples(cost, o.flags) && !per_sample &&
                         !(o.flags & (CGS_FLAG_TEXTURE_TAPS | CGS_FLAG_QUAD_TAPS)) &&
                         span_mi_plan(*mov, *fix, o, mi_bins, &sp);
    const bool quads = (o.flags & CGS_FLAG_QUAD_TAPS) || (fast_path && !(o.flags & CGS_FLAG_TEXTURE_TAPS)) || span_mi;
    const void *kfn = (span || span_mi) ? sp.kfn : getter(C, pl.G, pl.NW, quads);
    if (!kfn) return fail(CGS_ERROR_UNSUPPORTED, "no kernel for this channel count / tuning");
    if (ext && !(span || span_mi)) return fail(CGS_ERROR_UNSUPPORTED, "caller scratch: span searches only");

    DeviceInfo di;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;

    SearchParams p;
    int64_t n64;
    if ((s = fill_params(mov, fix, grid, o, mi_bins, &p, &n64)) != CGS_SUCCESS) return s;
    if (n64 <= 0) {
        if (query) {
            ext->bytes = 0;
            return CGS_SUCCESS;
        }
        empty_result_kernel<<<1, 1, 0, stream>>>(result);
        CGS_CUDA(cudaGetLastError(), "empty_result_kernel");
        return CGS_SUCCESS;
    }

    // staged layout
    const Staging st = staging_layout(*mov, *fix, di.tex_align, di.tex_pitch_align, false, false, quads);
    const int64_t stage_bytes = set_chunks(&p, st, C, fix->height);
    const size_t smem = (span || span_mi) ? sp.smem
                                          : cta_smem_bytes(pl.G, pl.NW, (size_t)stage_bytes,
                                                           acc_bytes(cost, pl.G, pl.NW, false, mi_bins));
    if (smem > 227 * 1024) return fail(CGS_ERROR_UNSUPPORTED, "shared-memory plan exceeds 227 KB");
    if (span || span_mi) {
        p.tile_h = sp.TH;
        p.tiles_x = sp.tiles_x;
        p.tiles_y = sp.tiles_y;
        p.win_cap = sp.cap;
        p.win_pitch_mod = sp.pitch_mod;
    }

    // the span kernels' tables follow the staging block: the ZNCC kernel's row prefix sums (W_f + 1
    // FP64 pairs per row), the MI kernel's fixed bins (int32, the fixed plane's pitch)
    const size_t prefix_off = (size_t)round_up((int64_t)(st.bytes - (size_t)di.tex_align), 256);
    const size_t prefix_bytes = span      ? (size_t)fix->height * (size_t)(fix->width + 1) * sizeof(double2)
                                : span_mi ? (size_t)fix->height * (size_t)st.fpitch * sizeof(int32_t)
                                          : 0;
    const size_t main_bytes = st.bytes + (prefix_bytes ? prefix_bytes + 256 : 0);
    const bool verify = !(o.flags & CGS_FLAG_NO_VERIFY) && verify_supported(cost);
    const size_t vbytes = verify ? verify_scratch_bytes() + (costs ? 0 : (size_t)p.n * 4) : 0;
    const size_t ext_bytes = (size_t)round_up((int64_t)main_bytes, 256) + vbytes;
    if (query) {
        ext->bytes = ext_bytes;
        ext->points_per_task = (uint32_t)(sp.NW * sp.G);
        return CGS_SUCCESS;
    }
    if (ext && ext->bytes < ext_bytes) return fail(CGS_ERROR_INVALID_VALUE, "caller scratch smaller than the search needs");
    cudaMemPool_t pool = nullptr;
    if (!ext && (s = get_pool(di.dev, &pool)) != CGS_SUCCESS) return s;
    void *scratch = nullptr;
    if (ext) scratch = ext->ptr;
    else CGS_CUDA(cudaMallocFromPoolAsync(&scratch, main_bytes, pool, stream), "cudaMallocFromPoolAsync");
    // pool blocks go back to the pool in stream order; a caller's block stays the caller's
    auto release = [&](void *ptr) {
        if (!ext && ptr) cudaFreeAsync(ptr, stream);
    };
    char *sb = staging_origin(scratch, di.tex_align);
    if (span) p.fix_prefix = reinterpret_cast<const double2 *>(sb + prefix_off);
    if (span_mi) {
        p.span_rows = reinterpret_cast<const float *>(sb + prefix_off);
        p.span_rows_header = reinterpret_cast<const float *>(sb + 32);  // zeroed with the header
    }
    p.key = reinterpret_cast<unsigned long long *>(sb);
    p.done = reinterpret_cast<unsigned int *>(sb + 8);
    p.status = reinterpret_cast<unsigned int *>(sb + 12);
    p.vmax = reinterpret_cast<float *>(sb + 16);
    p.shifts = reinterpret_cast<const float *>(sb + 24);
    float *mstage = reinterpret_cast<float *>(sb + st.mov_off);
    float *fstage = reinterpret_cast<float *>(sb + st.fix_off);
    p.mov = Plane{mstage, mov->height, mov->width, C, st.mpitch, st.mplane};
    p.fix = Plane{fstage, fix->height, fix->width, C, st.fpitch, st.fplane};
    p.costs = costs;
    p.result = result;
    // FP64 verification pass after the search: its header, and a cost dump when the caller
    // keeps none (the pass reads the FP32 costs of the band around the minimum)
    void *vblock = nullptr;
    if (verify) {
        if (ext) {
            vblock = ext->ptr + round_up((int64_t)main_bytes, 256);
        } else {
            cudaError_t ve = cudaMallocFromPoolAsync(&vblock, vbytes, pool, stream);
            if (ve != cudaSuccess) {
                release(scratch);
                return cuda_fail(ve, "cudaMallocFromPoolAsync");
            }
        }
        if (!costs) p.costs = reinterpret_cast<float *>(static_cast<char *>(vblock) + verify_scratch_bytes());
    }
    if (quads) {
        p.mov_quad = reinterpret_cast<const float4 *>(sb + st.quad_off);
        p.quad_pitch = mov->width;
        p.quad_plane = st.qplane;
    }

    PrepParams q = make_prep(mov, fix, st, sb, mstage, fstage);
    if (quads) {
        q.quad_dst = reinterpret_cast<float4 *>(sb + st.quad_off);
        q.qplane = st.qplane;
        q.quad_form = (span || span_mi) ? 1 : 0;
    }
    const int64_t prep_elems = (st.mplane + st.fplane) * C;
    const int prep_blocks = (int)std::min<int64_t>((prep_elems + 255) / 256, (int64_t)di.sms * 8);
    cudaError_t e = cudaMemsetAsync(sb, 0, 256, stream);
    if (e == cudaSuccess) {
        prep_kernel<<<prep_blocks, 256, 0, stream>>>(q);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && span)
        e = launch_span_prep(fstage, st.fpitch, fix->width, fix->height, const_cast<double2 *>(p.fix_prefix),
                             reinterpret_cast<float4 *>(sb + st.quad_off), st.qplane, p.shifts, stream);
    if (e == cudaSuccess && span_mi)
        e = launch_span_prep_mi(fstage, st.fpitch, fix->width, fix->height, mi_bins,
                                reinterpret_cast<int32_t *>(sb + prefix_off),
                                reinterpret_cast<const float4 *>(sb + st.quad_off), st.qplane,
                                reinterpret_cast<unsigned int *>(sb + 32), stream);
    if (e != cudaSuccess) {
        release(vblock);
        release(scratch);
        return cuda_fail(e, "prep_kernel");
    }

    const int threads = ((span || span_mi) ? sp.NW : pl.NW) * 32;
    const uint32_t per_task = (span || span_mi) ? (uint32_t)(sp.NW * sp.G) : (uint32_t)(pl.NW * pl.G);
    p.num_tasks = (p.n + per_task - 1) / per_task;
    e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && !span && !span_mi)
        e = cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxL1);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
    if (e != cudaSuccess || per_sm < 1) {
        release(vblock);
        release(scratch);
        return e != cudaSuccess ? cuda_fail(e, "search kernel setup")
                                : fail(CGS_ERROR_UNSUPPORTED, "search kernel does not fit on an SM");
    }
    const uint32_t blocks = std::min<uint32_t>(p.num_tasks, (uint32_t)(di.sms * per_sm));
    void *args[] = {&p};
    if (ext) {  // the span kernels read tap quads, no texture
        p.mov_tex = 0;
        e = cudaLaunchKernel(kfn, dim3(blocks), dim3(threads), args, smem, stream);
    } else {
        std::lock_guard<std::mutex> lock(g_tex_mu);
        TexEntry *te = nullptr;
        s = texture_for(di.dev, mstage, mov->width + 1, C * (mov->height + 1), (size_t)st.mpitch * 4, &te);
        if (s == CGS_SUCCESS) {
            p.mov_tex = te->tex;
            e = cudaLaunchKernel(kfn, dim3(blocks), dim3(threads), args, smem, stream);
            if (e == cudaSuccess) e = cudaEventRecord(te->last, stream);
        }
    }
    if (s == CGS_SUCCESS && e == cudaSuccess && verify) {
        e = cudaMemsetAsync(vblock, 0, 8, stream);  // band count and CTA ticket
        if (e == cudaSuccess) s = launch_verify(p, vblock, stream, di.sms);
    }
    release(vblock);
    release(scratch);
    if (s != CGS_SUCCESS) return s;
    if (e != cudaSuccess) return cuda_fail(e, "search kernel launch");
    return CGS_SUCCESS;
}

bool span_route_bytes(const cgs_pair &q, size_t *bytes, uint32_t *points_per_task) {
    static float dummy;  // stands for a caller's cost dump: only its presence matters here
    ExtScratch x;
    x.query = true;
    const std::string keep = g_last_error;
    const cgs_status s = search_core(&q.moving, &q.fixed, &q.grid, &q.options, q.costs ? &dummy : nullptr, nullptr,
                                     nullptr, &x);
    g_last_error = keep;  // "not a span search" is an answer here, not an error
    if (s != CGS_SUCCESS || x.bytes == 0) return false;
    *bytes = x.bytes;
    *points_per_task = x.points_per_task;
    return true;
}

cgs_status span_route_enqueue(const cgs_pair &q, char *scratch, size_t bytes, cudaStream_t stream) {
    ExtScratch x;
    x.ptr = scratch;
    x.bytes = bytes;
    return search_core(&q.moving, &q.fixed, &q.grid, &q.options, q.costs, q.result, stream, &x);
}

}  // namespace cgs

extern "C" {

cgs_status cgs_search(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid, const cgs_options *options,
                      float *costs, cgs_argmin *result, cgs_stream_t stream_) {
    return search_core(mov, fix, grid, options, costs, result, (cudaStream_t)stream_, nullptr);
}

cgs_status cgs_search_sync(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid,
                           const cgs_options *options, float *costs, cgs_argmin *host_result, cgs_stream_t stream_) {
    if (!host_result) return fail(CGS_ERROR_INVALID_VALUE, "host_result is null");
    cudaStream_t stream = (cudaStream_t)stream_;
    DeviceInfo di;
    cgs_status s;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;
    cudaMemPool_t pool;
    if ((s = get_pool(di.dev, &pool)) != CGS_SUCCESS) return s;
    void *dres = nullptr;
    CGS_CUDA(cudaMallocFromPoolAsync(&dres, sizeof(cgs_argmin), pool, stream), "cudaMallocFromPoolAsync");
    s = cgs_search(mov, fix, grid, options, costs, static_cast<cgs_argmin *>(dres), stream_);
    if (s == CGS_SUCCESS) {
        cudaError_t e = cudaMemcpyAsync(host_result, dres, sizeof(cgs_argmin), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) s = cuda_fail(e, "result copy");
        else if (host_result->status & (int32_t)kStatusSpanBounds)
            s = fail(CGS_ERROR_CUDA, "span kernel self-check: a sample's quad address left its window");
        else if (host_result->status != CGS_SUCCESS) s = fail((cgs_status)host_result->status, "device wait timed out");
    }
    cudaFreeAsync(dres, stream);
    return s;
}

// ================================================================= allocation-free search
//
// Some callers cannot allocate device memory while they run: a real-time or streaming loop
// that reserves its whole memory budget up front (an allocation there can block on an
// implicit synchronisation or fail once a caching allocator such as PyTorch's holds nearly
// all free memory), or a host that owns device memory through its own pool and forbids
// other allocations.  cgs_search takes its scratch from a stream-ordered pool;
// cgs_search_noalloc takes it from the fixed array below instead and calls no allocation
// routine at all.  Every GPU that loads this library holds the array until the process
// exits.

}  // extern "C"

namespace cgs {

// Maximum scratch of an allocation-free search: the staged moving and fixed images
// (C planes of (H_m + 1) x pitch and H_f x pitch floats) plus a 256-byte header.
constexpr size_t kStaticScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

static std::mutex g_static_mu;
static char *g_static_ptr[64] = {};

// The device address of g_static_scratch on the current device.  In host code the array's
// name stands for a host-side shadow, not a device address, so it is looked up once per
// device with cudaGetSymbolAddress while that device is current.  The address is kept for the
// life of the process: after cudaDeviceReset (or any teardown of the device's primary context)
// the module is loaded again and may be placed elsewhere, so this entry point must not be used
// across a device reset.
static cgs_status static_scratch(int dev, char **out) {
    if (dev < 0 || dev >= 64) return fail(CGS_ERROR_NO_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[dev]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        g_static_ptr[dev] = static_cast<char *>(ptr);
    }
    *out = g_static_ptr[dev];
    return CGS_SUCCESS;
}

static const void *loads_kernel_for(int cost, int C) {
    switch (cost) {
        case CGS_COST_SAD_AVG: return kernel_sad_avg_loads(C);
        case CGS_COST_SAD_AVG_H: return kernel_sad_avg_h_loads(C);
        case CGS_COST_SAD_SUM_T: return kernel_sad_sum_t_loads(C);
        case CGS_COST_SAD_SUM_T_REF: return kernel_sad_sum_t_ref_loads(C);
        case CGS_COST_SQD_REF: return kernel_sqd_ref_loads(C);
        case CGS_COST_NCC_REF: return kernel_ncc_ref_loads(C);
        case CGS_COST_ZNCC: return kernel_zncc_loads(C);
        default: return nullptr;
    }
}

}  // namespace cgs

extern "C" {

cgs_status cgs_search_noalloc(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid,
                              const cgs_options *options, float *costs, cgs_argmin *result, cgs_stream_t stream_) {
    cudaStream_t stream = (cudaStream_t)stream_;
    cgs_status s;
    int mi_bins = 32;
    if ((s = check_request(mov, fix, grid, options, &mi_bins)) != CGS_SUCCESS) return s;
    if (!result) return fail(CGS_ERROR_INVALID_VALUE, "result is null");
    const cgs_options o = *options;
    const int cost = o.cost;
    const int C = fix->channels;
    if (is_scanline(cost))
        return fail(CGS_ERROR_UNSUPPORTED,
                    "cgs_search_noalloc runs the pixel-loop costs only; the scanline functors (SQD_ALT, NCC_ALT, "
                    "MI_ALT) need cgs_search");
    // fixed tuning: the plan's MI shape, else 4 points per warp and 16 warps per CTA
    Plan pl;
    const void *kfn = nullptr;
    if (cost == CGS_COST_MI) {
        cgs_options od = o;
        od.points_per_warp = 0;
        od.warps_per_block = 0;
        pl = choose_plan(cost, od, mi_bins);
        kfn = kernel_mi(C, pl.G, pl.NW, false);
    } else {
        pl.G = 4;
        pl.NW = 16;
        kfn = loads_kernel_for(cost, C);
    }
    if (!kfn) return fail(CGS_ERROR_UNSUPPORTED, "no allocation-free kernel for this cost / channel count");

    DeviceInfo di;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;
    const Staging st = staging_layout(*mov, *fix, 256, di.tex_pitch_align);
    if (st.bytes > kStaticScratchBytes)
        return fail(CGS_ERROR_INVALID_VALUE,
                    "images too large for cgs_search_noalloc: staging needs " + std::to_string(st.bytes) +
                        " bytes, the static scratch holds " + std::to_string(kStaticScratchBytes));
    char *scratch = nullptr;
    if ((s = static_scratch(di.dev, &scratch)) != CGS_SUCCESS) return s;

    SearchParams p;
    int64_t n64;
    if ((s = fill_params(mov, fix, grid, o, mi_bins, &p, &n64)) != CGS_SUCCESS) return s;
    if (n64 <= 0) {
        empty_result_kernel<<<1, 1, 0, stream>>>(result);
        CGS_CUDA(cudaGetLastError(), "empty_result_kernel");
        return CGS_SUCCESS;
    }

    const int64_t stage_bytes = set_chunks(&p, st, C, fix->height);
    const size_t smem = cta_smem_bytes(pl.G, pl.NW, (size_t)stage_bytes, acc_bytes(cost, pl.G, pl.NW, false, mi_bins));
    if (smem > 227 * 1024) return fail(CGS_ERROR_UNSUPPORTED, "shared-memory plan exceeds 227 KB");

    // the static array is 256-byte aligned: the staging origin is its start
    char *sb = scratch;
    p.key = reinterpret_cast<unsigned long long *>(sb);
    p.done = reinterpret_cast<unsigned int *>(sb + 8);
    p.status = reinterpret_cast<unsigned int *>(sb + 12);
    p.vmax = reinterpret_cast<float *>(sb + 16);
    p.shifts = reinterpret_cast<const float *>(sb + 24);
    float *mstage = reinterpret_cast<float *>(sb + st.mov_off);
    float *fstage = reinterpret_cast<float *>(sb + st.fix_off);
    p.mov = Plane{mstage, mov->height, mov->width, C, st.mpitch, st.mplane};
    p.fix = Plane{fstage, fix->height, fix->width, C, st.fpitch, st.fplane};
    p.costs = costs;
    p.result = result;
    p.mov_tex = 0;  // the plain-load kernels read no texture

    PrepParams q = make_prep(mov, fix, st, sb, mstage, fstage);
    // the array keeps the previous call's contents: the header (argmin key, completion
    // counter, status, max |pixel|) is cleared here and the staging kernel rewrites every
    // staged element
    cudaError_t e = cudaMemsetAsync(sb, 0, 256, stream);
    if (e == cudaSuccess) {
        const int64_t prep_elems = (st.mplane + st.fplane) * C;
        prep_kernel<<<(int)std::min<int64_t>((prep_elems + 255) / 256, (int64_t)di.sms * 8), 256, 0, stream>>>(q);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(e, "prep_kernel");
    const int threads = pl.NW * 32;
    const uint32_t per_task = (uint32_t)(pl.NW * pl.G);
    p.num_tasks = (p.n + per_task - 1) / per_task;
    e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                   cudaSharedmemCarveoutMaxL1);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
    if (e != cudaSuccess) return cuda_fail(e, "search kernel setup");
    if (per_sm < 1) return fail(CGS_ERROR_UNSUPPORTED, "search kernel does not fit on an SM");
    const uint32_t blocks = std::min<uint32_t>(p.num_tasks, (uint32_t)(di.sms * per_sm));
    void *args[] = {&p};
    e = cudaLaunchKernel(kfn, dim3(blocks), dim3(threads), args, smem, stream);
    if (e != cudaSuccess) return cuda_fail(e, "search kernel launch");
    return CGS_SUCCESS;
}

cgs_status cgs_mi_histogram(const cgs_image *mov, const cgs_image *fix, const float params[8], int32_t bins,
                            uint32_t *hist, cgs_stream_t stream_) {
    cudaStream_t stream = (cudaStream_t)stream_;
    cgs_status s;
    if ((s = check_image(mov, "moving")) != CGS_SUCCESS) return s;
    if ((s = check_image(fix, "fixed")) != CGS_SUCCESS) return s;
    if (!params || !hist) return fail(CGS_ERROR_INVALID_VALUE, "params or hist is null");
    if (mov->channels != fix->channels) return fail(CGS_ERROR_INVALID_VALUE, "channel counts differ");
    if (bins < 2 || bins > 256 || (bins & (bins - 1)))
        return fail(CGS_ERROR_INVALID_VALUE, "bins must be a power of two in [2, 256]");
    DeviceInfo di;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;
    const int C = fix->channels;
    const Staging st = staging_layout(*mov, *fix, di.tex_align, di.tex_pitch_align);
    cudaMemPool_t pool;
    if ((s = get_pool(di.dev, &pool)) != CGS_SUCCESS) return s;
    void *scratch = nullptr;
    CGS_CUDA(cudaMallocFromPoolAsync(&scratch, st.bytes, pool, stream), "cudaMallocFromPoolAsync");
    char *sb = staging_origin(scratch, di.tex_align);
    float *mstage = reinterpret_cast<float *>(sb + st.mov_off);
    float *fstage = reinterpret_cast<float *>(sb + st.fix_off);
    PrepParams q{};  // every field zero unless set below
    q.mov_src = mov->data; q.fix_src = fix->data; q.mov_pix = mov->pixel; q.fix_pix = fix->pixel;
    q.mh = mov->height; q.mw = mov->width; q.fh = fix->height; q.fw = fix->width; q.c = C;
    q.mov_dst = mstage; q.fix_dst = fstage; q.mplane = st.mplane; q.fplane = st.fplane;
    q.mpitch = st.mpitch; q.fpitch = st.fpitch;
    q.key = reinterpret_cast<unsigned long long *>(sb);
    q.done = reinterpret_cast<unsigned int *>(sb + 8);
    q.status = reinterpret_cast<unsigned int *>(sb + 12);
    q.vmax = reinterpret_cast<float *>(sb + 16);
    cudaError_t e = cudaMemsetAsync(sb, 0, 256, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, (size_t)bins * bins * 4, stream);
    const int64_t prep_elems = (st.mplane + st.fplane) * C;
    if (e == cudaSuccess) {
        prep_kernel<<<(int)std::min<int64_t>((prep_elems + 255) / 256, (int64_t)di.sms * 8), 256, 0, stream>>>(q);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        HistParams hp{};
        hp.mov = Plane{mstage, mov->height, mov->width, C, st.mpitch, st.mplane};
        hp.fix = Plane{fstage, fix->height, fix->width, C, st.fpitch, st.fplane};
        hp.mov_wf = (float)mov->width;
        hp.mov_hf = (float)mov->height;
        for (int a = 0; a < 8; a++) hp.q[a] = params[a];
        hp.c = std::cos(params[0]);  // the host libm, as for cgs_search
        hp.s = std::sin(params[0]);
        hp.bins = bins;
        hp.hist = hist;
        const int64_t npix = (int64_t)fix->width * fix->height;
        hist_kernel<<<(int)std::min<int64_t>((npix + 255) / 256, (int64_t)di.sms * 4), 256, 0, stream>>>(hp);
        e = cudaGetLastError();
    }
    cudaFreeAsync(scratch, stream);
    if (e != cudaSuccess) return cuda_fail(e, "mi histogram");
    return CGS_SUCCESS;
}

cgs_status cgs_argmin_f32(const float *values, uint64_t n, cgs_argmin *result, cgs_stream_t stream_) {
    cudaStream_t stream = (cudaStream_t)stream_;
    if (!result) return fail(CGS_ERROR_INVALID_VALUE, "result is null");
    if (n > 0 && !values) return fail(CGS_ERROR_INVALID_VALUE, "values is null");
    if (n > 0xffffffffull) return fail(CGS_ERROR_GRID_TOO_LARGE, "more than 2^32 values");
    DeviceInfo di;
    cgs_status s;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;
    if (n == 0) {
        empty_result_kernel<<<1, 1, 0, stream>>>(result);
        CGS_CUDA(cudaGetLastError(), "empty_result_kernel");
        return CGS_SUCCESS;
    }
    cudaMemPool_t pool;
    if ((s = get_pool(di.dev, &pool)) != CGS_SUCCESS) return s;
    void *scratch = nullptr;
    CGS_CUDA(cudaMallocFromPoolAsync(&scratch, 16, pool, stream), "cudaMallocFromPoolAsync");
    cudaError_t e = cudaMemsetAsync(scratch, 0xff, 16, stream);
    const int blocks = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)di.sms * 4);
    if (e == cudaSuccess) {
        argmin_kernel<<<blocks, 256, 0, stream>>>(values, n, static_cast<unsigned long long *>(scratch),
                                                  reinterpret_cast<unsigned int *>(static_cast<char *>(scratch) + 8),
                                                  result);
        e = cudaGetLastError();
    }
    cudaFreeAsync(scratch, stream);
    if (e != cudaSuccess) return cuda_fail(e, "argmin");
    return CGS_SUCCESS;
}

}  // extern "C"
