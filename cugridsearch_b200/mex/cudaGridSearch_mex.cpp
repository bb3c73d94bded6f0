/*
 * cudaGridSearch_mex.cpp -- MATLAB entry point of the B200 grid search (the reference's
 * MEX target is src/gpu/cudaGridSearch_mex.cu, exported through Matlabdef.def; its body is
 * a placeholder matrix addition, so this is the search it was meant to expose).
 *
 *   [idx, cost, params, costs] = cudaGridSearch_mex(fixed, moving, start, end, count, costName, opts)
 *
 *   fixed, moving : H x W or H x W x C real arrays, both double, single, uint8 or uint16,
 *                   C in {1, 3} (the moving image is sampled, the fixed one iterated, as the
 *                   reference functors' img_moved / img_fixed).
 *   start, end, count : grid of D <= 8 axes, as CudaGrid::setStartPoint / setEndPoint /
 *                   setNumSamples (src/gpu/cudaGridSearch.cuh:198-215), parameter order
 *                   [theta, sx, sy, shear, tx, ty, kx, ky] for the homography costs.
 *   costName      : a library cost (SAD_AVG, SAD_AVG_H, SAD_SUM_T, SAD_SUM_T_REF, SQD_REF,
 *                   NCC_REF, SQD_ALT, NCC_ALT, MI_ALT, ZNCC, MI) or the reference functor
 *                   name it reproduces (averageAbsoluteDifference, calcNCC, calcMIAlt, ...).
 *   opts          : optional [mi_bins, overlap_gate, sampling] (sampling 1 = exact, 0 = fast,
 *                   -1 = the cost's default).
 *   idx           : 1-based linear index of the lowest cost (lowest index among equals;
 *                   NaN / +inf never win) into the cost volume; 0 when no cost is finite.
 *   cost, params  : that cost and its grid point (1 x D).
 *   costs         : single array of size count(1) x ... x count(D): MATLAB's column-major
 *                   order is the reference's index order (axis 0 fastest).
 *
 * Errors are raised with mexErrMsgIdAndTxt after every device buffer is released (MATLAB
 * unwinds without running destructors).  The call blocks until the search is done.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "cugridsearch_b200.h"
#include "mex.h"

namespace {

struct CostName {
    const char *lib, *ref;
    int code;
};
const CostName kCosts[] = {
    {"SAD_AVG", "averageAbsoluteDifference", CGS_COST_SAD_AVG},
    {"SAD_AVG_H", "averageAbsoluteDifferenceH", CGS_COST_SAD_AVG_H},
    {"SAD_SUM_T", "sumOfAbsoluteDifferences", CGS_COST_SAD_SUM_T},
    {"SAD_SUM_T_REF", "sumOfAbsoluteDifferencesByReference", CGS_COST_SAD_SUM_T_REF},
    {"SQD_REF", "calcSQD", CGS_COST_SQD_REF},
    {"NCC_REF", "calcNCC", CGS_COST_NCC_REF},
    {"SQD_ALT", "calcSQDAlt", CGS_COST_SQD_ALT},
    {"NCC_ALT", "calcNCCAlt", CGS_COST_NCC_ALT},
    {"MI_ALT", "calcMIAlt", CGS_COST_MI_ALT},
    {"ZNCC", "calcZNCC", CGS_COST_ZNCC},
    {"MI", "calcMI", CGS_COST_MI},
};

struct Image {
    std::vector<unsigned char> hwc;  // host copy in CudaImage layout
    int h = 0, w = 0, c = 0, pixel = -1;
    size_t elem = 0;
};

// MATLAB's column-major H x W x C (element (y, x, c) at y + H x + H W c) to HWC row-major
// (c + C (x + W y)).
std::string read_image(const mxArray *a, const char *name, Image *im) {
    if (mxIsComplex(a)) return std::string(name) + " must be real";
    switch (mxGetClassID(a)) {
        case mxDOUBLE_CLASS: im->pixel = CGS_PIXEL_F64; im->elem = 8; break;
        case mxSINGLE_CLASS: im->pixel = CGS_PIXEL_F32; im->elem = 4; break;
        case mxUINT8_CLASS: im->pixel = CGS_PIXEL_U8; im->elem = 1; break;
        case mxUINT16_CLASS: im->pixel = CGS_PIXEL_U16; im->elem = 2; break;
        default: return std::string(name) + " must be double, single, uint8 or uint16";
    }
    const mwSize nd = mxGetNumberOfDimensions(a);
    const mwSize *d = mxGetDimensions(a);
    if (nd > 3) return std::string(name) + " must be H x W or H x W x C";
    im->h = (int)d[0];
    im->w = (int)d[1];
    im->c = nd == 3 ? (int)d[2] : 1;
    if (im->h < 1 || im->w < 1) return std::string(name) + " is empty";
    const size_t H = im->h, W = im->w, C = im->c, E = im->elem;
    const unsigned char *src = static_cast<const unsigned char *>(mxGetData(a));
    im->hwc.resize(H * W * C * E);
    for (size_t c = 0; c < C; c++)
        for (size_t x = 0; x < W; x++)
            for (size_t y = 0; y < H; y++)
                memcpy(&im->hwc[(c + C * (x + W * y)) * E], src + (y + H * x + H * W * c) * E, E);
    return "";
}

std::string read_vector(const mxArray *a, const char *name, std::vector<double> *v) {
    if (mxGetClassID(a) != mxDOUBLE_CLASS || mxIsComplex(a)) return std::string(name) + " must be a real double vector";
    const size_t n = mxGetNumberOfElements(a);
    const double *p = mxGetPr(a);
    v->assign(p, p + n);
    return "";
}

std::string status_message(cgs_status s, const char *what) {
    return std::string(what) + ": " + cgs_status_string(s) + " (" + cgs_last_error() + ")";
}

// The whole call; returns an error message, or "" with the outputs set.
std::string run(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    if (nrhs < 6 || nrhs > 7) return "usage: [idx, cost, params, costs] = cudaGridSearch_mex(fixed, moving, start, end, count, costName, opts)";
    if (nlhs > 4) return "at most four outputs: idx, cost, params, costs";
    Image fix, mov;
    std::string e;
    if (!(e = read_image(prhs[0], "fixed", &fix)).empty()) return e;
    if (!(e = read_image(prhs[1], "moving", &mov)).empty()) return e;
    if (fix.pixel != mov.pixel) return "fixed and moving must have the same class";
    if (fix.c != mov.c) return "fixed and moving must have the same number of channels";
    std::vector<double> start, end, count, opts;
    if (!(e = read_vector(prhs[2], "start", &start)).empty()) return e;
    if (!(e = read_vector(prhs[3], "end", &end)).empty()) return e;
    if (!(e = read_vector(prhs[4], "count", &count)).empty()) return e;
    const size_t D = start.size();
    if (D < 1 || D > 8 || end.size() != D || count.size() != D) return "start, end and count must have the same length, 1 to 8";
    if (!mxIsChar(prhs[5])) return "costName must be a string";
    char *cname = mxArrayToString(prhs[5]);
    int cost = -1;
    for (const CostName &k : kCosts)
        if (cname && (strcmp(cname, k.lib) == 0 || strcmp(cname, k.ref) == 0)) cost = k.code;
    const std::string cname_s = cname ? cname : "";
    mxFree(cname);
    if (cost < 0) return "unknown cost '" + cname_s + "'";
    if (nrhs == 7 && !(e = read_vector(prhs[6], "opts", &opts)).empty()) return e;

    cgs_grid g;
    memset(&g, 0, sizeof(g));
    g.dims = (int32_t)D;
    for (size_t a = 0; a < D; a++) {
        g.start[a] = (float)start[a];
        g.end[a] = (float)end[a];
        g.count[a] = (float)count[a];
    }
    cgs_status s = cgs_grid_update(&g, -1);
    if (s != CGS_SUCCESS) return status_message(s, "grid");
    uint64_t n = 0;
    if ((s = cgs_grid_num_elements(&g, &n)) != CGS_SUCCESS) return status_message(s, "grid");

    cgs_options o;
    memset(&o, 0, sizeof(o));
    o.cost = cost;
    if (opts.size() > 0) o.mi_bins = (int32_t)opts[0];
    if (opts.size() > 1) o.overlap_gate = (float)opts[1];
    if (opts.size() > 2 && opts[2] >= 0) o.flags = opts[2] > 0 ? CGS_FLAG_EXACT_SAMPLES : CGS_FLAG_FAST_SAMPLES;

    // device buffers: released on every path below before returning
    void *d_fix = nullptr, *d_mov = nullptr;
    float *d_costs = nullptr;
    cgs_argmin res;
    memset(&res, 0, sizeof(res));
    std::string err;
    cudaError_t ce = cudaMalloc(&d_fix, fix.hwc.size());
    if (ce == cudaSuccess) ce = cudaMalloc(&d_mov, mov.hwc.size());
    if (ce == cudaSuccess && nlhs >= 4 && n > 0) ce = cudaMalloc(&d_costs, n * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMemcpy(d_fix, fix.hwc.data(), fix.hwc.size(), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(d_mov, mov.hwc.data(), mov.hwc.size(), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) err = std::string("CUDA: ") + cudaGetErrorString(ce);
    if (err.empty()) {
        const cgs_image fi = {d_fix, fix.h, fix.w, fix.c, fix.pixel};
        const cgs_image mi = {d_mov, mov.h, mov.w, mov.c, mov.pixel};
        s = cgs_search_sync(&mi, &fi, &g, &o, d_costs, &res, nullptr);
        if (s != CGS_SUCCESS) err = status_message(s, "search");
    }
    std::vector<float> host_costs;
    if (err.empty() && d_costs) {
        host_costs.resize(n);
        ce = cudaMemcpy(host_costs.data(), d_costs, n * sizeof(float), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) err = std::string("CUDA: ") + cudaGetErrorString(ce);
    }
    cudaFree(d_fix);
    cudaFree(d_mov);
    cudaFree(d_costs);
    if (!err.empty()) return err;

    plhs[0] = mxCreateDoubleScalar(res.valid ? (double)res.index + 1.0 : 0.0);
    if (nlhs >= 2) plhs[1] = mxCreateDoubleScalar((double)res.cost);
    if (nlhs >= 3) {
        plhs[2] = mxCreateDoubleMatrix(1, D, mxREAL);
        double *p = mxGetPr(plhs[2]);
        for (size_t a = 0; a < D; a++) p[a] = (double)res.params[a];
    }
    if (nlhs >= 4) {
        // count(1) x ... x count(D); fractional counts (which the reference allows) give a
        // grid that is not such a box, and then the costs come back as an n x 1 column
        mwSize dims[8];
        mwSize nd = (mwSize)D;
        uint64_t prod = 1;
        for (size_t a = 0; a < D; a++) {
            dims[a] = (mwSize)g.count[a];
            prod *= (uint64_t)dims[a];
        }
        if (D == 1 || prod != n) {
            dims[0] = (mwSize)n;
            dims[1] = 1;
            nd = 2;
        }
        plhs[3] = mxCreateNumericArray(nd, dims, mxSINGLE_CLASS, mxREAL);
        if (n > 0) memcpy(mxGetData(plhs[3]), host_costs.data(), n * sizeof(float));
    }
    return "";
}

}  // namespace

extern "C" void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    const std::string err = run(nlhs, plhs, nrhs, prhs);
    if (!err.empty()) mexErrMsgIdAndTxt("cudaGridSearch:error", "%s", err.c_str());
}
