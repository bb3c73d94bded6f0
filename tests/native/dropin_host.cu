// dropin_host.cu -- the drop-in functor bodies (include/cugridsearch/) called on the host,
// exported for the CPU tests, which compare them with the reference's own functors
// (oracle/_ref) and the oracle.  Same calling convention as the reference harness's
// cgsref_eval: images zero-padded past their end, pix 0 = float, 1 = uint8_t,
// 2 = double, 3 = uint16_t; channels 1 or 3.
#include "cugridsearch/cudaGridSearch.cuh"

namespace {

enum {
    SAD_AVG = 0, SAD_AVG_H = 1, SAD_SUM_T = 2, SAD_SUM_T_REF = 3, SQD_REF = 4, NCC_REF = 5, SQD_ALT = 6,
    NCC_ALT = 7, MI_ALT = 8, ZNCC = 9, MI = 10,
    // block-cooperative functors of the reference, single-thread here
    SAD_STREAM = 100, NCC_STREAM = 101, NCC_STREAM_ALT = 102, SQD_STREAM = 103, MI_STREAM = 104,
    MI_STREAM_ALT = 105
};

template <typename P, uint32_t C>
float eval_c(int cost, const float *params, const void *mov, int mh, int mw, const void *fix, int fh, int fw) {
    CudaImage<P, C> M(mh, mw), F(fh, fw);
    M.data() = (P *)mov;
    F.data() = (P *)fix;
    nv_ext::Vec<float, 8> v(params);
    switch (cost) {
        case SAD_AVG: return averageAbsoluteDifference<float, float, 8, C, P>(v, M, F);
        case SQD_REF: return calcSQD<float, float, 8, C, P>(v, M, F);
        case NCC_REF: return calcNCC<float, float, 8, C, P>(v, M, F);
        case SQD_ALT: return calcSQDAlt<float, float, 8, C, P>(v, M, F);
        case NCC_ALT: return calcNCCAlt<float, float, 8, C, P>(v, M, F);
        case MI_ALT: return calcMIAlt<float, float, 8, C, P>(v, M, F);
        case ZNCC: return calcZNCC<float, float, 8, C, P>(v, M, F);
        case MI: return calcMI<float, float, 8, C, P>(v, M, F);
        case SAD_STREAM: return averageAbsoluteDifference_stream<float, float, 8, C, P>(v, M, F);
        case NCC_STREAM: return calcNCCstream<float, float, 8, C, P>(v, M, F);
        case NCC_STREAM_ALT: return calcNCCstreamAlt<float, float, 8, C, P>(v, M, F);
        case SQD_STREAM: return calcSQDstream<float, float, 8, C, P>(v, M, F);
        case MI_STREAM: return calcMIstream<float, float, 8, C, P>(v, M, F);
        case MI_STREAM_ALT: return calcMIstreamAlt<float, float, 8, C, P>(v, M, F);
        default: break;
    }
    if (C == 1) {
        CudaImage<P> M1(mh, mw), F1(fh, fw);
        M1.data() = (P *)mov;
        F1.data() = (P *)fix;
        switch (cost) {
            case SAD_AVG_H: return averageAbsoluteDifferenceH<float, float, 8, 1, P>(v, M1, F1);
            case SAD_SUM_T: return sumOfAbsoluteDifferences<float, float, 8, 1, P>(v, M1, F1);
            case SAD_SUM_T_REF: return sumOfAbsoluteDifferences<float, float, 8, 1, P>(v, &M1, &F1);
            default: break;
        }
    }
    return NAN;
}

template <typename P>
float eval_p(int cost, const float *params, const void *mov, int mh, int mw, const void *fix, int fh, int fw, int c) {
    if (c == 1) return eval_c<P, 1>(cost, params, mov, mh, mw, fix, fh, fw);
    if (c == 3) return eval_c<P, 3>(cost, params, mov, mh, mw, fix, fh, fw);
    return NAN;
}

}  // namespace

extern "C" float dropin_eval(int cost, const float *params, int pix, const void *mov, int mh, int mw, const void *fix,
                             int fh, int fw, int channels) {
    switch (pix) {
        case 1: return eval_p<uint8_t>(cost, params, mov, mh, mw, fix, fh, fw, channels);
        case 2: return eval_p<double>(cost, params, mov, mh, mw, fix, fh, fw, channels);
        case 3: return eval_p<uint16_t>(cost, params, mov, mh, mw, fix, fh, fw, channels);
        default: return eval_p<float>(cost, params, mov, mh, mw, fix, fh, fw, channels);
    }
}

// The drop-in homography helper, for a direct comparison with the reference's.
extern "C" void dropin_params_to_h(const float *params, float cx, float cy, float *h) {
    nv_ext::Vec<float, 8> v(params);
    parametersToHomography<float, 8>(v, cx, cy, h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7]);
}
