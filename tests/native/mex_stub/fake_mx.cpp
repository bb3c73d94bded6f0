// fake_mx.cpp -- an in-process stand-in for MATLAB's mxArray / MEX runtime (test
// infrastructure; MATLAB is not installed).  Arrays are column-major with MATLAB's
// dimension rules; mexErrMsgIdAndTxt throws, and fake_mex_call turns that into a returned
// message.  The extern "C" helpers at the end let the Python tests build arguments, call
// mexFunction and read the outputs.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mex.h"

struct mxArray_tag {
    mxClassID cls = mxUNKNOWN_CLASS;
    std::vector<mwSize> dims;
    std::vector<unsigned char> data;
    std::string text;  // mxCHAR_CLASS
};

namespace {

size_t elem_size(mxClassID c) {
    switch (c) {
        case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
        case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
        case mxINT16_CLASS: case mxUINT16_CLASS: return 2;
        case mxINT8_CLASS: case mxUINT8_CLASS: case mxLOGICAL_CLASS: return 1;
        default: return 0;
    }
}

mxArray *make(mxClassID c, mwSize nd, const mwSize *dims) {
    mxArray *a = new mxArray_tag;
    a->cls = c;
    a->dims.assign(dims, dims + nd);
    while (a->dims.size() > 2 && a->dims.back() == 1) a->dims.pop_back();  // trailing singletons
    if (a->dims.size() < 2) a->dims.resize(2, 1);
    size_t n = 1;
    for (mwSize d : a->dims) n *= d;
    a->data.assign(n * elem_size(c), 0);
    return a;
}

}  // namespace

extern "C" {

mxClassID mxGetClassID(const mxArray *pa) { return pa->cls; }
mwSize mxGetNumberOfDimensions(const mxArray *pa) { return pa->dims.size(); }
const mwSize *mxGetDimensions(const mxArray *pa) { return pa->dims.data(); }
size_t mxGetM(const mxArray *pa) { return pa->dims[0]; }
size_t mxGetN(const mxArray *pa) {
    size_t n = 1;
    for (size_t i = 1; i < pa->dims.size(); i++) n *= pa->dims[i];
    return n;
}
size_t mxGetNumberOfElements(const mxArray *pa) {
    size_t n = 1;
    for (mwSize d : pa->dims) n *= d;
    return n;
}
void *mxGetData(const mxArray *pa) { return const_cast<unsigned char *>(pa->data.data()); }
double *mxGetPr(const mxArray *pa) { return pa->cls == mxDOUBLE_CLASS ? (double *)mxGetData(pa) : nullptr; }
bool mxIsChar(const mxArray *pa) { return pa->cls == mxCHAR_CLASS; }
bool mxIsComplex(const mxArray *) { return false; }
char *mxArrayToString(const mxArray *pa) {
    if (pa->cls != mxCHAR_CLASS) return nullptr;
    char *s = (char *)malloc(pa->text.size() + 1);
    memcpy(s, pa->text.c_str(), pa->text.size() + 1);
    return s;
}
void mxFree(void *ptr) { free(ptr); }
mxArray *mxCreateDoubleScalar(double value) {
    const mwSize d[2] = {1, 1};
    mxArray *a = make(mxDOUBLE_CLASS, 2, d);
    memcpy(a->data.data(), &value, 8);
    return a;
}
mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity) {
    const mwSize d[2] = {m, n};
    return make(mxDOUBLE_CLASS, 2, d);
}
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity) {
    return make(classid, ndim, dims);
}

void mexErrMsgIdAndTxt(const char *errorid, const char *errormsg, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, errormsg);
    vsnprintf(buf, sizeof(buf), errormsg, ap);
    va_end(ap);
    throw std::runtime_error(std::string(errorid) + ": " + buf);
}

int mexPrintf(const char *message, ...) {
    va_list ap;
    va_start(ap, message);
    const int r = vprintf(message, ap);
    va_end(ap);
    return r;
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

// ---- test helpers
mxArray *fake_mx_numeric(int cls, int ndim, const uint64_t *dims, const void *data) {
    std::vector<mwSize> d(dims, dims + ndim);
    mxArray *a = make((mxClassID)cls, (mwSize)ndim, d.data());
    memcpy(a->data.data(), data, a->data.size());
    return a;
}
mxArray *fake_mx_string(const char *s) {
    mxArray *a = new mxArray_tag;
    a->cls = mxCHAR_CLASS;
    a->text = s;
    a->dims = {1, strlen(s)};
    return a;
}
void fake_mx_destroy(mxArray *a) { delete a; }
int fake_mx_class(const mxArray *a) { return (int)a->cls; }
int fake_mx_ndim(const mxArray *a) { return (int)a->dims.size(); }
uint64_t fake_mx_dim(const mxArray *a, int i) { return a->dims[i]; }
const void *fake_mx_data(const mxArray *a) { return a->data.data(); }

// Calls mexFunction; returns "" or the raised error (valid until the next call).
const char *fake_mex_call(int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs) {
    static std::string err;
    err.clear();
    for (int i = 0; i < nlhs; i++) plhs[i] = nullptr;
    try {
        mexFunction(nlhs, plhs, nrhs, prhs);
    } catch (const std::exception &e) {
        err = e.what();
    }
    return err.c_str();
}

}  // extern "C"
