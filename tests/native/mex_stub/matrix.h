/*
 * matrix.h -- a minimal stand-in for MATLAB's mxArray API (MATLAB is not installed here),
 * declaring only the functions the MEX entry uses, with the signatures of MathWorks'
 * published C Matrix API.  tests/native/mex_stub/fake_mx.cpp implements them for the tests.
 * A real build uses MATLAB's own extern/include instead of this directory.
 */
#ifndef CGS_FAKE_MATRIX_H
#define CGS_FAKE_MATRIX_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef ptrdiff_t mwSignedIndex;

typedef enum {
    mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
    mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
    mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS, mxFUNCTION_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;

mxClassID mxGetClassID(const mxArray *pa);
mwSize mxGetNumberOfDimensions(const mxArray *pa);
const mwSize *mxGetDimensions(const mxArray *pa);
size_t mxGetM(const mxArray *pa);
size_t mxGetN(const mxArray *pa);
size_t mxGetNumberOfElements(const mxArray *pa);
void *mxGetData(const mxArray *pa);
double *mxGetPr(const mxArray *pa);
bool mxIsChar(const mxArray *pa);
bool mxIsComplex(const mxArray *pa);
char *mxArrayToString(const mxArray *pa);
void mxFree(void *ptr);
mxArray *mxCreateDoubleScalar(double value);
mxArray *mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity flag);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag);

#ifdef __cplusplus
}
#endif
#endif
