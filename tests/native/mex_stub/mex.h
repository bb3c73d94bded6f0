/*
 * mex.h -- a minimal stand-in for MATLAB's MEX API (see matrix.h in this directory).
 * mexErrMsgIdAndTxt does not return: the fake raises a C++ exception the test driver
 * catches, as MATLAB unwinds to its prompt.
 */
#ifndef CGS_FAKE_MEX_H
#define CGS_FAKE_MEX_H
#include "matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

void mexErrMsgIdAndTxt(const char *errorid, const char *errormsg, ...);
int mexPrintf(const char *message, ...);

#ifdef __cplusplus
}
#endif
#endif
