/*
 * mex.h -- minimal stand-in for the MATLAB MEX API, enough to compile and exercise MEX
 * gateway sources without MATLAB.  Arrays are plain structs; gpuArrays hold device
 * pointers.  mexErrMsgIdAndTxt throws (the caller of mexFunction catches).
 * When MATLAB is present, gateways are built against MATLAB's own headers instead.
 */
#ifndef EMC_MEX_SHIM_MEX_H
#define EMC_MEX_SHIM_MEX_H
#include <stddef.h>
#include <stdint.h>

#include "matrix.h"

#ifdef __cplusplus
extern "C" {
#endif
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexPrintf(const char* fmt, ...);
void mexMakeArrayPersistent(mxArray* a);
#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
extern "C"
#endif
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

#endif
