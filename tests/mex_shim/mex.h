/* mex.h -- the mex* calls of the MEX gateway, for its tests without MATLAB
 * (see matrix.h).  mexErrMsgIdAndTxt leaves the gateway through longjmp back
 * to shim_call, as MATLAB leaves a MEX function on an error. */
#pragma once
#include "matrix.h"

#ifdef __cplusplus
extern "C" {
#endif
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) __attribute__((noreturn));
void mexWarnMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexCallMATLAB(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* fn);
mxArray* mexCallMATLABWithTrap(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* fn);
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
#ifdef __cplusplus
}
#endif
