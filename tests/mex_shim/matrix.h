/* matrix.h -- a small stand-in for MATLAB's mxArray API, written for the
 * tests of the MEX gateway (opticrcwafdtd_b200/matlab/orf_fdtd_mex.c) on hosts
 * without MATLAB.  It implements only the calls the gateway makes, with the
 * documented meaning of the interleaved-complex (-R2018a) API, over plain C
 * arrays.  Not MathWorks code; test infrastructure only. */
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef bool mxLogical;
typedef struct mxArray_tag mxArray;
typedef struct { double real, imag; } mxComplexDouble;
typedef enum { mxUNKNOWN_CLASS = 0, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxDOUBLE_CLASS,
               mxFUNCTION_CLASS, mxOBJECT_CLASS } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

void* mxMalloc(size_t n);
mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name);
void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* v);
void mxSetFieldByNumber(mxArray* s, mwIndex i, int f, mxArray* v);
bool mxIsEmpty(const mxArray* a);
bool mxIsNumeric(const mxArray* a);
bool mxIsLogical(const mxArray* a);
bool mxIsDouble(const mxArray* a);
bool mxIsComplex(const mxArray* a);
bool mxIsChar(const mxArray* a);
bool mxIsStruct(const mxArray* a);
bool mxIsClass(const mxArray* a, const char* name);
size_t mxGetNumberOfElements(const mxArray* a);
double mxGetScalar(const mxArray* a);
double* mxGetDoubles(const mxArray* a);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
mxLogical* mxGetLogicals(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize n);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateLogicalScalar(bool v);
mxArray* mxCreateString(const char* s);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID cls, mxComplexity c);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
mxArray* mxDuplicateArray(const mxArray* a);
void mxDestroyArray(mxArray* a);

#ifdef __cplusplus
}
#endif
