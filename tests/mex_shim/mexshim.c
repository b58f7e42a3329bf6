/* mexshim.c -- implementation of the matrix.h / mex.h stand-in used to test the
 * MEX gateway without MATLAB, plus a small control API (shim_*) through which
 * the Python tests build sim structs, call mexFunction and read the results.
 * Arrays are column-major; complex doubles are interleaved (re, im).
 * Test infrastructure only. */
#define _POSIX_C_SOURCE 200809L
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
    mxClassID cls;
    int complex_;
    size_t nd;
    size_t dims[8];
    size_t numel;
    void* data;            /* double / mxComplexDouble / mxLogical / char string */
    int nfields;           /* struct: field names and numel * nfields values */
    char** names;
    mxArray** values;
    int (*fn)(double, const char*);   /* function handle: returns non-zero to throw */
    char* exc_id;          /* MException: identifier and message */
    char* exc_msg;
};

static jmp_buf g_jmp;
static int g_in_call = 0;
static char g_err_id[256], g_err_msg[4096], g_warn_id[256], g_warn_msg[4096];

static mxArray* alloc_arr(mxClassID c, size_t nd, const size_t* dims) {
    mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
    a->cls = c;
    a->nd = nd < 2 ? 2 : nd;
    a->dims[0] = a->dims[1] = 1;
    a->numel = 1;
    for (size_t k = 0; k < nd; ++k) {
        a->dims[k] = dims[k];
        a->numel *= dims[k];
    }
    if (nd == 0) a->numel = 1;
    return a;
}

void* mxMalloc(size_t n) { return calloc(1, n ? n : 1); }

static int field_index(const mxArray* s, const char* name) {
    for (int f = 0; f < s->nfields; ++f)
        if (!strcmp(s->names[f], name)) return f;
    return -1;
}

mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name) {
    if (!s || s->cls != mxSTRUCT_CLASS || i >= s->numel) return NULL;
    const int f = field_index(s, name);
    return f < 0 ? NULL : s->values[i * (size_t)s->nfields + (size_t)f];
}

static void add_field(mxArray* s, const char* name) {
    const int nf = s->nfields + 1;
    char** names = (char**)calloc((size_t)nf, sizeof(char*));
    mxArray** vals = (mxArray**)calloc(s->numel * (size_t)nf, sizeof(mxArray*));
    for (int f = 0; f < s->nfields; ++f) names[f] = s->names[f];
    names[nf - 1] = strdup(name);
    for (size_t i = 0; i < s->numel; ++i)
        for (int f = 0; f < s->nfields; ++f) vals[i * (size_t)nf + (size_t)f] = s->values[i * (size_t)s->nfields + (size_t)f];
    free(s->names);
    free(s->values);
    s->names = names;
    s->values = vals;
    s->nfields = nf;
}

void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* v) {
    int f = field_index(s, name);
    if (f < 0) {
        add_field(s, name);
        f = s->nfields - 1;
    }
    s->values[i * (size_t)s->nfields + (size_t)f] = v;
}

void mxSetFieldByNumber(mxArray* s, mwIndex i, int f, mxArray* v) { s->values[i * (size_t)s->nfields + (size_t)f] = v; }
bool mxIsEmpty(const mxArray* a) { return a->numel == 0; }
bool mxIsNumeric(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsLogical(const mxArray* a) { return a->cls == mxLOGICAL_CLASS; }
bool mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsComplex(const mxArray* a) { return a->complex_ != 0; }
bool mxIsChar(const mxArray* a) { return a->cls == mxCHAR_CLASS; }
bool mxIsStruct(const mxArray* a) { return a->cls == mxSTRUCT_CLASS; }
bool mxIsClass(const mxArray* a, const char* name) {
    if (!strcmp(name, "function_handle")) return a->cls == mxFUNCTION_CLASS;
    if (!strcmp(name, "double")) return a->cls == mxDOUBLE_CLASS;
    if (!strcmp(name, "MException")) return a->cls == mxOBJECT_CLASS;
    return false;
}
size_t mxGetNumberOfElements(const mxArray* a) { return a->numel; }
double mxGetScalar(const mxArray* a) {
    if (a->numel == 0) return 0.0;
    if (a->cls == mxDOUBLE_CLASS) return a->complex_ ? ((mxComplexDouble*)a->data)[0].real : ((double*)a->data)[0];
    if (a->cls == mxLOGICAL_CLASS) return ((mxLogical*)a->data)[0] ? 1.0 : 0.0;
    return 0.0;
}
double* mxGetDoubles(const mxArray* a) { return (a->cls == mxDOUBLE_CLASS && !a->complex_) ? (double*)a->data : NULL; }
mxComplexDouble* mxGetComplexDoubles(const mxArray* a) {
    return (a->cls == mxDOUBLE_CLASS && a->complex_) ? (mxComplexDouble*)a->data : NULL;
}
mxLogical* mxGetLogicals(const mxArray* a) { return a->cls == mxLOGICAL_CLASS ? (mxLogical*)a->data : NULL; }

int mxGetString(const mxArray* a, char* buf, mwSize n) {
    if (a->cls != mxCHAR_CLASS || n == 0) return 1;
    const char* s = (const char*)a->data;
    const size_t len = strlen(s);
    snprintf(buf, n, "%s", s);
    return len + 1 > n ? 1 : 0;
}

mxArray* mxCreateDoubleScalar(double v) {
    mxArray* a = alloc_arr(mxDOUBLE_CLASS, 0, NULL);
    a->data = calloc(1, sizeof(double));
    ((double*)a->data)[0] = v;
    return a;
}

mxArray* mxCreateLogicalScalar(bool v) {
    mxArray* a = alloc_arr(mxLOGICAL_CLASS, 0, NULL);
    a->data = calloc(1, sizeof(mxLogical));
    ((mxLogical*)a->data)[0] = v;
    return a;
}

mxArray* mxCreateString(const char* s) {
    const size_t d[2] = {1, strlen(s)};
    mxArray* a = alloc_arr(mxCHAR_CLASS, 2, d);
    a->data = strdup(s);
    return a;
}

mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID cls, mxComplexity c) {
    mxArray* a = alloc_arr(cls, nd, dims);
    a->complex_ = c == mxCOMPLEX;
    a->data = calloc(a->numel ? a->numel : 1, a->complex_ ? sizeof(mxComplexDouble) : sizeof(double));
    return a;
}

mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
    const mwSize d[2] = {m, n};
    return mxCreateNumericArray(2, d, mxDOUBLE_CLASS, c);
}

mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names) {
    const size_t d[2] = {m, n};
    mxArray* a = alloc_arr(mxSTRUCT_CLASS, 2, d);
    a->nfields = nfields;
    a->names = (char**)calloc((size_t)(nfields ? nfields : 1), sizeof(char*));
    for (int f = 0; f < nfields; ++f) a->names[f] = strdup(names[f]);
    a->values = (mxArray**)calloc(a->numel * (size_t)(nfields ? nfields : 1), sizeof(mxArray*));
    return a;
}

mxArray* mxDuplicateArray(const mxArray* a) {
    mxArray* r = (mxArray*)calloc(1, sizeof(mxArray));
    *r = *a;
    if (a->cls == mxDOUBLE_CLASS) {
        const size_t b = (a->numel ? a->numel : 1) * (a->complex_ ? sizeof(mxComplexDouble) : sizeof(double));
        r->data = malloc(b);
        memcpy(r->data, a->data, b);
    } else if (a->cls == mxLOGICAL_CLASS) {
        r->data = malloc(a->numel * sizeof(mxLogical) + 1);
        memcpy(r->data, a->data, a->numel * sizeof(mxLogical));
    } else if (a->cls == mxCHAR_CLASS) {
        r->data = strdup((const char*)a->data);
    } else if (a->cls == mxSTRUCT_CLASS) {
        r->names = (char**)calloc((size_t)(a->nfields ? a->nfields : 1), sizeof(char*));
        for (int f = 0; f < a->nfields; ++f) r->names[f] = strdup(a->names[f]);
        r->values = (mxArray**)calloc(a->numel * (size_t)(a->nfields ? a->nfields : 1), sizeof(mxArray*));
        for (size_t i = 0; i < a->numel * (size_t)a->nfields; ++i)
            r->values[i] = a->values[i] ? mxDuplicateArray(a->values[i]) : NULL;
    }
    return r;
}

void mxDestroyArray(mxArray* a) {
    if (!a) return;
    if (a->cls == mxSTRUCT_CLASS) {
        for (size_t i = 0; i < a->numel * (size_t)a->nfields; ++i) mxDestroyArray(a->values[i]);
        for (int f = 0; f < a->nfields; ++f) free(a->names[f]);
        free(a->names);
        free(a->values);
    }
    free(a->data);
    free(a->exc_id);
    free(a->exc_msg);
    free(a);
}

/* ------------------------------------------------------------- mex* ---- */
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
    snprintf(g_err_id, sizeof g_err_id, "%s", id);
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err_msg, sizeof g_err_msg, fmt, ap);
    va_end(ap);
    if (g_in_call) longjmp(g_jmp, 1);
    fprintf(stderr, "mexErrMsgIdAndTxt outside shim_call: %s: %s\n", g_err_id, g_err_msg);
    abort();
}

void mexWarnMsgIdAndTxt(const char* id, const char* fmt, ...) {
    snprintf(g_warn_id, sizeof g_warn_id, "%s", id);
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_warn_msg, sizeof g_warn_msg, fmt, ap);
    va_end(ap);
}

/* feval of a function handle: its C callback returns non-zero to throw
 * orf:cancelled.  rethrow(MException) raises that exception's error. */
mxArray* mexCallMATLABWithTrap(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* fn) {
    (void)nlhs;
    (void)plhs;
    if (!strcmp(fn, "feval") && nrhs >= 1 && prhs[0]->cls == mxFUNCTION_CLASS) {
        const double frac = nrhs > 1 ? mxGetScalar(prhs[1]) : 0.0;
        const char* msg = nrhs > 2 && prhs[2]->cls == mxCHAR_CLASS ? (const char*)prhs[2]->data : "";
        if (prhs[0]->fn(frac, msg) == 0) return NULL;
        mxArray* e = alloc_arr(mxOBJECT_CLASS, 0, NULL);
        e->exc_id = strdup("orf:cancelled");
        e->exc_msg = strdup("Cancelled by the user.");
        return e;
    }
    mxArray* e = alloc_arr(mxOBJECT_CLASS, 0, NULL);
    e->exc_id = strdup("shim:unsupported");
    e->exc_msg = strdup(fn);
    return e;
}

int mexCallMATLAB(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* fn) {
    (void)nlhs;
    (void)plhs;
    if (!strcmp(fn, "rethrow") && nrhs == 1 && prhs[0]->cls == mxOBJECT_CLASS)
        mexErrMsgIdAndTxt(prhs[0]->exc_id, "%s", prhs[0]->exc_msg);
    mexErrMsgIdAndTxt("shim:unsupported", "mexCallMATLAB(%s)", fn);
}

/* ------------------------------------------------------ control API ---- */
mxArray* shim_double(size_t nd, const size_t* dims, const double* data, int complex_) {
    mxArray* a = mxCreateNumericArray(nd, dims, mxDOUBLE_CLASS, complex_ ? mxCOMPLEX : mxREAL);
    if (data && a->numel) memcpy(a->data, data, a->numel * (complex_ ? 16 : 8));
    return a;
}
mxArray* shim_logical(int v) { return mxCreateLogicalScalar(v != 0); }
mxArray* shim_string(const char* s) { return mxCreateString(s); }
mxArray* shim_struct(size_t n) { return mxCreateStructMatrix(1, n, 0, NULL); }
void shim_set(mxArray* s, size_t i, const char* name, mxArray* v) { mxSetField(s, i, name, v); }
mxArray* shim_handle(int (*fn)(double, const char*)) {
    mxArray* a = alloc_arr(mxFUNCTION_CLASS, 0, NULL);
    a->fn = fn;
    return a;
}

int shim_call(int nlhs, mxArray** plhs, int nrhs, mxArray** prhs) {
    g_err_id[0] = g_err_msg[0] = g_warn_id[0] = g_warn_msg[0] = 0;
    g_in_call = 1;
    if (setjmp(g_jmp)) {
        g_in_call = 0;
        return 1;
    }
    mexFunction(nlhs, plhs, nrhs, (const mxArray**)prhs);
    g_in_call = 0;
    return 0;
}

const char* shim_error_id(void) { return g_err_id; }
const char* shim_error_msg(void) { return g_err_msg; }
const char* shim_warning_id(void) { return g_warn_id; }
mxArray* shim_get(const mxArray* s, size_t i, const char* name) { return mxGetField(s, i, name); }
int shim_nfields(const mxArray* s) { return s->cls == mxSTRUCT_CLASS ? s->nfields : -1; }
const char* shim_field_name(const mxArray* s, int f) { return s->names[f]; }
int shim_class(const mxArray* a) { return (int)a->cls; }
int shim_is_complex(const mxArray* a) { return a->complex_; }
size_t shim_numel(const mxArray* a) { return a->numel; }
size_t shim_ndims(const mxArray* a) { return a->nd; }
size_t shim_dim(const mxArray* a, size_t k) { return k < a->nd ? a->dims[k] : 1; }
const void* shim_data(const mxArray* a) { return a->data; }
void shim_free(mxArray* a) { mxDestroyArray(a); }
mxArray* shim_logicals(size_t n, const unsigned char* v) {
    const size_t d[2] = {1, n};
    mxArray* a = alloc_arr(mxLOGICAL_CLASS, 2, d);
    a->data = calloc(n ? n : 1, sizeof(mxLogical));
    for (size_t i = 0; i < n; ++i) ((mxLogical*)a->data)[i] = v[i] != 0;
    return a;
}
