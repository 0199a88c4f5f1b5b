/*
 * mexstub.c (test stub) - a minimal mxArray and MEX runtime for the shims
 * under mex/: numeric arrays (real or interleaved complex, up to 4-D),
 * 1 x 1 structs, mexCallMATLAB("randi") returning fixed draws, and
 * mexErrMsgIdAndTxt as a longjmp back to stub_run.  Test infrastructure only.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
    int ndim;
    size_t dims[4];
    int complex;
    double *data;
    int is_struct;
    int nfields;
    char names[4][32];
    mxArray *vals[4];
};

static jmp_buf g_jmp;
static char g_id[128], g_msg[512];
static int g_randi_calls;

static size_t numel(const mxArray *a)
{
    size_t n = 1;
    for (int k = 0; k < a->ndim; ++k) n *= a->dims[k];
    return a->is_struct ? 1 : n;
}

size_t mxGetM(const mxArray *a) { return a->dims[0]; }
size_t mxGetN(const mxArray *a)
{
    size_t n = 1;
    for (int k = 1; k < a->ndim; ++k) n *= a->dims[k];
    return n;
}
size_t mxGetNumberOfElements(const mxArray *a) { return numel(a); }
double *mxGetDoubles(const mxArray *a) { return a->complex ? NULL : a->data; }
mxComplexDouble *mxGetComplexDoubles(const mxArray *a) { return a->complex ? (mxComplexDouble *)a->data : NULL; }
int mxIsComplex(const mxArray *a) { return a->complex; }
int mxIsStruct(const mxArray *a) { return a->is_struct; }
int mxIsEmpty(const mxArray *a) { return !a->is_struct && numel(a) == 0; }
double mxGetScalar(const mxArray *a) { return numel(a) ? a->data[0] : 0.0; }

mxArray *mxGetField(const mxArray *a, size_t index, const char *name)
{
    (void)index;
    for (int i = 0; i < a->nfields; ++i)
        if (!strcmp(a->names[i], name)) return a->vals[i];
    return NULL;
}

mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID c, mxComplexity x)
{
    (void)c;
    mxArray *a = calloc(1, sizeof *a);
    a->ndim = (int)(ndim < 2 ? 2 : ndim);
    a->dims[0] = a->dims[1] = 1;
    for (mwSize k = 0; k < ndim; ++k) a->dims[k] = dims[k];
    a->complex = x == mxCOMPLEX;
    a->data = calloc(numel(a) * (a->complex ? 2 : 1) + 1, sizeof(double));
    return a;
}

mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x)
{
    mwSize d[2] = {m, n};
    return mxCreateNumericArray(2, d, c, x);
}

mxArray *mxCreateDoubleScalar(double v)
{
    mxArray *a = mxCreateNumericMatrix(1, 1, mxDOUBLE_CLASS, mxREAL);
    a->data[0] = v;
    return a;
}

void mxDestroyArray(mxArray *a)
{
    if (!a) return;
    for (int i = 0; i < a->nfields; ++i) mxDestroyArray(a->vals[i]);
    free(a->data);
    free(a);
}

int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[], const char *name)
{
    (void)nrhs;
    (void)prhs;
    if (strcmp(name, "randi") || nlhs != 1) return 1;
    plhs[0] = mxCreateNumericMatrix(1, 2, mxDOUBLE_CLASS, mxREAL);
    plhs[0]->data[0] = 123456789.0 + g_randi_calls;
    plhs[0]->data[1] = 987654321.0;
    ++g_randi_calls;
    return 0;
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
    snprintf(g_id, sizeof g_id, "%s", id);
    longjmp(g_jmp, 1);
}

/* ---- harness entry points (called from Python through ctypes) ---- */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

int stub_run(int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs)
{
    g_id[0] = g_msg[0] = 0;
    if (setjmp(g_jmp)) return 1;
    mexFunction(nlhs, plhs, nrhs, prhs);
    return 0;
}

const char *stub_err_id(void) { return g_id; }
const char *stub_err_msg(void) { return g_msg; }

/* m x n double, im may be NULL (real) */
mxArray *stub_double(size_t m, size_t n, const double *re, const double *im)
{
    mxArray *a = mxCreateNumericMatrix(m, n, mxDOUBLE_CLASS, im ? mxCOMPLEX : mxREAL);
    for (size_t k = 0; k < m * n; ++k) {
        if (im) {
            a->data[2 * k] = re[k];
            a->data[2 * k + 1] = im[k];
        } else {
            a->data[k] = re[k];
        }
    }
    return a;
}

/* a 1 x 1 struct with two fields (takes ownership of the values) */
mxArray *stub_struct2(const char *f1, mxArray *v1, const char *f2, mxArray *v2)
{
    mxArray *a = calloc(1, sizeof *a);
    a->ndim = 2;
    a->dims[0] = a->dims[1] = 1;
    a->is_struct = 1;
    a->nfields = 2;
    snprintf(a->names[0], 32, "%s", f1);
    snprintf(a->names[1], 32, "%s", f2);
    a->vals[0] = v1;
    a->vals[1] = v2;
    return a;
}

int stub_ndim(const mxArray *a) { return a->ndim; }
size_t stub_dim(const mxArray *a, int k) { return a->dims[k]; }
int stub_is_complex(const mxArray *a) { return a->complex; }
double *stub_data(const mxArray *a) { return a->data; }
