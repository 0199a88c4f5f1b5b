/*
 * mex.h (test stub) - the subset of MATLAB's MEX API (R2018a interleaved
 * complex) that the shims under mex/ use, so they compile and run on a
 * machine without MATLAB.  Test infrastructure only; mexstub.c implements it.
 */
#ifndef SCMC_TEST_MEX_STUB_H
#define SCMC_TEST_MEX_STUB_H
#include <stddef.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum { mxDOUBLE_CLASS = 6 } mxClassID;
typedef struct {
    double real, imag;
} mxComplexDouble;

size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
double *mxGetDoubles(const mxArray *a);
mxComplexDouble *mxGetComplexDoubles(const mxArray *a);
int mxIsComplex(const mxArray *a);
int mxIsStruct(const mxArray *a);
int mxIsEmpty(const mxArray *a);
mxArray *mxGetField(const mxArray *a, size_t index, const char *name);
double mxGetScalar(const mxArray *a);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID c, mxComplexity x);
mxArray *mxCreateDoubleScalar(double v);
void mxDestroyArray(mxArray *a);
int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[], const char *name);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);

#endif
