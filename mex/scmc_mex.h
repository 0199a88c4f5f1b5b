/*
 * scmc_mex.h - argument conversion shared by the MEX shims MCfield_mex.c,
 * MCcov_mex.c and MCfieldFourierQuad_mex.c.
 *
 * Built with `mex -R2018a` (interleaved complex: the library's layout).  The
 * shims take MATLAB's positional arguments exactly as the reference's .m
 * files do, apply the same checks with the same messages (MCfield.m:41-66,
 * MCcov.m:45-70), convert 1 x N angle rows of 2-D problems to [sin; cos],
 * draw the Philox key from MATLAB's global stream (so rng(seed) in
 * scmc.m:405-407 still fixes the result and parfor workers differ) and call
 * the C ABI of include/scmc_gpu.h.  GPU controls with no MATLAB slot come
 * from the environment: SCMC_PRECISION (fp64 | mixed | fp16 | fp32, default
 * mixed) and SCMC_DEVICE (default 0).
 */
#ifndef SCMC_MEX_H
#define SCMC_MEX_H

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "scmc_gpu.h"

/* Buffers a call allocates (converted direction rows, promoted tables);
 * freed by scmc_mex_release before the shim returns or raises. */
typedef struct {
    double *owned[8];
    int n;
} scmc_mex_scratch;

static void scmc_mex_release(scmc_mex_scratch *s)
{
    for (int i = 0; i < s->n; ++i) free(s->owned[i]);
    s->n = 0;
}

static double *scmc_mex_alloc(scmc_mex_scratch *s, size_t n)
{
    double *p = (double *)calloc(n ? n : 1, sizeof(double));
    if (!p || s->n >= 8) {
        free(p);
        scmc_mex_release(s);
        mexErrMsgIdAndTxt("scmc:gpu:nomem", "host allocation failed");
    }
    s->owned[s->n++] = p;
    return p;
}

static void scmc_mex_fail(scmc_mex_scratch *s, const char *id, const char *msg)
{
    scmc_mex_release(s);
    mexErrMsgIdAndTxt(id, "%s", msg);
}

/* narginchk(lo, hi) with MATLAB's messages. */
static void scmc_mex_nargin(int nrhs, int lo, int hi)
{
    if (nrhs < lo) mexErrMsgIdAndTxt("MATLAB:narginchk:notEnoughInputs", "Not enough input arguments.");
    if (nrhs > hi) mexErrMsgIdAndTxt("MATLAB:narginchk:tooManyInputs", "Too many input arguments.");
}

/* MCfield.m:44-49 / MCcov.m:48-53: box_min, box_max dim x 1 with dim 2 or 3. */
static int scmc_mex_box(const mxArray *bmin, const mxArray *bmax, double *lo, double *hi, scmc_mex_scratch *s)
{
    const size_t nb = mxGetNumberOfElements(bmax);
    if ((nb != 2 && nb != 3) || mxGetN(bmax) != 1 || mxGetM(bmax) != mxGetM(bmin) || mxGetN(bmin) != 1)
        scmc_mex_fail(s, "scmc:gpu:box", "Invalid box size");
    const int dim = (int)mxGetM(bmin);
    memcpy(lo, mxGetDoubles(bmin), (size_t)dim * sizeof(double));
    memcpy(hi, mxGetDoubles(bmax), (size_t)dim * sizeof(double));
    return dim;
}

/* MCfield.m:52-66: sources as dim x N; for dim 2 a 1 x N row of angles is
 * [sin(l); cos(l)]. */
static const double *scmc_mex_sources(const mxArray *x, int dim, const char *what, int64_t *n,
                                      scmc_mex_scratch *s)
{
    const size_t m = mxGetM(x), cols = mxGetN(x);
    if (m == (size_t)dim) {
        *n = (int64_t)cols;
        return mxGetDoubles(x);
    }
    if (dim == 2 && m == 1) {
        const double *a = mxGetDoubles(x);
        double *d = scmc_mex_alloc(s, 2 * cols);
        for (size_t j = 0; j < cols; ++j) {
            d[2 * j] = sin(a[j]);
            d[2 * j + 1] = cos(a[j]);
        }
        *n = (int64_t)cols;
        return d;
    }
    scmc_mex_fail(s, "scmc:gpu:source", what);
    return NULL;
}

/* (sct_type, ampfunc) of MCfield.m:1: 0 for isotropic, g for HG, the
 * tabulatedAmplitudeScatter struct (tabulatedAmplitudeScatter.m:75-99) for
 * tabulated.  A real-valued evalAmp (MATLAB drops all-zero imaginary parts)
 * is promoted to interleaved complex. */
static void scmc_mex_phase_fn(const mxArray *sct, const mxArray *amp, scmc_phase_function *pf, scmc_mex_scratch *s)
{
    memset(pf, 0, sizeof *pf);
    pf->sct_type = (int32_t)mxGetScalar(sct);
    if (pf->sct_type == SCMC_SCT_HG) pf->g = mxGetScalar(amp);
    if (pf->sct_type == SCMC_SCT_TABULATED) {
        const mxArray *ea = mxIsStruct(amp) ? mxGetField(amp, 0, "evalAmp") : NULL;
        const mxArray *ic = mxIsStruct(amp) ? mxGetField(amp, 0, "sampleIcdf") : NULL;
        if (!ea || !ic) scmc_mex_fail(s, "scmc:gpu:ampfunc", "tabulated ampfunc needs evalAmp and sampleIcdf");
        const size_t n = mxGetNumberOfElements(ic);
        if (mxGetNumberOfElements(ea) != n) scmc_mex_fail(s, "scmc:gpu:ampfunc", "evalAmp and sampleIcdf differ in length");
        pf->table_n = (int32_t)n;
        pf->sample_icdf = mxGetDoubles(ic);
        if (mxIsComplex(ea)) {
            pf->eval_amp = (const double *)mxGetComplexDoubles(ea);
        } else {
            const double *re = mxGetDoubles(ea);
            double *d = scmc_mex_alloc(s, 2 * n);
            for (size_t i = 0; i < n; ++i) d[2 * i] = re[i];
            pf->eval_amp = d;
        }
    }
}

/* The Philox key from MATLAB's global stream: two draws of randi. */
static uint64_t scmc_mex_seed(void)
{
    mxArray *key = NULL;
    mxArray *rin[3] = {mxCreateDoubleScalar(2147483646.0), mxCreateDoubleScalar(1.0), mxCreateDoubleScalar(2.0)};
    mexCallMATLAB(1, &key, 3, rin, "randi");
    const double *k = mxGetDoubles(key);
    const uint64_t seed = ((uint64_t)k[0] << 31) ^ (uint64_t)k[1];
    mxDestroyArray(key);
    for (int i = 0; i < 3; ++i) mxDestroyArray(rin[i]);
    return seed;
}

static int32_t scmc_mex_precision(void)
{
    const char *p = getenv("SCMC_PRECISION");
    if (!p || !strcmp(p, "mixed")) return SCMC_PREC_MIXED;
    if (!strcmp(p, "fp64")) return SCMC_PREC_FP64;
    if (!strcmp(p, "fp16")) return SCMC_PREC_FP16;
    if (!strcmp(p, "fp32")) return SCMC_PREC_FP32;
    return SCMC_PREC_MIXED;
}

static int32_t scmc_mex_device(void)
{
    const char *d = getenv("SCMC_DEVICE");
    return d ? (int32_t)atoi(d) : 0;
}

/* The 14 positional arguments shared by MCfield and MCcov (plus ampfunc0 as
 * the 15th and lmean0 as the 16th where given). */
static void scmc_mex_mc_args(int nrhs, const mxArray *prhs[], scmc_mc_args *a, scmc_mex_scratch *s)
{
    memset(a, 0, sizeof *a);
    a->dim = scmc_mex_box(prhs[2], prhs[3], a->box_min, a->box_max, s);
    a->sigt = mxGetScalar(prhs[0]);
    a->albedo = mxGetScalar(prhs[1]);
    a->l = scmc_mex_sources(prhs[4], a->dim, "Invalid light source input", &a->nl, s);
    a->v = scmc_mex_sources(prhs[5], a->dim, "Invalid view source input", &a->nv, s);
    a->is_ff_l = mxGetScalar(prhs[6]) != 0.0;
    a->is_ff_v = mxGetScalar(prhs[7]) != 0.0;
    a->max_itr = (int64_t)mxGetScalar(prhs[8]);
    a->lambda = mxGetScalar(prhs[9]);
    a->do_cbs = mxGetScalar(prhs[10]) != 0.0;
    a->smp_flg = (int32_t)mxGetScalar(prhs[11]);
    scmc_mex_phase_fn(prhs[12], prhs[13], &a->ampfunc, s);
    if (nrhs >= 15) {
        a->has_ampfunc0 = 1;
        scmc_mex_phase_fn(prhs[12], prhs[14], &a->ampfunc0, s);
    }
    if (nrhs >= 16 && !mxIsEmpty(prhs[15])) {
        if (mxGetNumberOfElements(prhs[15]) != (size_t)a->dim)
            scmc_mex_fail(s, "scmc:gpu:lmean0", "lmean0 must have one entry per dimension");
        a->has_lmean0 = 1;
        memcpy(a->lmean0, mxGetDoubles(prhs[15]), (size_t)a->dim * sizeof(double));
    }
    a->seed = scmc_mex_seed();
    a->precision = scmc_mex_precision();
    a->device = scmc_mex_device();
}

/* A non-zero status of the library as a MATLAB error. */
static void scmc_mex_check(int rc, scmc_mex_scratch *s)
{
    if (rc == SCMC_OK) return;
    scmc_mex_release(s);
    mexErrMsgIdAndTxt("scmc:gpu:failed", "%s", scmc_last_error());
}

#endif /* SCMC_MEX_H */
