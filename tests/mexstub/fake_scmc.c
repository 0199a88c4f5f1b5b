/*
 * fake_scmc.c (test stub) - stands in for libscmc_gpu.so behind the MEX
 * shims: records the argument structs it is given (with copies of the
 * direction and table arrays) and fills each output element k with
 * (k, -k), or fails with a message when fake_fail is set.  Test
 * infrastructure only.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "scmc_gpu.h"

scmc_mc_args fake_mc;
scmc_fq_args fake_fq;
double fake_l[4096], fake_v[4096], fake_amp[8192], fake_icdf[4096], fake_amp0[8192];
int fake_calls, fake_fail, fake_cov_mm_null;

static void copy_n(double *dst, const double *src, size_t n, size_t cap)
{
    if (src) memcpy(dst, src, (n < cap ? n : cap) * sizeof(double));
}

static void record_mc(const scmc_mc_args *a)
{
    fake_mc = *a;
    copy_n(fake_l, a->l, (size_t)(a->dim * a->nl), 4096);
    copy_n(fake_v, a->v, (size_t)(a->dim * a->nv), 4096);
    if (a->ampfunc.sct_type == SCMC_SCT_TABULATED) {
        copy_n(fake_amp, a->ampfunc.eval_amp, 2 * (size_t)a->ampfunc.table_n, 8192);
        copy_n(fake_icdf, a->ampfunc.sample_icdf, (size_t)a->ampfunc.table_n, 4096);
    }
    if (a->has_ampfunc0 && a->ampfunc0.sct_type == SCMC_SCT_TABULATED)
        copy_n(fake_amp0, a->ampfunc0.eval_amp, 2 * (size_t)a->ampfunc0.table_n, 8192);
    ++fake_calls;
}

static void fill(double *out, size_t n)
{
    for (size_t k = 0; k < n; ++k) {
        out[2 * k] = (double)k;
        out[2 * k + 1] = -(double)k;
    }
}

const char *scmc_last_error(void) { return "fake failure"; }

int scmc_field(const scmc_mc_args *a, double *u)
{
    record_mc(a);
    if (fake_fail) return SCMC_ERR_INVALID;
    fill(u, (size_t)(a->nv * a->nl));
    return SCMC_OK;
}

int scmc_cov(const scmc_mc_args *a, double *Ms, double *Mm)
{
    record_mc(a);
    if (fake_fail) return SCMC_ERR_INVALID;
    const size_t n = (size_t)(a->nv * a->nv * a->nl * a->nl);
    fill(Ms, n);
    fake_cov_mm_null = Mm == NULL;
    if (Mm) fill(Mm, n);
    return SCMC_OK;
}

int scmc_fq_grid_size(double v_max, double v_stp, int64_t *nv0)
{
    const double q = (2 * v_max) / v_stp;
    *nv0 = (int64_t)floor(q + 1e-10 * fmax(1.0, fabs(q))) + 1;
    return SCMC_OK;
}

int scmc_field_fourier_quad(const scmc_fq_args *a, double *u)
{
    fake_fq = *a;
    copy_n(fake_l, a->l, 3 * (size_t)a->nl, 4096);
    ++fake_calls;
    if (fake_fail) return SCMC_ERR_INVALID;
    int64_t nv0 = 0;
    scmc_fq_grid_size(a->v_max, a->v_stp, &nv0);
    fill(u, (size_t)(nv0 * nv0 * a->nl));
    return SCMC_OK;
}
