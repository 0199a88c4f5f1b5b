/*
 * postprocess.c - CPU FP64 restatement of SCMC's post-processing of rendered
 * fields and covariances.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle; never linked into the product).
 *
 *  refocus.m:1-34 - the field of a set of views (far-field directions)
 *      back-propagated onto a grid of points with one light direction:
 *      rU(p) = (sum_v conj(u_v) exp(-2 pi i/lambda v.p)) exp(2 pi i/lambda l.p).
 *      The grid is ndgrid(box_min(k):box_stp(k):box_max(k), ...) flattened
 *      column-major.  The reference fills rU in chunks jj = j+1 : min(j+Ns, N)
 *      for j = 1:Ns:N, so the first grid point is never written (stays 0);
 *      as_written = 1 keeps that.
 *
 *  samplingFromCovMatrix.m:47-64 (examples/samplingFromCovMatrix) - a field
 *      sample from a covariance C (N x N complex, N = nv*nl, index v + nv*l):
 *      Sigma = 0.5 [Re C, -Im C; Im C, Re C], s = g * chol(Sigma) for a row g
 *      of 2N standard normals (mvnrnd with zero mean; chol upper, Sigma =
 *      R'R), z = s(1:N) + i s(N+1:2N).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "scmc_oracle.h"

typedef double _Complex cplx;

/* MATLAB's a:s:b element count (small tolerance on (b-a)/s). */
static int64_t pp_colon_count(double a, double s, double b)
{
    if (s == 0 || (s > 0 && a > b) || (s < 0 && a < b)) return 0;
    double q = (b - a) / s;
    return (int64_t)floor(q + 1e-10 * fmax(1.0, fabs(q))) + 1;
}

int64_t oracle_refocus_grid(int32_t dim, const double *box_min, const double *box_max, const double *box_stp,
                            int64_t *dims)
{
    int64_t n = 1;
    for (int k = 0; k < dim; ++k) {
        dims[k] = pp_colon_count(box_min[k], box_stp[k], box_max[k]);
        n *= dims[k];
    }
    return n;
}

int oracle_refocus(const double *u, const double *v, int64_t nv, int32_t dim, const double *l,
                   const double *box_min, const double *box_max, const double *box_stp, double lambda,
                   int32_t as_written, double *rU)
{
    int64_t dims[3] = {1, 1, 1};
    const int64_t N = oracle_refocus_grid(dim, box_min, box_max, box_stp, dims);
    const cplx *uc = (const cplx *)u;
    cplx *out = (cplx *)rU;
    const double k = 2 * M_PI / lambda;
    for (int64_t p = 0; p < N; ++p) {
        out[p] = 0.0;
        if (as_written && p == 0) continue; /* refocus.m:27-31: jj starts at j+1 */
        double pos[3];
        int64_t r = p;
        for (int d = 0; d < dim; ++d) {
            pos[d] = box_min[d] + (double)(r % dims[d]) * box_stp[d];
            r /= dims[d];
        }
        cplx s = 0.0;
        for (int64_t i = 0; i < nv; ++i) {
            double dot = 0.0;
            for (int d = 0; d < dim; ++d) dot += v[dim * i + d] * pos[d];
            s += conj(uc[i]) * cexp(-I * k * dot);
        }
        double dl = 0.0;
        for (int d = 0; d < dim; ++d) dl += l[d] * pos[d];
        out[p] = s * cexp(I * k * dl);
    }
    return 0;
}

/* Cholesky Sigma = L L' (lower, column-major n x n, in place); -1 if not
 * positive definite.  chol's R is L'. */
static int chol_lower(double *A, int64_t n)
{
    for (int64_t j = 0; j < n; ++j) {
        double d = A[j + n * j];
        for (int64_t k = 0; k < j; ++k) d -= A[j + n * k] * A[j + n * k];
        if (!(d > 0)) return -1;
        d = sqrt(d);
        A[j + n * j] = d;
        for (int64_t i = j + 1; i < n; ++i) {
            double s = A[i + n * j];
            for (int64_t k = 0; k < j; ++k) s -= A[i + n * k] * A[j + n * k];
            A[i + n * j] = s / d;
        }
        for (int64_t i = 0; i < j; ++i) A[i + n * j] = 0.0;
    }
    return 0;
}

int oracle_sample_cov(const double *C, int64_t N, int64_t n_samples, const double *normals, double *Z)
{
    const int64_t n = 2 * N;
    const cplx *Cc = (const cplx *)C;
    double *S = malloc(sizeof(double) * n * n);
    if (!S) return -2;
    for (int64_t j = 0; j < N; ++j)
        for (int64_t i = 0; i < N; ++i) {
            const cplx c = Cc[i + N * j];
            S[i + n * j] = 0.5 * creal(c);
            S[(i + N) + n * (j + N)] = 0.5 * creal(c);
            S[i + n * (j + N)] = -0.5 * cimag(c);
            S[(i + N) + n * j] = 0.5 * cimag(c);
        }
    if (chol_lower(S, n)) {
        free(S);
        return -1;
    }
    cplx *Zc = (cplx *)Z;
    for (int64_t t = 0; t < n_samples; ++t) {
        const double *g = normals + n * t;
        /* s = g R = (L g)' */
        for (int64_t j = 0; j < N; ++j) {
            double re = 0.0, im = 0.0;
            for (int64_t i = 0; i <= j; ++i) re += S[j + n * i] * g[i];
            for (int64_t i = 0; i <= j + N; ++i) im += S[(j + N) + n * i] * g[i];
            Zc[j + N * t] = re + I * im;
        }
    }
    free(S);
    return 0;
}
