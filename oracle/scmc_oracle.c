/*
 * scmc_oracle.c - CPU FP64 restatement of SCMC's Monte Carlo path
 * (MCfield / MCcov and the coreFunctions they call).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never linked
 * into the product.  Each function cites the reference file:line it
 * restates (paths relative to the cmu-ci-lab/mcspeckle tree).  The
 * reference's quirks are kept on purpose: 1-based nearest-index table
 * lookups, the unnormalised mean light direction in expSmpX, the weight
 * starting at the albedo, near-field entrance directions taken from the
 * first scatterer for every event, the Ms/Mm split and the CBS /2.
 *
 * One documented deviation: where a cosine fed to acos() is outside
 * [-1, 1] by rounding, MATLAB would produce a complex angle and then fail on
 * the complex table subscript; here it is clamped to [-1, 1].
 */
#include "scmc_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

#define KILL_THR 0.2 /* MCfield.m:109, MCcov.m:110 */

/* ------------------------------------------------------------------------ */
/* Philox-4x32-10                                                            */
/* ------------------------------------------------------------------------ */

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 52 random bits -> a double strictly inside (0,1), exactly representable. */
static double u52_to_unit(uint32_t a, uint32_t b)
{
    uint64_t m = ((uint64_t)a << 20) | (uint64_t)(b >> 12);
    return ((double)m + 0.5) * 0x1p-52;
}

typedef struct {
    int mode;
    const double *ut; int64_t un, ui;
    const double *nt; int64_t nn, ni;
    int exhausted;
    uint32_t key[2];
    uint64_t path;
    uint32_t uctr, nctr;
    double ub[2]; int uh;
    double nb[2]; int nh;
} rng_t;

static void rng_block(rng_t *r, uint32_t idx, uint32_t tag, uint32_t out[4])
{
    uint32_t ctr[4] = {idx, tag, (uint32_t)r->path, (uint32_t)(r->path >> 32)};
    oracle_philox4x32_10(ctr, r->key, out);
}

static void rng_set_path(rng_t *r, uint64_t path)
{
    r->path = path;
    r->uctr = r->nctr = 0;
    r->uh = r->nh = 0;
}

/* MATLAB rand */
static double rand_u(rng_t *r)
{
    if (r->mode == ORACLE_RNG_TAPE) {
        if (r->ui >= r->un) { r->exhausted = 1; return 0.5; }
        return r->ut[r->ui++];
    }
    if (r->uh == 0) {
        uint32_t o[4];
        rng_block(r, r->uctr++, 0u, o);
        r->ub[0] = u52_to_unit(o[0], o[1]);
        r->ub[1] = u52_to_unit(o[2], o[3]);
        r->uh = 2;
    }
    return r->ub[2 - r->uh--];
}

/* MATLAB randn: Box-Muller pairs on stream tag 1 in Philox mode. */
static double rand_n(rng_t *r)
{
    if (r->mode == ORACLE_RNG_TAPE) {
        if (r->ni >= r->nn) { r->exhausted = 1; return 0.0; }
        return r->nt[r->ni++];
    }
    if (r->nh == 0) {
        uint32_t o[4];
        rng_block(r, r->nctr++, 1u, o);
        double u1 = u52_to_unit(o[0], o[1]);
        double u2 = u52_to_unit(o[2], o[3]);
        double rad = sqrt(-2.0 * log(u1));
        double ang = (2.0 * M_PI) * u2;
        r->nb[0] = rad * cos(ang);
        r->nb[1] = rad * sin(ang);
        r->nh = 2;
    }
    return r->nb[2 - r->nh--];
}

void oracle_philox_stream(uint64_t seed, uint64_t path, int32_t tag, int64_t n, double *out)
{
    rng_t r;
    memset(&r, 0, sizeof r);
    r.mode = ORACLE_RNG_PHILOX;
    r.key[0] = (uint32_t)seed;
    r.key[1] = (uint32_t)(seed >> 32);
    rng_set_path(&r, path);
    for (int64_t i = 0; i < n; ++i) out[i] = tag ? rand_n(&r) : rand_u(&r);
}

static void rng_init(rng_t *r, const oracle_rng_spec *rs, uint64_t seed)
{
    memset(r, 0, sizeof *r);
    r->mode = rs->mode;
    r->ut = rs->utape; r->un = rs->utape ? rs->un : 0;
    r->nt = rs->ntape; r->nn = rs->ntape ? rs->nn : 0;
    r->key[0] = (uint32_t)seed;
    r->key[1] = (uint32_t)(seed >> 32);
}

/* MATLAB round(): half away from zero. */
static double mround(double x) { return x < 0 ? -floor(-x + 0.5) : floor(x + 0.5); }

/* ------------------------------------------------------------------------ */
/* coreFunctions                                                             */
/* ------------------------------------------------------------------------ */

/* cubeDist.m:1-11: distance from x along direction v to the box boundary. */
static double cube_dist(const double *x, const double *vmin, const double *vmax,
                        const double *v, int dim)
{
    const double thr = pow(0.1, 7);
    double d = INFINITY;
    for (int j = 0; j < dim; ++j) {
        double den = fmax(fabs(v[j]), thr);
        double bd = (v[j] <= 0) ? (x[j] - vmin[j]) / den : (-x[j] + vmax[j]) / den;
        d = fmin(d, bd);
    }
    return d;
}

/* evalphaseatt.m:1-21 for one direction / position v. */
cplx oracle_internal_evalphaseatt1(const double *x, const double *v, int is_ff, double sigt,
                                   double lambda, const double *bmin, const double *bmax, int dim);
static cplx evalphaseatt1(const double *x, const double *v, int is_ff, double sigt,
                          double lambda, const double *bmin, const double *bmax, int dim)
{
    double pv, rv, bdv;
    if (is_ff) {
        double nv[3];
        pv = 0.0;
        for (int k = 0; k < dim; ++k) { pv += x[k] * v[k]; nv[k] = -v[k]; }
        rv = 1.0;
        bdv = cube_dist(x, bmin, bmax, nv, dim);
    } else {
        double d[3], nd = 0.0, nu[3];
        for (int k = 0; k < dim; ++k) { d[k] = x[k] - v[k]; nd += d[k] * d[k]; }
        nd = sqrt(nd);
        for (int k = 0; k < dim; ++k) nu[k] = -(d[k] / nd);
        pv = nd;
        rv = 1.0 / pow(nd + 0.01 * lambda, (dim - 1) / 2.0);
        bdv = fmin(cube_dist(x, bmin, bmax, nu, dim), nd);
    }
    double ph = (M_PI * 2.0 / lambda) * pv;
    double at = sigt / 2.0 * bdv;
    return exp(-at) * (cos(ph) + I * sin(ph)) * rv;
}

cplx oracle_internal_evalphaseatt1(const double *x, const double *v, int is_ff, double sigt,
                                   double lambda, const double *bmin, const double *bmax, int dim)
{
    return evalphaseatt1(x, v, is_ff, sigt, lambda, bmin, bmax, dim);
}

/* evaluateHG.m:25-39 (cosineFlag = 1). */
static double evaluate_hg(double c, double g, int dim)
{
    double den = 1.0 + (g * g + (-2.0 * (g * c)));
    if (dim == 3) return (1.0 / 4.0 / M_PI) * ((1.0 - g * g) / pow(den, 1.5));
    return (1.0 / 2.0 / M_PI) * ((1.0 - g * g) / den);
}

/* evalampfunc_general.m:1-19 with evalampfunc_amplitude.m:1-9. */
static cplx evalampfunc(double c, const scmc_phase_function *pf, int dim)
{
    switch (pf->sct_type) {
    case SCMC_SCT_ISOTROPIC:
        return 1.0 / sqrt(pow(2.0, dim - 1) * M_PI);
    case SCMC_SCT_TABULATED: {
        double cc = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
        if (pf->table_in_cos) { /* extension: cos(theta) bins cos_i = 1 - 2i/(n-1) */
            int64_t i = (int64_t)mround((1.0 - cc) * 0.5 * (double)(pf->table_n - 1));
            if (i < 0) i = 0;
            if (i > pf->table_n - 1) i = pf->table_n - 1;
            return pf->eval_amp[2 * i] + I * pf->eval_amp[2 * i + 1];
        }
        double ang = acos(cc);
        int n = pf->table_n;
        double span = (dim == 2) ? 2.0 * M_PI : M_PI;
        int64_t idx = (int64_t)mround(ang * (double)(n - 1) / span); /* 0-based */
        if (idx < 0) idx = 0;
        if (idx > n - 1) idx = n - 1;
        return pf->eval_amp[2 * idx] + I * pf->eval_amp[2 * idx + 1];
    }
    default:
        return sqrt(evaluate_hg(c, pf->g, dim));
    }
}

/* sampleHG.m:1-18 */
static double sample_hg(double g, int dim, rng_t *r)
{
    if (fabs(g) < 0.001) return 2.0 * rand_u(r) - 1.0;
    if (dim == 3) {
        double t = (1.0 - g * g) / (1.0 - g + 2.0 * g * rand_u(r));
        return (1.0 / (2.0 * g)) * ((1.0 + g * g) - t * t);
    }
    double th = 2.0 * atan((1.0 - g) / (1.0 + g) * tan(M_PI / 2.0 * (1.0 - 2.0 * rand_u(r))));
    return cos(th);
}

/* smpampfunc.m:1-8 */
static double smpampfunc(const scmc_phase_function *pf, rng_t *r)
{
    int n = pf->table_n;
    double stp = 1.0 / (double)(n - 1);
    double a = rand_u(r);
    int64_t i = (int64_t)mround(a / stp); /* 0-based */
    if (i > n - 1) i = n - 1;
    return pf->sample_icdf[i];
}

/* rotateBytheta.m:1-28 */
static void rotate_by_theta(const double *ow, double c, int dim, double *w, rng_t *r)
{
    double s = 1.0 - c * c;
    s = s > 0 ? sqrt(s) : 0.0; /* real(sqrt(.)) */
    if (dim == 2) {
        s = ((rand_u(r) > 0.5) * 2.0 - 1.0) * s;
        double w0 = c * ow[0] + s * ow[1];
        double w1 = -s * ow[0] + c * ow[1];
        w[0] = w0; w[1] = w1;
        return;
    }
    double phi = M_PI * 2.0 * rand_u(r);
    double sp = sin(phi), cp = cos(phi);
    if (fabs(ow[2]) > 0.999999999) {
        w[0] = s * cp;
        w[1] = s * sp;
        w[2] = c * ow[2] / fabs(ow[2]);
    } else {
        double tmp = sqrt(1.0 - ow[2] * ow[2]);
        double w0 = s * (ow[0] * ow[2] * cp - ow[1] * sp) / tmp + ow[0] * c;
        double w1 = s * (ow[1] * ow[2] * cp + ow[0] * sp) / tmp + ow[1] * c;
        double w2 = -s * cp * tmp + ow[2] * c;
        w[0] = w0; w[1] = w1; w[2] = w2;
    }
}

static void randn_dir(int dim, double *w, rng_t *r)
{
    double n2 = 0.0;
    for (int k = 0; k < dim; ++k) { w[k] = rand_n(r); n2 += w[k] * w[k]; }
    double nrm = sqrt(n2);
    for (int k = 0; k < dim; ++k) w[k] = w[k] / nrm;
}

/* smpampfunc_general.m:1-21 */
static void smpampfunc_general(const double *ow, const scmc_phase_function *pf, int dim,
                               double *w, rng_t *r)
{
    if (pf->sct_type == SCMC_SCT_ISOTROPIC) { randn_dir(dim, w, r); return; }
    double c = (pf->sct_type == SCMC_SCT_TABULATED)
                   ? (pf->table_in_cos ? smpampfunc(pf, r) : cos(smpampfunc(pf, r)))  /* cos bins: icdf holds cosines */
                   : sample_hg(pf->g, dim, r);
    rotate_by_theta(ow, c, dim, w, r);
}

/* expSmpX.m:1-12 (lmean is the unnormalised mean light direction). */
static void exp_smp_x(const double *bmin, const double *bmax, const double *lmean,
                      double sigs, int dim, double *x, double *px, rng_t *r)
{
    double lz = fabs(lmean[dim - 1]);
    double s = sigs / lz;
    double dmax = bmax[dim - 1] - bmin[dim - 1];
    double rmax = 1.0 - exp(-dmax * s);
    double d = -log(-rand_u(r) * rmax + 1.0) / s;
    for (int k = 0; k < dim - 1; ++k) x[k] = rand_u(r) * (bmax[k] - bmin[k]) + bmin[k];
    x[dim - 1] = (lmean[dim - 1] > 0) ? (d + bmin[dim - 1]) : (-d + bmax[dim - 1]);
    *px = exp(-s * d) / rmax * s * dmax;
}

static double dotn(const double *a, const double *b, int dim)
{
    double s = 0.0;
    for (int k = 0; k < dim; ++k) s += a[k] * b[k];
    return s;
}

/* ------------------------------------------------------------------------ */
/* Per-path NEE context shared by MCfield and MCcov                         */
/* ------------------------------------------------------------------------ */

typedef struct {
    int dim, nv, nl, is_ff_l, is_ff_v, cbs;
    double sigt, lambda;
    const double *bmin, *bmax;
    const double *l, *v;          /* dim x n */
    double *vs;                   /* ff_sign * v */
    double meanl[3], unmeanl[3];
    const scmc_phase_function *pf, *pf0;
    int has_pf0;
    /* per path */
    double *rv, *rl;              /* entrance directions (dim x n) */
    cplx *af_vl;                  /* nv x nl single-scatter amplitudes */
    cplx *e_l0, *e_l0_ms, *e_v0, *e_v0_ms;
    double w0p;
    /* per event */
    cplx *e_v_ms, *e_l_ms;
} nee_t;

static void nee_alloc(nee_t *c, const scmc_mc_args *a)
{
    memset(c, 0, sizeof *c);
    c->dim = a->dim; c->nv = (int)a->nv; c->nl = (int)a->nl;
    c->is_ff_l = a->is_ff_l; c->is_ff_v = a->is_ff_v; c->cbs = a->do_cbs;
    c->sigt = a->sigt; c->lambda = a->lambda;
    c->bmin = a->box_min; c->bmax = a->box_max;
    c->l = a->l; c->v = a->v;
    c->pf = &a->ampfunc; c->pf0 = &a->ampfunc0; c->has_pf0 = a->has_ampfunc0;
    int dim = c->dim, nv = c->nv, nl = c->nl;
    c->vs = malloc(sizeof(double) * dim * nv);
    double ff_sign = -2.0 * (a->is_ff_v ? 1 : 0) + 1.0; /* MCfield.m:106 */
    for (int i = 0; i < dim * nv; ++i) c->vs[i] = ff_sign * a->v[i];
    c->rv = malloc(sizeof(double) * dim * nv);
    c->rl = malloc(sizeof(double) * dim * nl);
    c->af_vl = malloc(sizeof(cplx) * nv * nl);
    c->e_l0 = malloc(sizeof(cplx) * nl);
    c->e_l0_ms = malloc(sizeof(cplx) * nl);
    c->e_l_ms = malloc(sizeof(cplx) * nl);
    c->e_v0 = malloc(sizeof(cplx) * nv);
    c->e_v0_ms = malloc(sizeof(cplx) * nv);
    c->e_v_ms = malloc(sizeof(cplx) * nv);
    /* MCfield.m:77-82: unmeanl = mean(l,2) unless lmean0 is given */
    for (int k = 0; k < dim; ++k) {
        double s = 0.0;
        for (int j = 0; j < nl; ++j) s += a->l[dim * j + k];
        c->unmeanl[k] = a->has_lmean0 ? a->lmean0[k] : s / nl;
    }
    double n = sqrt(dotn(c->unmeanl, c->unmeanl, dim));
    for (int k = 0; k < dim; ++k) c->meanl[k] = c->unmeanl[k] / n;
    /* MCfield.m:90-104: far-field amplitudes and entrance directions */
    if (c->is_ff_v) memcpy(c->rv, a->v, sizeof(double) * dim * nv);
    if (c->is_ff_l) memcpy(c->rl, a->l, sizeof(double) * dim * nl);
    if (c->is_ff_v && c->is_ff_l)
        for (int j = 0; j < nl; ++j)
            for (int i = 0; i < nv; ++i)
                c->af_vl[i + nv * j] = evalampfunc(dotn(a->l + dim * j, a->v + dim * i, dim), c->pf, dim);
}

static void nee_free(nee_t *c)
{
    free(c->vs); free(c->rv); free(c->rl); free(c->af_vl);
    free(c->e_l0); free(c->e_l0_ms); free(c->e_l_ms);
    free(c->e_v0); free(c->e_v0_ms); free(c->e_v_ms);
}

/* MCfield.m:130-181 / MCcov.m:128-179: everything that depends on the first
 * scatterer x and the first direction w. */
static void nee_path(nee_t *c, const double *x, const double *w)
{
    int dim = c->dim, nv = c->nv, nl = c->nl;
    if (!c->is_ff_v)
        for (int i = 0; i < nv; ++i) {
            double d[3], s = 0.0;
            for (int k = 0; k < dim; ++k) { d[k] = c->v[dim * i + k] - x[k]; s += d[k] * d[k]; }
            s = sqrt(s);
            for (int k = 0; k < dim; ++k) c->rv[dim * i + k] = d[k] / s;
        }
    if (!c->is_ff_l)
        for (int j = 0; j < nl; ++j) {
            double d[3], s = 0.0;
            for (int k = 0; k < dim; ++k) { d[k] = x[k] - c->l[dim * j + k]; s += d[k] * d[k]; }
            s = sqrt(s);
            for (int k = 0; k < dim; ++k) c->rl[dim * j + k] = d[k] / s;
        }
    if (!(c->is_ff_v && c->is_ff_l))
        for (int j = 0; j < nl; ++j)
            for (int i = 0; i < nv; ++i)
                c->af_vl[i + nv * j] = evalampfunc(dotn(c->rl + dim * j, c->rv + dim * i, dim), c->pf, dim);
    /* first-direction pdf w0p (MCfield.m:149-155) */
    if (!c->has_pf0) c->w0p = 1.0 / sqrt(pow(2.0, dim - 1) * M_PI);
    else c->w0p = creal(evalampfunc(dotn(c->meanl, w, dim), c->pf0, dim));
    for (int j = 0; j < nl; ++j) {
        cplx af_l = evalampfunc(dotn(w, c->rl + dim * j, dim), c->pf, dim) / c->w0p;
        c->e_l0[j] = evalphaseatt1(x, c->l + dim * j, c->is_ff_l, c->sigt, c->lambda, c->bmin, c->bmax, dim);
        c->e_l0_ms[j] = c->e_l0[j] * af_l;
    }
    for (int i = 0; i < nv; ++i) {
        c->e_v0[i] = evalphaseatt1(x, c->vs + dim * i, c->is_ff_v, c->sigt, c->lambda, c->bmin, c->bmax, dim);
        if (c->cbs) {
            cplx af_v = evalampfunc(-dotn(w, c->rv + dim * i, dim), c->pf, dim) / c->w0p;
            c->e_v0_ms[i] = c->e_v0[i] * af_v;
        }
    }
}

/* MCfield.m:196-205 / MCcov.m:205-219: last-scatterer vectors for pL > 1. */
static void nee_event(nee_t *c, const double *x, const double *ow)
{
    int dim = c->dim, nv = c->nv, nl = c->nl;
    for (int i = 0; i < nv; ++i) {
        cplx e_v = evalphaseatt1(x, c->vs + dim * i, c->is_ff_v, c->sigt, c->lambda, c->bmin, c->bmax, dim);
        cplx af_v = evalampfunc(dotn(ow, c->rv + dim * i, dim), c->pf, dim);
        c->e_v_ms[i] = e_v * af_v;
    }
    if (c->cbs)
        for (int j = 0; j < nl; ++j) {
            cplx e_l = evalphaseatt1(x, c->l + dim * j, c->is_ff_l, c->sigt, c->lambda, c->bmin, c->bmax, dim);
            cplx af_l = evalampfunc(-dotn(ow, c->rl + dim * j, dim), c->pf, dim);
            c->e_l_ms[j] = e_l * af_l;
        }
}

/* MCfield.m:207-222: u += sqrt(weight/px) * tpath * exp(2*pi*i*xi) */
static void field_update(nee_t *c, int pL, double wpx, double xi, cplx *u)
{
    int nv = c->nv, nl = c->nl;
    double s = sqrt(wpx);
    double ph = 2.0 * M_PI * xi;
    cplx rot = cos(ph) + I * sin(ph);
    for (int j = 0; j < nl; ++j)
        for (int i = 0; i < nv; ++i) {
            cplx t;
            if (pL == 1) {
                t = c->af_vl[i + nv * j] * (c->e_v0[i] * c->e_l0[j]);
            } else {
                t = c->e_v_ms[i] * c->e_l0_ms[j];
                if (c->cbs) t = 1.0 / sqrt(2.0) * (t + c->e_v0_ms[i] * c->e_l_ms[j]);
            }
            u[i + nv * j] += (s * t) * rot;
        }
}

/* MCcov.m:190, 217-263: covariance updates, following the reference's
 * four-term M00/Mnn/Mn0/M0n form. */
static void cov_update(nee_t *c, int pL, double wpx, cplx *Ms, cplx *Mm, int threads)
{
    const int nv = c->nv, nl = c->nl;
    const int64_t nvv = (int64_t)nv * nv;
    const cplx *ev0 = (pL > 1 && c->cbs) ? c->e_v0_ms : c->e_v0; /* M00 (MCcov.m:190, 227-229) */
    (void)threads;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) if (threads > 1) num_threads(threads > 1 ? threads : 1)
#endif
    for (int j2 = 0; j2 < nl; ++j2)
        for (int j1 = 0; j1 < nl; ++j1) {
            cplx *Mout = (pL == 1 ? Ms : Mm) + nvv * (j1 + (int64_t)nl * j2);
            if (pL == 1) {
                cplx sl = conj(c->e_l0[j2]) * c->e_l0[j1];
                for (int v2 = 0; v2 < nv; ++v2)
                    for (int v1 = 0; v1 < nv; ++v1) {
                        cplx m00 = ev0[v1] * conj(ev0[v2]);
                        cplx af = c->af_vl[v1 + nv * j1] * conj(c->af_vl[v2 + nv * j2]);
                        Mout[v1 + (int64_t)nv * v2] += wpx * m00 * sl * af;
                    }
            } else if (c->cbs) {
                cplx s00 = conj(c->e_l_ms[j2]) * c->e_l_ms[j1];
                cplx snn = conj(c->e_l0_ms[j2]) * c->e_l0_ms[j1];
                cplx sn0 = conj(c->e_l_ms[j2]) * c->e_l0_ms[j1];
                cplx s0n = conj(c->e_l0_ms[j2]) * c->e_l_ms[j1];
                for (int v2 = 0; v2 < nv; ++v2)
                    for (int v1 = 0; v1 < nv; ++v1) {
                        cplx m00 = ev0[v1] * conj(ev0[v2]);
                        cplx mnn = c->e_v_ms[v1] * conj(c->e_v_ms[v2]);
                        cplx mn0 = c->e_v_ms[v1] * conj(c->e_v0_ms[v2]);
                        cplx m0n = c->e_v0_ms[v1] * conj(c->e_v_ms[v2]);
                        Mout[v1 + (int64_t)nv * v2] += wpx * (m00 * s00 + mnn * snn + mn0 * sn0 + m0n * s0n);
                    }
            } else {
                cplx snn = conj(c->e_l0_ms[j2]) * c->e_l0_ms[j1];
                for (int v2 = 0; v2 < nv; ++v2)
                    for (int v1 = 0; v1 < nv; ++v1) {
                        cplx mnn = c->e_v_ms[v1] * conj(c->e_v_ms[v2]);
                        Mout[v1 + (int64_t)nv * v2] += wpx * (mnn * snn);
                    }
            }
        }
}

/* ------------------------------------------------------------------------ */
/* The walk (MCfield.m:112-250, MCcov.m:112-290)                             */
/* ------------------------------------------------------------------------ */

/* MCfieldOnWave.m:177-222: the lights combined with weights Wl before the
 * update.  Single scattering: u_i += e_v0_i * sum_j af_ij e_l0_j Wl_j
 * (line 221); multiple: u_i += e_v_ms_i * sum_j e_l0_ms_j Wl_j, with CBS
 * (u + e_v0_ms_i * sum_j e_l_ms_j Wl_j) / sqrt2 (lines 177, 212, 223-226). */
static void field_update_onwave(nee_t *c, int pL, double wpx, double xi, const cplx *Wl, cplx *u)
{
    int nv = c->nv, nl = c->nl;
    double s = sqrt(wpx);
    double ph = 2.0 * M_PI * xi;
    cplx rot = cos(ph) + I * sin(ph);
    if (pL == 1) {
        for (int i = 0; i < nv; ++i) {
            cplx acc = 0.0;
            for (int j = 0; j < nl; ++j) acc += c->af_vl[i + nv * j] * (c->e_l0[j] * Wl[j]);
            u[i] += (s * (c->e_v0[i] * acc)) * rot;
        }
        return;
    }
    cplx b = 0.0, b2 = 0.0;
    for (int j = 0; j < nl; ++j) b += c->e_l0_ms[j] * Wl[j];
    if (c->cbs)
        for (int j = 0; j < nl; ++j) b2 += c->e_l_ms[j] * Wl[j];
    for (int i = 0; i < nv; ++i) {
        cplx t = c->e_v_ms[i] * b;
        if (c->cbs) t = 1.0 / sqrt(2.0) * (t + c->e_v0_ms[i] * b2);
        u[i] += (s * t) * rot;
    }
}

typedef struct {
    int kind;          /* 0 field, 1 cov, 2 records, 3 field on a wave (weighted lights) */
    cplx *u, *Ms, *Mm;
    const cplx *Wl;    /* kind 3: light weights */
    int threads;
    /* records */
    int64_t cap, n;
    double *x, *ow, *x1, *w1, *wpx, *xi;
    int32_t *plen;
    int64_t *path;
} sink_t;

static int walk(const scmc_mc_args *a, oracle_rng_spec *rs, int with_phase, sink_t *sk)
{
    const int dim = a->dim;
    rng_t r;
    rng_init(&r, rs, a->seed);
    nee_t c;
    nee_alloc(&c, a);
    double box_w[3];
    for (int k = 0; k < dim; ++k) box_w[k] = a->box_max[k] - a->box_min[k];
    int rc = 0;

    for (int64_t itr = 0; itr < a->max_itr; ++itr) {
        if (r.mode == ORACLE_RNG_PHILOX) rng_set_path(&r, a->path_offset + (uint64_t)itr);
        double x[3] = {0, 0, 0}, x1[3], w[3] = {0, 0, 0}, w1[3] = {0, 0, 0}, ow[3] = {0, 0, 0}, px;
        /* first scatter (MCfield.m:118-125) */
        if (a->smp_flg == 1) {
            for (int k = 0; k < dim; ++k) x[k] = rand_u(&r) * box_w[k] + a->box_min[k];
            px = 1.0;
        } else {
            exp_smp_x(a->box_min, a->box_max, c.unmeanl, a->sigt, dim, x, &px, &r);
        }
        memcpy(x1, x, sizeof x);
        /* first direction (MCfield.m:149-155) */
        if (!a->has_ampfunc0) randn_dir(dim, w, &r);
        else smpampfunc_general(c.meanl, &a->ampfunc0, dim, w, &r);
        memcpy(w1, w, sizeof w);
        if (sk->kind != 2) nee_path(&c, x, w);

        int pL = 0;
        double weight = a->albedo;
        for (;;) {
            ++pL;
            double xi = 0.0;
            if (with_phase) xi = rand_u(&r); /* MCfield.m:220 */
            double wpx = weight / px;
            if (sk->kind == 2) {
                if (sk->n < sk->cap) {
                    int64_t e = sk->n;
                    for (int k = 0; k < 3; ++k) {
                        sk->x[3 * e + k] = k < dim ? x[k] : 0.0;
                        sk->ow[3 * e + k] = k < dim ? ow[k] : 0.0;
                        sk->x1[3 * e + k] = k < dim ? x1[k] : 0.0;
                        sk->w1[3 * e + k] = k < dim ? w1[k] : 0.0;
                    }
                    sk->wpx[e] = wpx;
                    sk->xi[e] = xi;
                    sk->plen[e] = pL;
                    sk->path[e] = itr;
                }
                sk->n++;
            } else {
                if (pL > 1) nee_event(&c, x, ow);
                if (sk->kind == 0) field_update(&c, pL, wpx, xi, sk->u);
                else if (sk->kind == 3) field_update_onwave(&c, pL, wpx, xi, sk->Wl, sk->u);
                else cov_update(&c, pL, wpx, sk->Ms, sk->Mm, sk->threads);
            }
            /* free flight (MCfield.m:225-232) */
            double d = -log(-rand_u(&r) + 1.0) / a->sigt;
            int out = 0;
            for (int k = 0; k < dim; ++k) {
                x[k] = x[k] + d * w[k];
                if (x[k] > a->box_max[k] || x[k] < a->box_min[k]) out = 1;
            }
            if (out) break;
            /* roulette (MCfield.m:236-242) */
            if (weight < KILL_THR) {
                if (rand_u(&r) > a->albedo) break;
            } else {
                weight = weight * a->albedo;
            }
            memcpy(ow, w, sizeof w);
            smpampfunc_general(ow, &a->ampfunc, dim, w, &r);
            if (a->max_events_per_path > 0 && pL >= a->max_events_per_path) { rc = -3; break; }
        }
        if (r.exhausted) { rc = -1; break; }
        if (rc) break;
    }
    rs->used_u = r.ui;
    rs->used_n = r.ni;
    nee_free(&c);
    return rc;
}

static double box_volume(const scmc_mc_args *a)
{
    double V = 1.0;
    for (int k = 0; k < a->dim; ++k) V *= a->box_max[k] - a->box_min[k];
    return V;
}

static double norm_count(const scmc_mc_args *a)
{
    return (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
}

static void field_normalise(const scmc_mc_args *a, cplx *u)
{
    /* MCfield.m:253-254 */
    double f = sqrt(1.0 / norm_count(a) * box_volume(a) * a->sigt);
    for (int64_t i = 0; i < a->nv * a->nl; ++i) u[i] *= f;
}

static void cov_normalise(const scmc_mc_args *a, cplx *Ms, cplx *Mm)
{
    /* MCcov.m:293-299 */
    int64_t n = a->nv * a->nv * a->nl * a->nl;
    double V = box_volume(a), m = norm_count(a);
    for (int64_t i = 0; i < n; ++i) {
        if (a->do_cbs) Mm[i] = Mm[i] / 2.0;
        Mm[i] = Mm[i] / m * V * a->sigt;
        Ms[i] = Ms[i] / m * V * a->sigt;
    }
}

int oracle_field(const scmc_mc_args *a, oracle_rng_spec *rs, double *u)
{
    cplx *uc = (cplx *)u;
    memset(u, 0, sizeof(double) * 2 * a->nv * a->nl);
    sink_t sk;
    memset(&sk, 0, sizeof sk);
    sk.kind = 0;
    sk.u = uc;
    int rc = walk(a, rs, 1, &sk);
    field_normalise(a, uc);
    return rc;
}

int oracle_field_onwave(const scmc_mc_args *a, const double *Wl, oracle_rng_spec *rs, double *u)
{
    cplx *uc = (cplx *)u;
    memset(u, 0, sizeof(double) * 2 * a->nv);
    sink_t sk;
    memset(&sk, 0, sizeof sk);
    sk.kind = 3;
    sk.u = uc;
    sk.Wl = (const cplx *)Wl;
    int rc = walk(a, rs, 1, &sk);
    /* MCfield.m:253-254 normalisation over the nv entries */
    scmc_mc_args one = *a;
    one.nl = 1;
    field_normalise(&one, uc);
    return rc;
}

int oracle_cov(const scmc_mc_args *a, oracle_rng_spec *rs, double *Ms, double *Mm, int threads)
{
    int64_t n = a->nv * a->nv * a->nl * a->nl;
    memset(Ms, 0, sizeof(double) * 2 * n);
    memset(Mm, 0, sizeof(double) * 2 * n);
    sink_t sk;
    memset(&sk, 0, sizeof sk);
    sk.kind = 1;
    sk.Ms = (cplx *)Ms;
    sk.Mm = (cplx *)Mm;
    sk.threads = threads;
    int rc = walk(a, rs, 0, &sk);
    cov_normalise(a, (cplx *)Ms, (cplx *)Mm);
    return rc;
}

int oracle_records(const scmc_mc_args *a, oracle_rng_spec *rs, int32_t want_phase,
                   int64_t capacity, double *x, double *ow, double *x1, double *w1,
                   double *wpx, double *xi, int32_t *plen, int64_t *path, int64_t *n_events)
{
    sink_t sk;
    memset(&sk, 0, sizeof sk);
    sk.kind = 2;
    sk.cap = capacity;
    sk.x = x; sk.ow = ow; sk.x1 = x1; sk.w1 = w1; sk.wpx = wpx; sk.xi = xi;
    sk.plen = plen; sk.path = path;
    int rc = walk(a, rs, want_phase, &sk);
    *n_events = sk.n;
    if (!rc && sk.n > capacity) rc = -2;
    return rc;
}

/* Replay: the same NEE and update rules applied to externally walked events. */
static void replay(const scmc_mc_args *a, int64_t n, const double *x, const double *ow,
                   const double *x1, const double *w1, const double *wpx, const double *xi,
                   const int32_t *plen, int kind, cplx *u, cplx *Ms, cplx *Mm, int threads)
{
    nee_t c;
    nee_alloc(&c, a);
    int dim = a->dim;
    for (int64_t e = 0; e < n; ++e) {
        double xe[3], owe[3], x1e[3], w1e[3];
        for (int k = 0; k < 3; ++k) {
            xe[k] = x[3 * e + k]; owe[k] = ow[3 * e + k];
            x1e[k] = x1[3 * e + k]; w1e[k] = w1[3 * e + k];
        }
        (void)dim;
        if (plen[e] == 1) nee_path(&c, x1e, w1e);
        else nee_event(&c, xe, owe);
        if (kind == 0) field_update(&c, plen[e], wpx[e], xi[e], u);
        else cov_update(&c, plen[e], wpx[e], Ms, Mm, threads);
    }
    nee_free(&c);
}

int oracle_field_from_records(const scmc_mc_args *a, int64_t n, const double *x,
                              const double *ow, const double *x1, const double *w1,
                              const double *wpx, const double *xi, const int32_t *plen,
                              double *u)
{
    memset(u, 0, sizeof(double) * 2 * a->nv * a->nl);
    replay(a, n, x, ow, x1, w1, wpx, xi, plen, 0, (cplx *)u, NULL, NULL, 1);
    field_normalise(a, (cplx *)u);
    return 0;
}

int oracle_cov_from_records(const scmc_mc_args *a, int64_t n, const double *x,
                            const double *ow, const double *x1, const double *w1,
                            const double *wpx, const int32_t *plen,
                            double *Ms, double *Mm, int threads)
{
    int64_t m = a->nv * a->nv * a->nl * a->nl;
    memset(Ms, 0, sizeof(double) * 2 * m);
    memset(Mm, 0, sizeof(double) * 2 * m);
    replay(a, n, x, ow, x1, w1, wpx, NULL, plen, 1, NULL, (cplx *)Ms, (cplx *)Mm, threads);
    cov_normalise(a, (cplx *)Ms, (cplx *)Mm);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* MCfieldFourierQuad.m:154-213: the isotropic walk recording every vertex  */
/* ------------------------------------------------------------------------ */
int oracle_internal_fq_walk(const scmc_fq_args *a, const double *bmin, const double *bmax,
                            const double *unmeanl, oracle_rng_spec *rs, int64_t cap,
                            double *xL, double *x1L, double *pxr, double *pxi, int64_t *n_vert)
{
    rng_t r;
    rng_init(&r, rs, a->seed);
    const int dim = 3;
    double bw[3];
    for (int k = 0; k < 3; ++k) bw[k] = bmax[k] - bmin[k];
    int64_t c = 0;
    int rc = 0;
    for (int64_t itr = 0; itr < a->max_itr; ++itr) {
        if (r.mode == ORACLE_RNG_PHILOX) rng_set_path(&r, a->path_offset + (uint64_t)itr);
        double x[3], x1[3], w[3], px;
        if (a->smp_flg == 1) {
            for (int k = 0; k < dim; ++k) x[k] = rand_u(&r) * bw[k] + bmin[k];
            px = 1.0;
        } else {
            exp_smp_x(bmin, bmax, unmeanl, a->sigt, dim, x, &px, &r);
        }
        memcpy(x1, x, sizeof x);
        randn_dir(dim, w, &r);
        double weight = a->albedo;
        int p_len = 0;
        for (;;) {
            ++p_len;
            if (c < cap) {
                for (int k = 0; k < 3; ++k) { xL[3 * c + k] = x[k]; x1L[3 * c + k] = x1[k]; }
                double s = sqrt(weight / px);
                double ph = 2 * M_PI * rand_u(&r);
                double re = s * cos(ph), im = s * sin(ph);
                if (a->do_cbs && p_len > 1) { re = 1 / sqrt(2.0) * re; im = 1 / sqrt(2.0) * im; }
                pxr[c] = re;
                pxi[c] = im;
            } else {
                (void)rand_u(&r);
            }
            ++c;
            double d = -log(-rand_u(&r) + 1.0) / a->sigt;
            int out = 0;
            for (int k = 0; k < dim; ++k) {
                x[k] = x[k] + d * w[k];
                if (x[k] > bmax[k] || x[k] < bmin[k]) out = 1;
            }
            if (out) break;
            if (weight < KILL_THR) {
                if (rand_u(&r) > a->albedo) break;
            } else {
                weight = weight * a->albedo;
            }
            if (a->sct_type == SCMC_SCT_HG) {
                /* extension: the smpampfunc_general(ow, sct_type, ampfunc) call that
                 * MCfieldFourierQuad.m:208 leaves commented out, with HG(g) */
                double ow[3];
                memcpy(ow, w, sizeof ow);
                scmc_phase_function pf;
                memset(&pf, 0, sizeof pf);
                pf.sct_type = SCMC_SCT_HG;
                pf.g = a->g;
                smpampfunc_general(ow, &pf, dim, w, &r);
            } else {
                randn_dir(dim, w, &r);
            }
        }
        if (r.exhausted) { rc = -1; break; }
    }
    rs->used_u = r.ui;
    rs->used_n = r.ni;
    *n_vert = c;
    if (!rc && c > cap) rc = -2;
    return rc;
}

/* ======================================================================== */
/* Heterogeneous (voxel) medium: MCCovHetro.m, MCsampleHetro.m              */
/* ======================================================================== */

typedef struct {
    int dim;
    const double *sigt, *alb;
    double alb_scalar;
    double bmin[3], bmax[3], bbin[3];
    int64_t nb[3];
    double sigt_max;
    int bad;  /* a voxel march ran away (guard) */
    int trilinear; /* extension: sigt trilinear between voxel centres */
} grid_t;

static void grid_init(grid_t *g, const scmc_hetero_args *a)
{
    memset(g, 0, sizeof *g);
    g->dim = a->mc.dim;
    g->sigt = a->sigt_grid;
    g->alb = a->albedo_grid;
    g->alb_scalar = a->mc.albedo;
    int64_t n = 1;
    for (int k = 0; k < g->dim; ++k) {
        g->bmin[k] = a->mc.box_min[k];
        g->bmax[k] = a->mc.box_max[k];
        g->bbin[k] = a->box_bin[k];
        g->nb[k] = (int64_t)mround((g->bmax[k] - g->bmin[k]) / g->bbin[k]); /* findBin.m:4 */
        n *= g->nb[k];
    }
    g->sigt_max = -INFINITY;
    for (int64_t i = 0; i < n; ++i) g->sigt_max = fmax(g->sigt_max, g->sigt[i]);
    g->trilinear = a->trilinear;
}

static int64_t grid_count(const grid_t *g)
{
    int64_t n = 1;
    for (int k = 0; k < g->dim; ++k) n *= g->nb[k];
    return n;
}

/* findBin.m:1-17: 0-based linear voxel index (x fastest) and the voxel's
 * bounds.  Subscripts outside 1..nb (a point on the lower face, or rounding)
 * are clamped; the reference would index out of range there. */
static int64_t find_bin(const grid_t *g, const double *x, double *bmn, double *bmx)
{
    int64_t ind = 0, stride = 1;
    for (int j = 0; j < g->dim; ++j) {
        double ii = ceil((x[j] - g->bmin[j]) / g->bbin[j]);
        if (ii < 1) ii = 1;
        if (ii > (double)g->nb[j]) ii = (double)g->nb[j];
        ind += (int64_t)(ii - 1) * stride;
        stride *= g->nb[j];
        if (bmn) {
            bmn[j] = g->bmin[j] + g->bbin[j] * (ii - 1);
            bmx[j] = bmn[j] + g->bbin[j];
        }
    }
    return ind;
}

static double grid_albedo(const grid_t *g, const double *x)
{
    return g->alb ? g->alb[find_bin(g, x, NULL, NULL)] : g->alb_scalar;
}

static int outside(const grid_t *g, const double *x)
{
    for (int k = 0; k < g->dim; ++k)
        if (x[k] > g->bmax[k] || x[k] < g->bmin[k]) return 1;
    return 0;
}

/* cubeDist.m:1-17 with the nudged exit point xd = x + (d + ep) v,
 * ep = 1e-4 max|vmax - vmin|. */
static double cube_dist_exit(const double *x, const double *vmin, const double *vmax, const double *v, int dim,
                             double *xd)
{
    double d = cube_dist(x, vmin, vmax, v, dim);
    double ep = 0.0;
    for (int k = 0; k < dim; ++k) ep = fmax(ep, fabs(vmax[k] - vmin[k]));
    ep = pow(0.1, 4) * ep;
    for (int k = 0; k < dim; ++k) xd[k] = x[k] + (d + ep) * v[k];
    return d;
}

/* Extension: sigma interpolated trilinearly between the voxel centres
 * bmin + (i + 1/2) bbin, clamped to the outer centres. */
static double sigma_tri(const grid_t *g, const double *x)
{
    int64_t i0[3] = {0, 0, 0};
    double f[3] = {0, 0, 0};
    for (int k = 0; k < g->dim; ++k) {
        double u = (x[k] - g->bmin[k]) / g->bbin[k] - 0.5;
        if (u < 0) u = 0;
        if (u > (double)(g->nb[k] - 1)) u = (double)(g->nb[k] - 1);
        int64_t i = (int64_t)floor(u);
        if (i > g->nb[k] - 2) i = g->nb[k] - 2;
        if (i < 0) i = 0;
        i0[k] = i;
        f[k] = g->nb[k] > 1 ? u - (double)i : 0.0;
    }
    double s = 0.0;
    for (int c = 0; c < (1 << g->dim); ++c) {
        int64_t idx = 0, stride = 1;
        double w = 1.0;
        for (int k = 0; k < g->dim; ++k) {
            int b = (c >> k) & 1;
            idx += ((g->nb[k] > 1) ? i0[k] + b : 0) * stride;
            stride *= g->nb[k];
            w *= b ? f[k] : 1.0 - f[k];
        }
        if (w != 0.0) s += w * g->sigt[idx];
    }
    return s;
}

/* Extension: the optical depth of the trilinear sigma from x along m over
 * min(nd, distance to the box), cut at every voxel-centre plane crossing;
 * sigma is a cubic in t on each piece and Simpson's rule is exact there. */
static double optical_depth_tri(const grid_t *g, const double *x, const double *m, double nd)
{
    const int dim = g->dim;
    double tend = INFINITY, tn[3], dt[3];
    for (int k = 0; k < dim; ++k) {
        if (m[k] > 0) tend = fmin(tend, (g->bmax[k] - x[k]) / m[k]);
        else if (m[k] < 0) tend = fmin(tend, (x[k] - g->bmin[k]) / -m[k]);
        double u = (x[k] - g->bmin[k]) / g->bbin[k] - 0.5;
        if (m[k] > 0) { tn[k] = (floor(u) + 1.0 - u) * g->bbin[k] / m[k]; dt[k] = g->bbin[k] / m[k]; }
        else if (m[k] < 0) { tn[k] = (u - (ceil(u) - 1.0)) * g->bbin[k] / -m[k]; dt[k] = g->bbin[k] / -m[k]; }
        else { tn[k] = INFINITY; dt[k] = INFINITY; }
    }
    tend = fmax(fmin(tend, nd), 0.0);
    double t0 = 0.0, s0 = sigma_tri(g, x), tau = 0.0, p[3] = {0, 0, 0};
    while (t0 < tend) {
        double t1 = tend;
        for (int k = 0; k < dim; ++k) t1 = fmin(t1, tn[k]);
        for (int k = 0; k < dim; ++k) if (tn[k] <= t1) tn[k] += dt[k];
        double tm = 0.5 * (t0 + t1);
        for (int k = 0; k < dim; ++k) p[k] = x[k] + tm * m[k];
        double sm = sigma_tri(g, p);
        for (int k = 0; k < dim; ++k) p[k] = x[k] + t1 * m[k];
        double s1 = sigma_tri(g, p);
        tau += (t1 - t0) / 6.0 * (s0 + 4.0 * sm + s1);
        t0 = t1;
        s0 = s1;
    }
    return tau;
}

/* evalphaseattHetro.m:1-52 for one direction / position. */
static cplx phaseatt_hetero(grid_t *g, const double *x, const double *v, int is_ff, double lambda)
{
    const int dim = g->dim;
    double pv, rv, nd, dir[3];
    if (is_ff) {
        pv = dotn(x, v, dim);
        rv = 1.0;
        nd = pow(10.0, 12);
        for (int k = 0; k < dim; ++k) dir[k] = v[k];
    } else {
        double d[3], s = 0.0;
        for (int k = 0; k < dim; ++k) { d[k] = x[k] - v[k]; s += d[k] * d[k]; }
        nd = sqrt(s);
        for (int k = 0; k < dim; ++k) dir[k] = d[k] / nd;
        pv = nd;
        rv = 1.0 / pow(nd + 0.01 * lambda, (dim - 1) / 2.0);
    }
    double m[3], nx[3], bmn[3], bmx[3];
    for (int k = 0; k < dim; ++k) { m[k] = -dir[k]; nx[k] = x[k]; }
    double bdv = 0.0, wbdv = 0.0;
    if (g->trilinear) {
        wbdv = optical_depth_tri(g, x, m, nd);
        double ph = (M_PI * 2.0 / lambda) * pv;
        return exp(-(1.0 / 2.0 * wbdv)) * (cos(ph) + I * sin(ph)) * rv;
    }
    for (int guard = 0; guard < 1000000; ++guard) {
        int64_t bi = find_bin(g, nx, bmn, bmx);
        double dd = cube_dist_exit(nx, bmn, bmx, m, dim, nx);
        bdv = bdv + dd;
        wbdv = wbdv + dd * g->sigt[bi];
        if (bdv >= nd) {
            double md = bdv - nd;
            bdv = nd;
            wbdv = wbdv - md * g->sigt[bi];
            break;
        }
        if (outside(g, nx)) break;
        if (guard == 999999) g->bad = 1;
    }
    double ph = (M_PI * 2.0 / lambda) * pv;
    return exp(-(1.0 / 2.0 * wbdv)) * (cos(ph) + I * sin(ph)) * rv;
}

/* smpWoodcock.m:1-15: delta tracking against max(sigt). */
static double smp_woodcock(grid_t *g, const double *x, const double *v, rng_t *r)
{
    double d = 0.0, nx[3];
    for (int guard = 0; guard < 100000000; ++guard) {
        d = d - log(1 - rand_u(r)) / g->sigt_max;
        for (int k = 0; k < g->dim; ++k) nx[k] = x[k] + d * v[k];
        if (outside(g, nx)) break;
        double sg = g->trilinear ? sigma_tri(g, nx) : g->sigt[find_bin(g, nx, NULL, NULL)];
        if (rand_u(r) <= (sg / g->sigt_max)) break;
        if (r->exhausted) break;
    }
    return d;
}

/* cubeProj.m:1-18.  Returns 0 and the entry point when d >= 0. */
static int cube_proj(const double *x, const double *vmin, const double *vmax, const double *v, int dim, double *xd)
{
    const double thr = pow(0.1, 7);
    double d = -INFINITY;
    for (int j = 0; j < dim; ++j) {
        double den = fmax(fabs(v[j]), thr);
        double bd = (v[j] <= 0) ? (x[j] - vmax[j]) / den : (-x[j] + vmin[j]) / den;
        d = fmax(d, bd);
    }
    if (d < 0) return -1;
    double ep = 0.0;
    for (int k = 0; k < dim; ++k) ep = fmax(ep, fabs(vmax[k] - vmin[k]));
    ep = pow(0.1, 4) * ep;
    for (int k = 0; k < dim; ++k) xd[k] = x[k] + (d + ep) * v[k];
    return 0;
}

/* expSmpXHetro.m:1-31.  `basis` is null(lmean') (dim x (dim-1), column-major). */
static int exp_smp_x_hetero(grid_t *g, const double *lmean, double lrad, const double *basis, double *x, double *px,
                            rng_t *r)
{
    const int dim = g->dim;
    double mx = 0.0;
    for (int k = 0; k < dim; ++k) mx = fmax(mx, fmax(fabs(g->bmax[k]), fabs(g->bmin[k])));
    double q[2];
    for (int k = 0; k < dim - 1; ++k) q[k] = (rand_u(r) - 0.5) * lrad;
    double x0[3];
    for (int k = 0; k < dim; ++k) {
        double s = 0.0;
        for (int c = 0; c < dim - 1; ++c) s += basis[k + dim * c] * q[c];
        x0[k] = s - lmean[k] * mx * dim;
    }
    if (cube_proj(x0, g->bmin, g->bmax, lmean, dim, x) != 0 || outside(g, x)) { *px = 0; return -1; }
    double d = smp_woodcock(g, x, lmean, r);
    for (int k = 0; k < dim; ++k) x[k] = x[k] + d * lmean[k];
    if (outside(g, x)) { *px = 0; return -1; }
    cplx e = phaseatt_hetero(g, x, lmean, 1, 1.0);
    double p = cabs(e) * cabs(e);
    *px = p / pow(lrad, dim - 1);
    return 0;
}

/* invCDFvec.m:1-7 = cumsum(hist(cdf, N)): N equal bins between min and max
 * of cdf, [e_k, e_k+1) with the last bin closed; smpicdf.m: icdf(ceil(rand*N)). */
static int64_t *inv_cdf_vec(const double *cdf, int64_t n, int64_t N)
{
    int64_t *h = calloc(N, sizeof(int64_t));
    double lo = cdf[0], hi = cdf[0];
    for (int64_t i = 0; i < n; ++i) { lo = fmin(lo, cdf[i]); hi = fmax(hi, cdf[i]); }
    double norm = (double)N / (hi - lo);
    for (int64_t i = 0; i < n; ++i) {
        int64_t b = (hi > lo) ? (int64_t)((cdf[i] - lo) * norm) : 0;
        if (b >= N) b = N - 1;
        /* keep the bin consistent with its edges lo + k (hi-lo)/N */
        double step = (hi - lo) / (double)N;
        if (b > 0 && cdf[i] < lo + b * step) b -= 1;
        if (b < N - 1 && cdf[i] >= lo + (b + 1) * step) b += 1;
        h[b]++;
    }
    for (int64_t i = 1; i < N; ++i) h[i] += h[i - 1];
    return h;
}

typedef struct {
    int cov;              /* 1: MCCovHetro, 0: MCsampleHetro */
    cplx *Ms, *Mm, *mean1, *u;
    int threads;
} hsink_t;

static int hetero_walk(const scmc_hetero_args *a, oracle_rng_spec *rs, hsink_t *sk)
{
    const scmc_mc_args *mc = &a->mc;
    const int dim = mc->dim;
    const int nv = (int)mc->nv, nl = (int)mc->nl;
    grid_t g;
    grid_init(&g, a);
    rng_t r;
    rng_init(&r, rs, mc->seed);
    nee_t c;
    nee_alloc(&c, mc); /* directions, far-field amplitude table, unmeanl (lmean0 honoured) */
    if (sk->cov) {     /* MCCovHetro.m:38: always mean(l,2) */
        for (int k = 0; k < dim; ++k) {
            double s = 0.0;
            for (int j = 0; j < nl; ++j) s += mc->l[dim * j + k];
            c.unmeanl[k] = s / nl;
        }
        double n = sqrt(dotn(c.unmeanl, c.unmeanl, dim));
        for (int k = 0; k < dim; ++k) c.meanl[k] = c.unmeanl[k] / n;
    }
    const int64_t ng = grid_count(&g);
    double ssum = 0.0;
    for (int64_t i = 0; i < ng; ++i) ssum += g.sigt[i];
    double *cdf = malloc(sizeof(double) * ng);
    double acc = 0.0;
    for (int64_t i = 0; i < ng; ++i) { acc += g.sigt[i] / ssum; cdf[i] = acc; }
    const int64_t Nicdf = ng * 100;
    int64_t *icdf = inv_cdf_vec(cdf, ng, Nicdf);
    free(cdf);
    double vb = 1.0;
    for (int k = 0; k < dim; ++k) vb *= g.bbin[k];
    const double V = ssum * vb; /* MCCovHetro.m:64 */
    double lrad = 0.0;
    for (int k = 0; k < dim; ++k) lrad += (g.bmax[k] - g.bmin[k]) * (g.bmax[k] - g.bmin[k]);
    lrad = a->has_lrad ? a->lrad : sqrt(lrad);
    cplx *ul0 = malloc(sizeof(cplx) * nl);
    int rc = 0;
    for (int64_t itr = 0; itr < mc->max_itr; ++itr) {
        if (r.mode == ORACLE_RNG_PHILOX) rng_set_path(&r, mc->path_offset + (uint64_t)itr);
        double x[3] = {0, 0, 0}, w[3] = {0, 0, 0}, ow[3] = {0, 0, 0}, px;
        if (mc->smp_flg == 1) {
            /* smpicdf.m + MCCovHetro.m:93-95 */
            int64_t i = (int64_t)ceil(rand_u(&r) * (double)Nicdf);
            if (i < 1) i = 1;
            int64_t bin = icdf[i - 1] - 1; /* 1-based voxel index -> 0-based */
            int64_t rem = bin;
            for (int k = 0; k < dim; ++k) {
                int64_t ii = rem % g.nb[k];
                rem /= g.nb[k];
                double bmn = g.bmin[k] + g.bbin[k] * (double)ii;
                x[k] = rand_u(&r) * g.bbin[k] + bmn;
            }
            px = 1.0 / V;
            /* extension: voxel pick density sigma_nearest / V, medium sigma_trilinear */
            if (g.trilinear) px = g.sigt[find_bin(&g, x, NULL, NULL)] / (V * sigma_tri(&g, x));
        } else {
            if (exp_smp_x_hetero(&g, c.meanl, lrad, a->null_basis, x, &px, &r) != 0) {
                if (r.exhausted) { rc = -1; break; }
                continue; /* MCCovHetro.m:113-115 */
            }
        }
        if (outside(&g, x)) continue;
        double x1[3], w1[3];
        memcpy(x1, x, sizeof x);
        if (!mc->has_ampfunc0) randn_dir(dim, w, &r);
        else smpampfunc_general(c.meanl, &mc->ampfunc0, dim, w, &r);
        memcpy(w1, w, sizeof w);
        /* per-path vectors with the voxel-marched attenuation */
        if (!c.is_ff_v)
            for (int i = 0; i < nv; ++i) {
                double d[3], s = 0.0;
                for (int k = 0; k < dim; ++k) { d[k] = c.v[dim * i + k] - x[k]; s += d[k] * d[k]; }
                s = sqrt(s);
                for (int k = 0; k < dim; ++k) c.rv[dim * i + k] = d[k] / s;
            }
        if (!c.is_ff_l)
            for (int j = 0; j < nl; ++j) {
                double d[3], s = 0.0;
                for (int k = 0; k < dim; ++k) { d[k] = x[k] - c.l[dim * j + k]; s += d[k] * d[k]; }
                s = sqrt(s);
                for (int k = 0; k < dim; ++k) c.rl[dim * j + k] = d[k] / s;
            }
        if (!(c.is_ff_v && c.is_ff_l))
            for (int j = 0; j < nl; ++j)
                for (int i = 0; i < nv; ++i)
                    c.af_vl[i + nv * j] = evalampfunc(dotn(c.rl + dim * j, c.rv + dim * i, dim), c.pf, dim);
        c.w0p = !c.has_pf0 ? 1.0 / sqrt(pow(2.0, dim - 1) * M_PI) : creal(evalampfunc(dotn(c.meanl, w, dim), c.pf0, dim));
        for (int j = 0; j < nl; ++j) {
            cplx af_l = evalampfunc(dotn(w, c.rl + dim * j, dim), c.pf, dim) / c.w0p;
            c.e_l0[j] = phaseatt_hetero(&g, x, c.l + dim * j, c.is_ff_l, mc->lambda);
            c.e_l0_ms[j] = c.e_l0[j] * af_l;
            if (sk->cov) ul0[j] = evalphaseatt1(x, c.l + dim * j, c.is_ff_l, 0.0, mc->lambda, c.bmin, c.bmax, dim);
        }
        for (int i = 0; i < nv; ++i) {
            c.e_v0[i] = phaseatt_hetero(&g, x, c.vs + dim * i, c.is_ff_v, mc->lambda);
            if (c.cbs) {
                cplx af_v = evalampfunc(-dotn(w, c.rv + dim * i, dim), c.pf, dim) / c.w0p;
                c.e_v0_ms[i] = c.e_v0[i] * af_v;
            }
        }
        int pL = 0;
        double weight = grid_albedo(&g, x);
        for (;;) {
            ++pL;
            if (pL > 1) {
                for (int i = 0; i < nv; ++i) {
                    cplx e_v = phaseatt_hetero(&g, x, c.vs + dim * i, c.is_ff_v, mc->lambda);
                    c.e_v_ms[i] = e_v * evalampfunc(dotn(ow, c.rv + dim * i, dim), c.pf, dim);
                }
                if (c.cbs)
                    for (int j = 0; j < nl; ++j) {
                        cplx e_l = phaseatt_hetero(&g, x, c.l + dim * j, c.is_ff_l, mc->lambda);
                        c.e_l_ms[j] = e_l * evalampfunc(-dotn(ow, c.rl + dim * j, dim), c.pf, dim);
                    }
            }
            const double wpx = weight / px;
            if (sk->cov) {
                if (pL == 1)
                    for (int j = 0; j < nl; ++j)
                        for (int i = 0; i < nv; ++i)
                            sk->mean1[i + nv * j] += wpx * c.af_vl[i + nv * j] * (c.e_v0[i] * ul0[j]);
                cov_update(&c, pL, wpx, sk->Ms, sk->Mm, sk->threads);
            } else {
                double xi = rand_u(&r); /* MCsampleHetro.m:187, after the NEE */
                field_update(&c, pL, wpx, xi, sk->u);
            }
            double d = smp_woodcock(&g, x, w, &r);
            for (int k = 0; k < dim; ++k) x[k] = x[k] + d * w[k];
            if (outside(&g, x)) break;
            if (weight < KILL_THR) {
                if (rand_u(&r) > grid_albedo(&g, x)) break;
            } else {
                weight = weight * grid_albedo(&g, x);
            }
            memcpy(ow, w, sizeof w);
            smpampfunc_general(ow, &mc->ampfunc, dim, w, &r);
            if (r.exhausted) break;
        }
        if (r.exhausted) { rc = -1; break; }
    }
    if (g.bad) rc = -5;
    rs->used_u = r.ui;
    rs->used_n = r.ni;
    free(icdf);
    free(ul0);
    nee_free(&c);
    return rc;
}

int oracle_cov_hetero(const scmc_hetero_args *a, oracle_rng_spec *rs, double *Ms, double *Mm, double *mean1,
                      int threads)
{
    const scmc_mc_args *mc = &a->mc;
    int64_t n = mc->nv * mc->nv * mc->nl * mc->nl;
    memset(Ms, 0, sizeof(double) * 2 * n);
    memset(Mm, 0, sizeof(double) * 2 * n);
    memset(mean1, 0, sizeof(double) * 2 * mc->nv * mc->nl);
    hsink_t sk = {1, (cplx *)Ms, (cplx *)Mm, (cplx *)mean1, NULL, threads};
    int rc = hetero_walk(a, rs, &sk);
    /* MCCovHetro.m:262-276: CBS /2, then /maxItr only (px carries the volume) */
    double m = (double)(mc->norm_itr > 0 ? mc->norm_itr : mc->max_itr);
    for (int64_t i = 0; i < n; ++i) {
        if (mc->do_cbs) sk.Mm[i] = sk.Mm[i] / 2.0;
        sk.Mm[i] = sk.Mm[i] / m;
        sk.Ms[i] = sk.Ms[i] / m;
    }
    /* cs = 1 (for tabulated tables the reference reads a missing field) */
    for (int64_t i = 0; i < mc->nv * mc->nl; ++i) sk.mean1[i] = sk.mean1[i] / m / sqrt(1.0);
    return rc;
}

int oracle_field_hetero(const scmc_hetero_args *a, oracle_rng_spec *rs, double *u)
{
    const scmc_mc_args *mc = &a->mc;
    memset(u, 0, sizeof(double) * 2 * mc->nv * mc->nl);
    hsink_t sk = {0, NULL, NULL, NULL, (cplx *)u, 1};
    int rc = hetero_walk(a, rs, &sk);
    double m = (double)(mc->norm_itr > 0 ? mc->norm_itr : mc->max_itr);
    double f = sqrt(1.0 / m); /* MCsampleHetro.m:222 */
    for (int64_t i = 0; i < mc->nv * mc->nl; ++i) sk.u[i] *= f;
    return rc;
}
