/*
 * fourier_quad.c - CPU FP64 restatement of MCfieldFourierQuad.m (the file
 * declares `function MCfield`; MATLAB dispatches it by file name).
 *
 * TEST INFRASTRUCTURE ONLY (the oracle; never linked into the product).
 *
 * MCfieldFourierQuad.m:77-303: an isotropic walk that records every vertex
 * (x, first scatterer x1, sqrt(w/px) e^{2 pi i xi} [/sqrt2 for CBS, pL>1]),
 * vertices sorted by the depth of x1 and grouped into z planes; per plane and
 * light the contributions are gridded on the lateral pixel grid at x1, padded,
 * transformed with fftshift(fft2(ifftshift(.))), flipped, cropped, multiplied
 * by exp(zexp0 * tz) and summed; finally multiplied by boxexp0 and normalised
 * by the VERTEX count (line 214).
 *
 * Extensions (flagged in scmc_fq_args, not in the reference): HG(g) direction
 * sampling in the walk (the smpampfunc_general call commented out at line
 * 208; the first direction stays isotropic as at line 171, and the NEE terms
 * keep the reference's isotropic couplings, because a view-side amplitude
 * would depend on the output direction and could not be a per-vertex factor),
 * and point sources: the light factor of line 272 replaced by the near-field
 * branch of evalphaseatt.m:10-16.
 *
 * The 2-D FFT is restated as the centred DFT it computes:
 *   X[q] = sum_p x[p] exp(-2 pi i (q - c)(p - c) / M),  c = floor(M/2),
 * followed by the flip q -> M-1-q and the crop of Nva_padd_size rows and
 * columns on each side.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "scmc_oracle.h"

typedef double _Complex cplx;

/* The walk and RNG live in scmc_oracle.c; this file reuses them through a
 * narrow internal interface. */
cplx oracle_internal_evalphaseatt1(const double *x, const double *v, int is_ff, double sigt,
                                   double lambda, const double *bmin, const double *bmax, int dim);
int oracle_internal_fq_walk(const scmc_fq_args *a, const double *bmin, const double *bmax,
                            const double *unmeanl, oracle_rng_spec *rs, int64_t cap,
                            double *xL, double *x1L, double *pxr, double *pxi, int64_t *n_vert);

/* MATLAB's a:s:b element count (small tolerance on (b-a)/s). */
static int64_t colon_count(double a, double s, double b)
{
    if (s == 0 || (s > 0 && a > b) || (s < 0 && a < b)) return 0;
    double q = (b - a) / s;
    return (int64_t)floor(q + 1e-10 * fmax(1.0, fabs(q))) + 1;
}

static double mround(double x) { return x < 0 ? -floor(-x + 0.5) : floor(x + 0.5); }

typedef struct {
    int64_t i;
    double key;
} sort_item;

static int cmp_item(const void *p, const void *q)
{
    const sort_item *a = p, *b = q;
    if (a->key < b->key) return -1;
    if (a->key > b->key) return 1;
    return (a->i < b->i) ? -1 : (a->i > b->i); /* stable, as MATLAB's sort */
}

/* Wl == NULL: MCfieldFourierQuad.m.  Wl != NULL: MCfieldFourierQuadOnWave.m,
 * which differs in four places: the lateral pixel count is made to have the
 * parity of the angular grid (lines 97-99), zexp0 has the opposite phase sign
 * (line 140), the light term is twl = sum_j Wl_j exp(vsign 2 pi i/lambda
 * l_j.x) times the slab attenuation atl (lines 278-295; see the note on
 * which vertex twl reads), and the vertex
 * phase is exp(vsign 2 pi i/lambda (-z1 + tz)) (line 302); the lights are
 * summed into one output. */
static int fq_core(const scmc_fq_args *a, const cplx *Wl, int as_written, oracle_rng_spec *rs, double *u_out)
{
    const double lambda = a->lambda, sigt = a->sigt;
    const double PI = M_PI;
    double bmin[3], bmax[3], bw[3];
    for (int k = 0; k < 3; ++k) {
        bmin[k] = a->box_min[k];
        bmax[k] = a->box_max[k];
        bw[k] = bmax[k] - bmin[k];
    }
    /* MCfieldFourierQuad.m:59-64 */
    double unmeanl[3] = {0, 0, 1};
    if (a->has_lmean0) memcpy(unmeanl, a->lmean0, sizeof unmeanl);
    const double vsign = a->vsign;
    /* lines 80-89 */
    const double v_max = a->v_max, v_stp = a->v_stp;
    const int64_t Nv = colon_count(-v_max, v_stp, v_max);
    double *theta_v = malloc(sizeof(double) * Nv);
    for (int64_t k = 0; k < Nv; ++k) theta_v[k] = -v_max + (double)k * v_stp;
    /* lines 92-98: lateral pitch and the box padded to an odd pixel count */
    const double box_stp = lambda / (v_max * 2 + v_stp);
    int64_t Nx = (int64_t)ceil(bw[0] / box_stp / 2) * 2 + 1;
    if (Wl && (((Nv - Nx) % 2) + 2) % 2 == 1) Nx = Nx + 1; /* OnWave: mod(Nv - Nx, 2) == 1 */
    const double box_w_n = Nx * box_stp;
    const double grow = (box_w_n - bw[0]) / 2; /* box_w(1) for both x and y, as line 96-97 */
    for (int k = 0; k < 2; ++k) {
        bmin[k] = bmin[k] - grow;
        bmax[k] = bmax[k] + grow;
        bw[k] = box_w_n;
    }
    const double gx1 = bmin[0] + box_stp / 2, gy1 = bmin[1] + box_stp / 2;
    /* lines 103-106.  The reference needs integer padding sizes (padarray,
     * subscripts); with an even grid length they are half-integers and it
     * stops.  The same centred-DFT formula below is then evaluated with the
     * half-integer offsets (this build's extension; unpinned). */
    const double nx_pad = fmax((double)(Nv - Nx) / 2, 0.0);
    const double nv_pad = fmax((double)(Nx - Nv) / 2, 0.0);
    const double M = (double)Nx + 2 * nx_pad;
    /* lines 108-113: vx, vy = ndgrid(-theta_v, -theta_v), vz (complex outside the disk) */
    cplx *vz = malloc(sizeof(cplx) * Nv * Nv);
    double maxdiff = -INFINITY;
    for (int64_t j = 0; j < Nv; ++j)
        for (int64_t i = 0; i < Nv; ++i) {
            double vx = -theta_v[i], vy = -theta_v[j];
            double r = 1 - vx * vx - vy * vy;
            cplx s = r >= 0 ? sqrt(r) : I * sqrt(-r);
            vz[i + Nv * j] = vsign * s;
            maxdiff = fmax(maxdiff, 1 - cabs(vz[i + Nv * j]));
        }
    /* lines 116-121: z planes */
    double z_bin = lambda / maxdiff / 5;
    z_bin = z_bin / 2;
    int64_t ng = colon_count(bmin[2], z_bin, bmax[2]);
    int64_t Nz = ng + 1;
    double *gz = malloc(sizeof(double) * Nz);
    for (int64_t k = 0; k < ng; ++k) gz[k] = bmin[2] + (double)k * z_bin;
    gz[ng] = bmax[2];
    /* lines 124-138 */
    cplx *zexp0 = malloc(sizeof(cplx) * Nv * Nv), *boxexp0 = malloc(sizeof(cplx) * Nv * Nv);
    for (int64_t q = 0; q < Nv * Nv; ++q) {
        cplx z = vz[q];
        double av = cabs(z);
        double diratt = (creal(z) < 0) ? 1.0 / av : 0.0;
        double idiratt = (creal(z) > 0) ? 1.0 / av : 0.0;
        if (Wl) zexp0[q] = (2 * PI * I / lambda) * z * vsign - sigt / 2 * (diratt - idiratt);
        else zexp0[q] = (-2 * PI * I / lambda) * z * vsign - sigt / 2 * (diratt - idiratt);
        cplx b1 = cexp(-sigt / 2 * (-bmin[2] * diratt + bmax[2] * idiratt));
        cplx ph = (-bmin[2] * (creal(z) < 0) * z + bmax[2] * (creal(z) > 0) * z);
        boxexp0[q] = b1 * cexp(2 * PI * I / lambda * ph);
    }
    const double l_end = a->l[3 * (a->nl - 1) + 2];
    const double l_diratt = (l_end > 0) ? 1.0 / fabs(l_end) : 0.0;
    const double l_idiratt = (l_end < 0) ? 1.0 / fabs(l_end) : 0.0;

    /* lines 146-218: the walk, every vertex recorded */
    const double ExpOD = sigt * bw[2] + 1;
    int64_t cap = (int64_t)(a->max_itr * ExpOD * 4 + 1024);
    double *xL = malloc(sizeof(double) * 3 * cap), *x1L = malloc(sizeof(double) * 3 * cap);
    double *pr = malloc(sizeof(double) * cap), *pi_ = malloc(sizeof(double) * cap);
    int64_t nvert = 0;
    int rc;
    for (;;) {
        rc = oracle_internal_fq_walk(a, bmin, bmax, unmeanl, rs, cap, xL, x1L, pr, pi_, &nvert);
        if (rc != -2) break;
        cap *= 4;
        xL = realloc(xL, sizeof(double) * 3 * cap);
        x1L = realloc(x1L, sizeof(double) * 3 * cap);
        pr = realloc(pr, sizeof(double) * cap);
        pi_ = realloc(pi_, sizeof(double) * cap);
    }
    const int64_t nl = a->nl;
    const int64_t nout = Wl ? 1 : nl; /* output planes */
    cplx *u = calloc(Nv * Nv * nout, sizeof(cplx));
    if (rc == 0) {
        /* twiddles exp(-2 pi i m' P / M) for the centred, flipped, cropped DFT:
         * output r is FFT bin q = r + Nva_padd, flipped to M-1-q, centred by
         * c = floor(M/2); pixel p sits at padded index p + Nx_padd. */
        const double c = floor(M / 2);
        cplx *tw = malloc(sizeof(cplx) * Nv * Nx);  /* [r][pixel] */
        for (int64_t r = 0; r < Nv; ++r) {
            double q = (double)r + nv_pad;
            double m = (M - 1 - q) - c;
            for (int64_t p = 0; p < Nx; ++p) {
                double P = ((double)p + nx_pad) - c;
                double t = fmod(m * P, M);
                double ang = -2 * PI * t / M;
                tw[r * Nx + p] = cos(ang) + I * sin(ang);
            }
        }
        sort_item *it = malloc(sizeof(sort_item) * (nvert > 0 ? nvert : 1));
        double *sx = malloc(sizeof(double) * 3 * (nvert + 1)), *sx1 = malloc(sizeof(double) * 3 * (nvert + 1));
        cplx *sp = malloc(sizeof(cplx) * (nvert + 1));
        cplx *acc = malloc(sizeof(cplx) * Nv * Nv);
        for (int tt = 1; tt <= 2; ++tt) {
            if (tt == 2 && !a->do_cbs) continue;
            /* tt == 2: swap the roles of x and x1 (line 226-232) */
            const double *X = tt == 1 ? xL : x1L, *X1 = tt == 1 ? x1L : xL;
            for (int64_t e = 0; e < nvert; ++e) { it[e].i = e; it[e].key = X1[3 * e + 2]; }
            qsort(it, nvert, sizeof(sort_item), cmp_item);
            for (int64_t e = 0; e < nvert; ++e) {
                int64_t o = it[e].i;
                for (int k = 0; k < 3; ++k) { sx[3 * e + k] = X[3 * o + k]; sx1[3 * e + k] = X1[3 * o + k]; }
                sp[e] = pr[o] + I * pi_[o];
            }
            /* lines 242-286 */
            int64_t zmax_ind = 0; /* 1-based z_ind_max */
            for (int64_t j1 = 1; j1 <= Nz - 1; ++j1) {
                int64_t citr = zmax_ind + 1;
                double z_max = gz[j1];
                while (citr <= nvert && sx1[3 * (citr - 1) + 2] < z_max) citr++;
                int64_t zmin_ind = zmax_ind + 1;
                zmax_ind = citr - 1;
                if (zmax_ind < zmin_ind) continue;
                double tz = (gz[j1 - 1] + gz[j1]) / 2;
                for (int64_t j2 = 0; j2 < nout; ++j2) {
                    const double *lj = a->l + 3 * j2;
                    memset(acc, 0, sizeof(cplx) * Nv * Nv);
                    for (int64_t e = zmin_ind - 1; e < zmax_ind; ++e) {
                        const double *xe = sx + 3 * e, *x1e = sx1 + 3 * e;
                        int64_t p1 = (int64_t)mround((x1e[0] - gx1) / box_stp) + 1;
                        int64_t p2 = (int64_t)mround((x1e[1] - gy1) / box_stp) + 1;
                        if (p1 < 1) p1 = 1;
                        if (p1 > Nx) p1 = Nx;
                        if (p2 < 1) p2 = 1;
                        if (p2 > Nx) p2 = Nx;
                        cplx w;
                        if (Wl) {
                            /* lines 282-292 evaluate twl at xL(:, 1:numel(jj)): the plane's
                             * j3-th weight comes from the j3-th vertex of the whole
                             * depth-sorted list, not from the plane's own vertex jj(j3).
                             * as_written = 1 keeps that; 0 uses the plane's own vertex,
                             * the formula of the commented-out line 279 (and of
                             * MCfieldFourierQuad), which the GPU computes. */
                            const double *xt = as_written ? sx + 3 * (e - (zmin_ind - 1)) : xe;
                            cplx twl = 0.0;
                            for (int64_t j = 0; j < nl; ++j) {
                                const double *l = a->l + 3 * j;
                                twl += Wl[j] * cexp(vsign * 2 * PI * I / lambda * (l[0] * xt[0] + l[1] * xt[1] + l[2] * xt[2]));
                            }
                            const double atl =
                                exp(-sigt / 2 * ((xe[2] - bmin[2]) * l_diratt + (bmax[2] - xe[2]) * l_idiratt));
                            w = sp[e] * cexp(vsign * 2 * PI * I / lambda * (-x1e[2] + tz)) * twl * atl;
                        } else if (a->light_point) {
                            /* extension: a point source at l_j, the near-field term of
                             * evalphaseatt.m:10-16 (cubeDist in the padded box the walk uses) */
                            w = sp[e] * cexp(-2 * PI * I / lambda * (-x1e[2] + tz)) *
                                oracle_internal_evalphaseatt1(xe, lj, 0, sigt, lambda, bmin, bmax, 3);
                        } else {
                            w = sp[e] * cexp(-2 * PI * I / lambda * (-x1e[2] + tz)) *
                                cexp(2 * PI * I / lambda * (lj[0] * xe[0] + lj[1] * xe[1] + lj[2] * xe[2]) -
                                     sigt / 2 * ((xe[2] - bmin[2]) * l_diratt + (bmax[2] - xe[2]) * l_idiratt));
                        }
                        for (int64_t r2 = 0; r2 < Nv; ++r2) {
                            cplx w2 = w * tw[r2 * Nx + (p2 - 1)];
                            for (int64_t r1 = 0; r1 < Nv; ++r1) acc[r1 + Nv * r2] += w2 * tw[r1 * Nx + (p1 - 1)];
                        }
                    }
                    cplx *uj = u + Nv * Nv * j2;
                    for (int64_t q = 0; q < Nv * Nv; ++q) uj[q] += acc[q] * cexp(zexp0[q] * tz);
                }
            }
        }
        free(tw); free(it); free(sx); free(sx1); free(sp); free(acc);
        /* lines 291-303 */
        double V = bw[0] * bw[1] * bw[2];
        double f = sqrt(1.0 / (double)nvert * V * sigt);
        for (int64_t j2 = 0; j2 < nout; ++j2)
            for (int64_t q = 0; q < Nv * Nv; ++q) u[Nv * Nv * j2 + q] = u[Nv * Nv * j2 + q] * boxexp0[q] * f;
        memcpy(u_out, u, sizeof(cplx) * Nv * Nv * nout);
    }
    free(u); free(xL); free(x1L); free(pr); free(pi_);
    free(theta_v); free(vz); free(gz); free(zexp0); free(boxexp0);
    return rc;
}

int oracle_field_fourier_quad(const scmc_fq_args *a, oracle_rng_spec *rs, double *u_out)
{
    return fq_core(a, NULL, 0, rs, u_out);
}

int oracle_field_fourier_quad_onwave(const scmc_fq_args *a, const double *Wl, int32_t as_written,
                                     oracle_rng_spec *rs, double *u_out)
{
    return fq_core(a, (const cplx *)Wl, as_written, rs, u_out);
}
