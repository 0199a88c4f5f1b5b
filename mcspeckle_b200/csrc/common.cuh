// common.cuh - shared device code of the SCMC Monte Carlo path on sm_100a.
//
// Philox-4x32-10 streams (one counter-based stream pair per path, so any path
// can be regenerated from (seed, path index)), and FP64 restatements of the
// reference's coreFunctions used by the walk and by next-event estimation.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#ifndef SCMC_PI
#define SCMC_PI 3.141592653589793238462643383279502884
#endif

namespace scmc {

constexpr double kKillThr = 0.2;  // MCfield.m:109, MCcov.m:110

// ---------------------------------------------------------------------------
// Phase functions as the device sees them (scmc_phase_function with device
// copies of the tables).
// ---------------------------------------------------------------------------
struct PhaseFn {
    int sct_type;        // 1 iso, 2 tabulated, 3 HG
    double g;
    int table_n;
    const double2 *eval_amp;   // table_n complex (evalAmp)
    const double *sample_icdf; // table_n angles (sampleIcdf), or cosines with cos_bins
    int cos_bins;              // tables on cos(theta) bins (extension) instead of angle bins
};

// Voxel medium of MCCovHetro.m / MCsampleHetro.m (device functions in hgrid.cuh).
struct HGrid {
    int dim;
    const double *sigt;      // prod(nb) values, x fastest (findBin.m order)
    const double *alb;       // prod(nb) albedos or nullptr
    double alb_scalar;
    double bmin[3], bmax[3], bbin[3];
    double ibbin[3];         // 1 / bbin (the attenuation march)
    int nb[3];
    double sigt_max;
    // first-scatter sampling
    const double *cdf;       // cumsum(sigt / sum(sigt)), prod(nb) values (MCCovHetro.m:62)
    int64_t n_vox;
    int64_t n_icdf;          // prod(nb) * 100 (MCCovHetro.m:63)
    double cdf_lo, cdf_step; // hist bins of invCDFvec.m
    double inv_V;            // px = 1/V, V = sum(sigt) prod(box_bin)
    double lrad;
    double basis[6];         // null(meanl'), dim x (dim-1) column-major
    int trilinear;           // extension: sigt trilinear between voxel centres
    const float *sigt_f;     // FP32 copy of sigt for the reduced-precision NEE march (trilinear), or nullptr
};

// Everything the walk needs, passed by value.
struct WalkParams {
    int dim;
    int smp_flg;
    int has_pf0;
    int want_phase;            // MCfield draws a random phase per event
    double sigt, albedo;
    double box_min[3], box_max[3], box_w[3];
    double unmeanl[3], meanl[3];
    PhaseFn pf, pf0;
    uint32_t key0, key1;
    uint64_t path_base;        // global index of path 0 of this batch
    int64_t n_paths;
    int64_t max_events;        // 0 = unlimited
    int hetero;                // voxel medium (Woodcock flights, voxel albedo)
    HGrid hg;
    int any_order;             // records may be written in any order (one-pass walk); 0 keeps path order
};

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).
// ---------------------------------------------------------------------------
__host__ __device__ inline void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t out[4])
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// 52 random bits -> double strictly inside (0,1), exactly representable.
__host__ __device__ inline double u52_to_unit(uint32_t a, uint32_t b)
{
    uint64_t m = ((uint64_t)a << 20) | (uint64_t)(b >> 12);
    return ((double)m + 0.5) * 0x1p-52;
}

// The two streams of one path: tag 0 feeds MATLAB's rand, tag 1 randn
// (Box-Muller pairs).  Counter = (block, tag, path_lo, path_hi).
struct PathRng {
    uint32_t k0, k1, plo, phi;
    uint32_t uctr, nctr;
    double ub0, ub1, nb0, nb1;
    int uh, nh;

    __host__ __device__ void init(uint32_t key0, uint32_t key1, uint64_t path)
    {
        k0 = key0; k1 = key1;
        plo = (uint32_t)path; phi = (uint32_t)(path >> 32);
        uctr = nctr = 0;
        uh = nh = 0;
        ub0 = ub1 = nb0 = nb1 = 0.0;
    }
    __host__ __device__ double rand()
    {
        if (uh == 0) {
            uint32_t o[4];
            philox4x32_10(uctr++, 0u, plo, phi, k0, k1, o);
            ub0 = u52_to_unit(o[0], o[1]);
            ub1 = u52_to_unit(o[2], o[3]);
            uh = 2;
            return ub0;
        }
        uh = 0;
        return ub1;
    }
    __host__ __device__ double randn()
    {
        if (nh == 0) {
            uint32_t o[4];
            philox4x32_10(nctr++, 1u, plo, phi, k0, k1, o);
            double u1 = u52_to_unit(o[0], o[1]);
            double u2 = u52_to_unit(o[2], o[3]);
            double rad = sqrt(-2.0 * log(u1));
            double ang = (2.0 * SCMC_PI) * u2;
            nb0 = rad * cos(ang);
            nb1 = rad * sin(ang);
            nh = 2;
            return nb0;
        }
        nh = 0;
        return nb1;
    }
};

// MATLAB round(): half away from zero.
__device__ __forceinline__ double mround(double x)
{
    return x < 0 ? -floor(-x + 0.5) : floor(x + 0.5);
}

// ---------------------------------------------------------------------------
// coreFunctions in FP64
// ---------------------------------------------------------------------------

// cubeDist.m:1-11 - distance from x along direction v to the box boundary.
template <int DIM>
__device__ __forceinline__ double cube_dist(const double *x, const double *bmin, const double *bmax,
                                            const double *v)
{
    const double thr = 1.0000000000000004e-07;  // 0.1^7 as MATLAB evaluates it
    double d = INFINITY;
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
        double den = fmax(fabs(v[j]), thr);
        double bd = (v[j] <= 0) ? (x[j] - bmin[j]) / den : (-x[j] + bmax[j]) / den;
        d = fmin(d, bd);
    }
    return d;
}

// evaluateHG.m:25-39 with cosineFlag = 1.
template <int DIM>
__device__ __forceinline__ double evaluate_hg(double c, double g)
{
    double den = 1.0 + (g * g + (-2.0 * (g * c)));
    if (DIM == 3) return (1.0 / 4.0 / SCMC_PI) * ((1.0 - g * g) / pow(den, 1.5));
    return (1.0 / 2.0 / SCMC_PI) * ((1.0 - g * g) / den);
}

// Nearest entry of a table on cos(theta) bins cos_i = 1 - 2i/(n-1) (the
// extension; evaluated in FP64 in every precision mode so all modes read the
// same entry).
__device__ __forceinline__ int tab_cos_index(double cc, int n)
{
    long long idx = (long long)mround((1.0 - cc) * 0.5 * (double)(n - 1));
    return (int)(idx < 0 ? 0 : (idx > n - 1 ? n - 1 : idx));
}

// evalampfunc_general.m:1-19 / evalampfunc_amplitude.m:1-9.
template <int DIM>
__device__ __forceinline__ double2 evalampfunc(double c, const PhaseFn &pf)
{
    if (pf.sct_type == 1) {
        return make_double2(1.0 / sqrt((DIM == 3 ? 4.0 : 2.0) * SCMC_PI), 0.0);
    }
    if (pf.sct_type == 2) {
        double cc = fmin(fmax(c, -1.0), 1.0);
        if (pf.cos_bins) return pf.eval_amp[tab_cos_index(cc, pf.table_n)];
        double ang = acos(cc);
        double span = (DIM == 2) ? 2.0 * SCMC_PI : SCMC_PI;
        long long idx = (long long)mround(ang * (double)(pf.table_n - 1) / span);
        idx = idx < 0 ? 0 : (idx > pf.table_n - 1 ? pf.table_n - 1 : idx);
        return pf.eval_amp[idx];
    }
    return make_double2(sqrt(evaluate_hg<DIM>(c, pf.g)), 0.0);
}

// sampleHG.m:1-18
template <int DIM>
__device__ __forceinline__ double sample_hg(double g, PathRng &r)
{
    if (fabs(g) < 0.001) return 2.0 * r.rand() - 1.0;
    if (DIM == 3) {
        double t = (1.0 - g * g) / (1.0 - g + 2.0 * g * r.rand());
        return (1.0 / (2.0 * g)) * ((1.0 + g * g) - t * t);
    }
    double th = 2.0 * atan((1.0 - g) / (1.0 + g) * tan(SCMC_PI / 2.0 * (1.0 - 2.0 * r.rand())));
    return cos(th);
}

// rotateBytheta.m:1-28
template <int DIM>
__device__ __forceinline__ void rotate_by_theta(const double *ow, double c, double *w, PathRng &r)
{
    double s = 1.0 - c * c;
    s = s > 0 ? sqrt(s) : 0.0;
    if (DIM == 2) {
        s = ((r.rand() > 0.5) * 2.0 - 1.0) * s;
        double w0 = c * ow[0] + s * ow[1];
        double w1 = -s * ow[0] + c * ow[1];
        w[0] = w0; w[1] = w1;
        return;
    }
    double phi = SCMC_PI * 2.0 * r.rand();
    double sp, cp;
    sincos(phi, &sp, &cp);
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

template <int DIM>
__device__ __forceinline__ void randn_dir(double *w, PathRng &r)
{
    double n2 = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) { w[k] = r.randn(); n2 += w[k] * w[k]; }
    double nrm = sqrt(n2);
#pragma unroll
    for (int k = 0; k < DIM; ++k) w[k] = w[k] / nrm;
}

// smpampfunc_general.m:1-21 (smpampfunc.m:1-8 for tables).
template <int DIM>
__device__ __forceinline__ void smpampfunc_general(const double *ow, const PhaseFn &pf, double *w, PathRng &r)
{
    if (pf.sct_type == 1) { randn_dir<DIM>(w, r); return; }
    double c;
    if (pf.sct_type == 2) {
        double stp = 1.0 / (double)(pf.table_n - 1);
        long long i = (long long)mround(r.rand() / stp);
        i = i > pf.table_n - 1 ? pf.table_n - 1 : i;
        c = pf.cos_bins ? pf.sample_icdf[i] : cos(pf.sample_icdf[i]);
    } else {
        c = sample_hg<DIM>(pf.g, r);
    }
    rotate_by_theta<DIM>(ow, c, w, r);
}

// expSmpX.m:1-12 (lmean is the unnormalised mean light direction).
template <int DIM>
__device__ __forceinline__ void exp_smp_x(const WalkParams &P, double *x, double *px, PathRng &r)
{
    double lz = fabs(P.unmeanl[DIM - 1]);
    double s = P.sigt / lz;
    double dmax = P.box_max[DIM - 1] - P.box_min[DIM - 1];
    double rmax = 1.0 - exp(-dmax * s);
    double d = -log(-r.rand() * rmax + 1.0) / s;
#pragma unroll
    for (int k = 0; k < DIM - 1; ++k) x[k] = r.rand() * (P.box_max[k] - P.box_min[k]) + P.box_min[k];
    x[DIM - 1] = (P.unmeanl[DIM - 1] > 0) ? (d + P.box_min[DIM - 1]) : (-d + P.box_max[DIM - 1]);
    *px = exp(-s * d) / rmax * s * dmax;
}

}  // namespace scmc
