// nee.cuh - next-event estimation vectors (evalphaseatt.m, evalampfunc_general.m)
// in three arithmetic policies.
//
//   P64  - FP64 throughout (reference arithmetic).
//   PMIX - positions, dot products and the phase argument k*(w.x) in FP64,
//          the argument reduced mod 2*pi in FP64, then FP32 sincos / exp.
//   P32  - plain FP32: FP32 positions, FP32 phase argument without reduction.
//
// For an event at x with first scatterer x1 and first direction w1 the
// vectors are (MCfield.m:159-215, MCcov.m:157-219):
//   e_v0[i]    = phaseatt(x1, vs_i)                         single scattering
//   e_l0[j]    = phaseatt(x1, l_j)
//   a[i]       = phaseatt(x,  vs_i) * af(ow . rv_i)          e_v_ms
//   b[j]       = phaseatt(x1, l_j)  * af(w1 . rl_j) / w0p    e_l0_ms
//   a0[i]      = phaseatt(x1, vs_i) * af(-w1 . rv_i) / w0p   e_v0_ms (CBS)
//   b2[j]      = phaseatt(x,  l_j)  * af(-ow . rl_j)         e_l_ms  (CBS)
// with vs = ff_sign*v and the entrance directions rv, rl taken from x1 for
// near-field sources (the reference keeps them fixed along the path).
#pragma once

#include "common.cuh"
#include "hgrid.cuh"

namespace scmc {

struct NeeParams {
    int nv, nl, is_ff_l, is_ff_v, cbs;
    double sigt_half;        // sigt/2
    double kw;               // pi*2/lambda
    double lambda;
    double box_min[3], box_max[3];
    const double *l;         // [nl][3]
    const double *vs;        // [nv][3] = ff_sign * v
    const double *v;         // [nv][3]
    int has_pf0;
    double meanl[3];
    PhaseFn pf, pf0;
    int hetero;              // voxel medium: attenuation marched through hg
    HGrid hg;
    float fbox_min[3], fbox_max[3];  // FP32 copies for the attenuation of PMIX / P32
};

// Fill the FP32 copies of the box (call after box_min / box_max are set).
inline void nee_set_fbox(NeeParams &Q)
{
    for (int k = 0; k < 3; ++k) {
        Q.fbox_min[k] = (float)Q.box_min[k];
        Q.fbox_max[k] = (float)Q.box_max[k];
    }
}

template <typename T> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

enum PrecPolicy { P64 = 0, PMIX = 1, P32 = 2 };

// Reduce a phase (radians, FP64) to [-pi, pi] in FP64: 2*pi is split into a
// head that multiplies integers exactly and a tail.
__device__ __forceinline__ double reduce_2pi(double ph)
{
    const double inv2pi = 0.15915494309189535;
    const double twopi_hi = 6.28318530717958623200;   // 2*pi rounded to double
    const double twopi_lo = 2.4492935982947064e-16;   // 2*pi - twopi_hi
    double q = rint(ph * inv2pi);
    return fma(-q, twopi_lo, fma(-q, twopi_hi, ph));
}

// phaseatt for one direction / position, FP64 inputs.  evalphaseatt.m:1-21.
// evalphaseattHetro.m:1-52: as evalphaseatt, with the optical depth marched
// voxel by voxel (far field: to the box; near field: to the source).
template <int DIM, int POL>
__device__ __noinline__ typename cplx_t<typename std::conditional<POL == P64, double, float>::type>::type
phaseatt_hetero(const double *x, const double *d, int is_ff, const NeeParams &Q)
{
    double pv, rv, nd, dir[3] = {0, 0, 0};
    if (is_ff) {
        pv = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) { pv += x[k] * d[k]; dir[k] = d[k]; }
        rv = 1.0;
        nd = 1.0e12;
    } else {
        double dd[3];
        nd = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) { dd[k] = x[k] - d[k]; nd += dd[k] * dd[k]; }
        nd = sqrt(nd);
#pragma unroll
        for (int k = 0; k < DIM; ++k) dir[k] = dd[k] / nd;
        pv = nd;
        rv = (DIM == 3) ? 1.0 / (nd + 0.01 * Q.lambda) : 1.0 / sqrt(nd + 0.01 * Q.lambda);
    }
    double wbdv;
    if constexpr (POL != P64) {  // reduced precisions: the trilinear march in FP32 when the grid has a copy
        wbdv = (Q.hg.trilinear && Q.hg.sigt_f) ? (double)hg_optical_depth_tri_f32<DIM>(Q.hg, x, dir, nd)
                                               : hg_optical_depth<DIM>(Q.hg, x, dir, nd);
    } else {
        wbdv = hg_optical_depth<DIM>(Q.hg, x, dir, nd);
    }
    const double ph = Q.kw * pv;
    if constexpr (POL == P64) {
        double s, c;
        sincos(ph, &s, &c);
        const double a = exp(-(1.0 / 2.0 * wbdv)) * rv;
        return make_double2(a * c, a * s);
    } else {
        float s, c;
        if (POL == PMIX) sincosf((float)reduce_2pi(ph), &s, &c);
        else sincosf((float)ph, &s, &c);
        const float a = expf(-(float)(0.5 * wbdv)) * (float)rv;
        return make_float2(a * c, a * s);
    }
}

template <int DIM, int POL>
__device__ __forceinline__ typename cplx_t<typename std::conditional<POL == P64, double, float>::type>::type
phaseatt(const double *x, const double *d, int is_ff, const NeeParams &Q)
{
    if (Q.hetero) return phaseatt_hetero<DIM, POL>(x, d, is_ff, Q);
    if constexpr (POL == P32) {
        float xf[3], df[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) { xf[k] = (float)x[k]; df[k] = (float)d[k]; }
        float pv, rv, bdv;
        const float thr = 1.0000000000000004e-07f;
        float u[3];
        if (is_ff) {
            pv = 0.f;
#pragma unroll
            for (int k = 0; k < DIM; ++k) { pv += xf[k] * df[k]; u[k] = -df[k]; }
            rv = 1.f;
        } else {
            float dd[3], nd = 0.f;
#pragma unroll
            for (int k = 0; k < DIM; ++k) { dd[k] = xf[k] - df[k]; nd += dd[k] * dd[k]; }
            nd = sqrtf(nd);
#pragma unroll
            for (int k = 0; k < DIM; ++k) u[k] = -(dd[k] / nd);
            pv = nd;
            rv = (DIM == 3) ? 1.f / (nd + 0.01f * (float)Q.lambda) : rsqrtf(nd + 0.01f * (float)Q.lambda);
        }
        bdv = INFINITY;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            float den = fmaxf(fabsf(u[j]), thr);
            float bd = (u[j] <= 0.f) ? (xf[j] - (float)Q.box_min[j]) / den : (-xf[j] + (float)Q.box_max[j]) / den;
            bdv = fminf(bdv, bd);
        }
        if (!is_ff) bdv = fminf(bdv, pv);
        float s, c;
        sincosf((float)Q.kw * pv, &s, &c);
        float a = expf(-(float)Q.sigt_half * bdv) * rv;
        return make_float2(a * c, a * s);
    } else if constexpr (POL == PMIX) {
        // Only the phase argument k*pv needs FP64: it is formed and reduced
        // mod 2pi in FP64.  The attenuation exp(-sigt/2*bdv)*rv, whose
        // relative error is that of bdv, is evaluated in FP32.
        float xf[3], u[3], rv = 1.f;
        double pv = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) xf[k] = (float)x[k];
        float nearest = INFINITY;
        if (is_ff) {
#pragma unroll
            for (int k = 0; k < DIM; ++k) { pv += x[k] * d[k]; u[k] = -(float)d[k]; }
        } else {
            double dd[3], nd = 0.0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) { dd[k] = x[k] - d[k]; nd += dd[k] * dd[k]; }
            nd = sqrt(nd);
            const float ndf = (float)nd, inv = 1.f / ndf;
#pragma unroll
            for (int k = 0; k < DIM; ++k) u[k] = -(float)dd[k] * inv;
            pv = nd;
            const float t = ndf + 0.01f * (float)Q.lambda;
            rv = (DIM == 3) ? __frcp_rn(t) : rsqrtf(t);
            nearest = ndf;
        }
        float bdv = nearest;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            const float den = fmaxf(fabsf(u[j]), 1.0000000000000004e-07f);
            const float num = (u[j] <= 0.f) ? (xf[j] - Q.fbox_min[j]) : (Q.fbox_max[j] - xf[j]);
            bdv = fminf(bdv, __fdividef(num, den));
        }
        float s, c;
        __sincosf((float)reduce_2pi(Q.kw * pv), &s, &c);
        const float a = __expf(-(float)Q.sigt_half * bdv) * rv;
        return make_float2(a * c, a * s);
    } else {
        double pv, rv, bdv, u[3];
        if (is_ff) {
            pv = 0.0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) { pv += x[k] * d[k]; u[k] = -d[k]; }
            rv = 1.0;
            bdv = cube_dist<DIM>(x, Q.box_min, Q.box_max, u);
        } else {
            double dd[3], nd = 0.0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) { dd[k] = x[k] - d[k]; nd += dd[k] * dd[k]; }
            nd = sqrt(nd);
#pragma unroll
            for (int k = 0; k < DIM; ++k) u[k] = -(dd[k] / nd);
            pv = nd;
            rv = (DIM == 3) ? 1.0 / (nd + 0.01 * Q.lambda) : 1.0 / sqrt(nd + 0.01 * Q.lambda);
            bdv = fmin(cube_dist<DIM>(x, Q.box_min, Q.box_max, u), nd);
        }
        double ph = Q.kw * pv;
        double at = Q.sigt_half * bdv;
        double s, c;
        sincos(ph, &s, &c);
        double a = exp(-at) * rv;
        return make_double2(a * c, a * s);
    }
}

// Scattering amplitude af(c) in the arithmetic of the policy.  P64 is
// evalampfunc (FP64, evalampfunc_general.m:1-19).  PMIX / P32 evaluate it in
// FP32: HG as sqrt((1-g^2)/(4pi)) * den^(-3/4) (3-D) or sqrt((1-g^2)/(2pi)) *
// den^(-1/2) (2-D) with den = 1 + g^2 - 2gc (formed in FP64 for PMIX, where
// it cancels for forward lobes); tabulated as the nearest entry of the
// angle acos(c), taken as 2 asin(sqrt((1-c)/2)) (or pi minus its mirror for
// c < 0) so that FP32 keeps the angle accurate near 0 and pi.
template <int DIM, int POL>
__device__ __forceinline__ typename cplx_t<typename std::conditional<POL == P64, double, float>::type>::type
amp_eval(double c, const PhaseFn &pf)
{
    if constexpr (POL == P64) {
        return evalampfunc<DIM>(c, pf);
    } else {
        if (pf.sct_type == 1) return make_float2((float)(1.0 / sqrt((DIM == 3 ? 4.0 : 2.0) * SCMC_PI)), 0.f);
        if (pf.sct_type == 2) {
            const double cc = fmin(fmax(c, -1.0), 1.0);
            if (pf.cos_bins) {
                const double2 t = pf.eval_amp[tab_cos_index(cc, pf.table_n)];
                return make_float2((float)t.x, (float)t.y);
            }
            float ang;
            if (cc >= 0.0) ang = 2.f * asinf(sqrtf((float)(0.5 * (1.0 - cc))));
            else ang = (float)SCMC_PI - 2.f * asinf(sqrtf((float)(0.5 * (1.0 + cc))));
            const float span = (DIM == 2) ? (float)(2.0 * SCMC_PI) : (float)SCMC_PI;
            int idx = (int)roundf(ang * (float)(pf.table_n - 1) / span);
            idx = idx < 0 ? 0 : (idx > pf.table_n - 1 ? pf.table_n - 1 : idx);
            const double2 t = pf.eval_amp[idx];
            return make_float2((float)t.x, (float)t.y);
        }
        const double g = pf.g;
        float den;
        if (POL == PMIX) den = (float)fma(-2.0 * g, c, 1.0 + g * g);
        else den = 1.f + (float)g * (float)g - 2.f * (float)g * (float)c;
        const float r = rsqrtf(den);
        if (DIM == 3) return make_float2((float)sqrt((1.0 - g * g) / (4.0 * SCMC_PI)) * r * sqrtf(r), 0.f);
        return make_float2((float)sqrt((1.0 - g * g) / (2.0 * SCMC_PI)) * r, 0.f);
    }
}

// evalphaseatt with sigt = 0 (MCCovHetro.m:152: u_l0 for the mean field):
// exp(i k pv) rv, no attenuation.
template <int DIM, int POL>
__device__ __forceinline__ typename cplx_t<typename std::conditional<POL == P64, double, float>::type>::type
phase_plain(const double *x, const double *d, int is_ff, const NeeParams &Q)
{
    double pv = 0.0, rv = 1.0;
    if (is_ff) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) pv += x[k] * d[k];
    } else {
        double nd = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) nd += (x[k] - d[k]) * (x[k] - d[k]);
        nd = sqrt(nd);
        pv = nd;
        rv = (DIM == 3) ? 1.0 / (nd + 0.01 * Q.lambda) : 1.0 / sqrt(nd + 0.01 * Q.lambda);
    }
    const double ph = Q.kw * pv;
    if constexpr (POL == P64) {
        double sn, cs;
        sincos(ph, &sn, &cs);
        return make_double2(rv * cs, rv * sn);
    } else {
        float sn, cs;
        sincosf((float)reduce_2pi(ph), &sn, &cs);
        return make_float2((float)rv * cs, (float)rv * sn);
    }
}

template <typename C> __device__ __forceinline__ C to_c(double2 v);
template <> __device__ __forceinline__ double2 to_c<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 to_c<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

template <typename C> __device__ __forceinline__ C cscale(C v, double s);
template <> __device__ __forceinline__ double2 cscale<double2>(double2 v, double s) { return make_double2(v.x * s, v.y * s); }
template <> __device__ __forceinline__ float2 cscale<float2>(float2 v, double s) { return make_float2(v.x * (float)s, v.y * (float)s); }

// Entrance direction of view i / light j as seen from x1 (MCfield.m:130-137).
template <int DIM>
__device__ __forceinline__ void view_dir(const NeeParams &Q, int i, const double *x1, double *rv)
{
    const double *vi = Q.v + 3 * i;
    if (Q.is_ff_v) {
#pragma unroll
        for (int k = 0; k < 3; ++k) rv[k] = vi[k];
        return;
    }
    double s = 0.0, d[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < DIM; ++k) { d[k] = vi[k] - x1[k]; s += d[k] * d[k]; }
    s = sqrt(s);
#pragma unroll
    for (int k = 0; k < 3; ++k) rv[k] = k < DIM ? d[k] / s : 0.0;
}

template <int DIM>
__device__ __forceinline__ void light_dir(const NeeParams &Q, int j, const double *x1, double *rl)
{
    const double *lj = Q.l + 3 * j;
    if (Q.is_ff_l) {
#pragma unroll
        for (int k = 0; k < 3; ++k) rl[k] = lj[k];
        return;
    }
    double s = 0.0, d[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < DIM; ++k) { d[k] = x1[k] - lj[k]; s += d[k] * d[k]; }
    s = sqrt(s);
#pragma unroll
    for (int k = 0; k < 3; ++k) rl[k] = k < DIM ? d[k] / s : 0.0;
}

template <int DIM>
__device__ __forceinline__ double dot3(const double *a, const double *b)
{
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) s += a[k] * b[k];
    return s;
}

// First-direction density w0p (MCfield.m:149-155).
template <int DIM>
__device__ __forceinline__ double first_dir_pdf(const NeeParams &Q, const double *w1)
{
    if (!Q.has_pf0) return 1.0 / sqrt((DIM == 3 ? 4.0 : 2.0) * SCMC_PI);
    return evalampfunc<DIM>(dot3<DIM>(Q.meanl, w1), Q.pf0).x;
}

// View-side entries of a multiple-scattering event: a = e_v_ms, a0 = e_v0_ms.
template <int DIM, int POL, typename C>
__device__ __forceinline__ void nee_view(const NeeParams &Q, int i, const double *x, const double *ow,
                                         const double *x1, const double *w1, double w0p, C &a, C &a0)
{
    double rv[3];
    view_dir<DIM>(Q, i, x1, rv);
    const double *vsi = Q.vs + 3 * i;
    C e = phaseatt<DIM, POL>(x, vsi, Q.is_ff_v, Q);
    C af = amp_eval<DIM, POL>(dot3<DIM>(ow, rv), Q.pf);
    a = cmul(e, af);
    if (Q.cbs) {
        C e0 = phaseatt<DIM, POL>(x1, vsi, Q.is_ff_v, Q);
        C af0 = amp_eval<DIM, POL>(-dot3<DIM>(w1, rv), Q.pf);
        af0 = cscale<C>(af0, 1.0 / w0p);
        a0 = cmul(e0, af0);
    } else {
        a0 = C{};
    }
}

// Light-side entries: b = e_l0_ms, b2 = e_l_ms.
template <int DIM, int POL, typename C>
__device__ __forceinline__ void nee_light(const NeeParams &Q, int j, const double *x, const double *ow,
                                          const double *x1, const double *w1, double w0p, C &b, C &b2)
{
    double rl[3];
    light_dir<DIM>(Q, j, x1, rl);
    const double *lj = Q.l + 3 * j;
    C e0 = phaseatt<DIM, POL>(x1, lj, Q.is_ff_l, Q);
    C af = amp_eval<DIM, POL>(dot3<DIM>(w1, rl), Q.pf);
    af = cscale<C>(af, 1.0 / w0p);
    b = cmul(e0, af);
    if (Q.cbs) {
        C e = phaseatt<DIM, POL>(x, lj, Q.is_ff_l, Q);
        C af2 = amp_eval<DIM, POL>(-dot3<DIM>(ow, rl), Q.pf);
        b2 = cmul(e, af2);
    } else {
        b2 = C{};
    }
}

// Single-scattering amplitude af(rl_j . rv_i) for one (view, light) pair.
template <int DIM>
__device__ __forceinline__ double2 single_amp(const NeeParams &Q, int i, int j, const double *x1)
{
    double rv[3], rl[3];
    view_dir<DIM>(Q, i, x1, rv);
    light_dir<DIM>(Q, j, x1, rl);
    return evalampfunc<DIM>(dot3<DIM>(rl, rv), Q.pf);
}

}  // namespace scmc
