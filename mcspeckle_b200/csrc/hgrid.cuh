// hgrid.cuh - voxel medium for the heterogeneous path (MCCovHetro.m,
// MCsampleHetro.m): the grid, findBin.m, smpWoodcock.m and the voxel-marched
// attenuation of evalphaseattHetro.m, in FP64.
#pragma once

#include "common.cuh"

namespace scmc {


__device__ __forceinline__ bool hg_outside(const HGrid &g, const double *x)
{
    bool o = false;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (k < g.dim) o |= (x[k] > g.bmax[k]) || (x[k] < g.bmin[k]);
    return o;
}

// findBin.m:1-17 (0-based index; subscripts clamped to the grid).
__device__ __forceinline__ int64_t hg_find_bin(const HGrid &g, const double *x, double *bmn, double *bmx)
{
    int64_t ind = 0, stride = 1;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        if (j >= g.dim) break;
        double ii = ceil((x[j] - g.bmin[j]) / g.bbin[j]);
        ii = fmin(fmax(ii, 1.0), (double)g.nb[j]);
        ind += (int64_t)(ii - 1) * stride;
        stride *= g.nb[j];
        if (bmn) {
            bmn[j] = g.bmin[j] + g.bbin[j] * (ii - 1);
            bmx[j] = bmn[j] + g.bbin[j];
        }
    }
    return ind;
}

__device__ __forceinline__ double hg_albedo(const HGrid &g, const double *x)
{
    return g.alb ? g.alb[hg_find_bin(g, x, nullptr, nullptr)] : g.alb_scalar;
}

// evalphaseattHetro.m:29-51: path length and optical depth from x along -dir
// to the box (or to distance nd), voxel by voxel; the exit point of each
// voxel is nudged by 1e-4 of the voxel size (cubeDist.m:13-16).  The
// divisions of findBin.m and cubeDist.m are multiplications by reciprocals
// (per grid and per ray); after the first step every position lies 1e-4 of
// a voxel past a face, far beyond the last-bit differences this makes.  Each
// voxel's sigma_t is added one step later, so its load overlaps the next
// step's arithmetic.
template <int DIM>
__device__ __forceinline__ double hg_optical_depth_tri(const HGrid &g, const double *x, const double *dir, double nd);

template <int DIM>
__device__ __forceinline__ double hg_optical_depth(const HGrid &g, const double *x, const double *dir, double nd)
{
    if (g.trilinear) return hg_optical_depth_tri<DIM>(g, x, dir, nd);
    double m[3], nx[3], iden[3];
    const double thr = 1.0000000000000004e-07;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        m[k] = -dir[k];
        nx[k] = x[k];
        iden[k] = 1.0 / fmax(fabs(m[k]), thr);
    }
    double ep = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) ep = fmax(ep, fabs(g.bbin[k]));
    ep = 1.0000000000000002e-04 * ep;  // 0.1^4 as MATLAB evaluates it
    double bdv = 0.0, wbdv = 0.0, d_prev = 0.0, s_prev = 0.0;
    for (int guard = 0; guard < (1 << 22); ++guard) {
        // findBin.m with the subscripts clamped to the grid
        int64_t bi = 0, stride = 1;
        double d = INFINITY;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            double ii = ceil((nx[j] - g.bmin[j]) * g.ibbin[j]);
            ii = fmin(fmax(ii, 1.0), (double)g.nb[j]);
            bi += (int64_t)(ii - 1) * stride;
            stride *= g.nb[j];
            const double bmn = g.bmin[j] + g.bbin[j] * (ii - 1), bmx = bmn + g.bbin[j];
            const double bd = (m[j] <= 0) ? (nx[j] - bmn) * iden[j] : (-nx[j] + bmx) * iden[j];
            d = fmin(d, bd);
        }
        const double s = g.sigt[bi];
        wbdv = wbdv + d_prev * s_prev;
#pragma unroll
        for (int k = 0; k < DIM; ++k) nx[k] = nx[k] + (d + ep) * m[k];
        bdv = bdv + d;
        d_prev = d;
        s_prev = s;
        if (bdv >= nd) {
            d_prev = d - (bdv - nd);
            break;
        }
        if (hg_outside(g, nx)) break;
    }
    return wbdv + d_prev * s_prev;
}

// ---------------------------------------------------------------------------
// Trilinear sigma (extension): sigma(x) interpolated between the voxel
// centres bmin + (i + 1/2) bbin, clamped to the outer centres, so that it is
// continuous and, between two neighbouring voxel-centre planes per axis, a
// product of linear functions of the coordinates.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ double hg_sigma_tri(const HGrid &g, const double *x)
{
    int i0[3] = {0, 0, 0};
    double f[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        double u = (x[k] - g.bmin[k]) * g.ibbin[k] - 0.5;
        u = fmin(fmax(u, 0.0), (double)(g.nb[k] - 1));
        int i = (int)floor(u);
        i = i > g.nb[k] - 2 ? g.nb[k] - 2 : i;
        i = i < 0 ? 0 : i;
        i0[k] = i;
        f[k] = g.nb[k] > 1 ? u - (double)i : 0.0;
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < (1 << DIM); ++c) {
        int64_t idx = 0, stride = 1;
        double wgt = 1.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            const int b = (c >> k) & 1;
            const int ik = (g.nb[k] > 1) ? i0[k] + b : 0;
            idx += (int64_t)ik * stride;
            stride *= g.nb[k];
            wgt *= b ? f[k] : 1.0 - f[k];
        }
        if (wgt != 0.0) s += wgt * g.sigt[idx];
    }
    return s;
}

// The optical depth of trilinear sigma from x along -dir over min(nd, the
// distance to the box): the ray is cut where it crosses a voxel-centre plane
// of any axis; on each piece sigma(t) is a polynomial of degree <= 3 and
// Simpson's rule (t1 - t0)/6 (s0 + 4 s_mid + s1) is exact.  Per axis the
// march keeps the integer floor of the centre coordinate on the current piece
// (stepped by one at each crossing, so no rounding per piece), from which the
// piece's dual cell and its fraction follow: f = u - cell inside the grid of
// centres, 0 or 1 in the outer half voxels (sigma is clamped to the outer
// centres there).  The cell's 2^DIM corner values stay in registers until the
// cell changes; indices are 32-bit.
template <int DIM>
__device__ __forceinline__ double hg_optical_depth_tri(const HGrid &g, const double *x, const double *dir, double nd)
{
    constexpr int NC = 1 << DIM;
    double tn[3], dt[3], u0[3], du[3];
    int fl[3], st[3], off[3], nbm2[3], strd[3];
    double tend = INFINITY;
    int stride = 1;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const double m = -dir[k];
        // distance to the box face along m (cubeDist.m without the 1e-7 floor for |m| = 0)
        if (m > 0) tend = fmin(tend, (g.bmax[k] - x[k]) / m);
        else if (m < 0) tend = fmin(tend, (x[k] - g.bmin[k]) / -m);
        // the centre coordinate u(t) = u0 + t du, the next plane crossing, the spacing of crossings
        const double u = (x[k] - g.bmin[k]) * g.ibbin[k] - 0.5;
        u0[k] = u;
        du[k] = m * g.ibbin[k];
        if (m > 0) {
            tn[k] = (floor(u) + 1.0 - u) * g.bbin[k] / m;
            dt[k] = g.bbin[k] / m;
            fl[k] = (int)floor(u);
            st[k] = 1;
        } else if (m < 0) {
            tn[k] = (u - (ceil(u) - 1.0)) * g.bbin[k] / -m;
            dt[k] = g.bbin[k] / -m;
            fl[k] = (int)ceil(u) - 1;
            st[k] = -1;
        } else {
            tn[k] = INFINITY;
            dt[k] = INFINITY;
            fl[k] = (int)floor(u);
            st[k] = 0;
        }
        nbm2[k] = g.nb[k] - 2;
        off[k] = g.nb[k] > 1 ? stride : 0;  // a corner's step along axis k (none on a one-voxel axis)
        strd[k] = stride;
        stride *= g.nb[k];
    }
    tend = fmax(fmin(tend, nd), 0.0);
    double cs[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) cs[c] = 0.0;
    int loaded = -1;  // base index of the corners in cs
    double t0 = 0.0, s0 = 0.0, tau = 0.0;
    for (int guard = 0; guard < (1 << 22) && t0 < tend; ++guard) {
        double t1 = tend;
#pragma unroll
        for (int k = 0; k < DIM; ++k) t1 = fmin(t1, tn[k]);
        // this piece's cell and fractions f_k(t) = c0_k + c1_k t
        double c0[3], c1[3];
        int base = 0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            int cell;
            if (nbm2[k] < 0) {  // one voxel along k
                cell = 0;
                c0[k] = 0.0;
                c1[k] = 0.0;
            } else if (fl[k] < 0) {
                cell = 0;
                c0[k] = 0.0;
                c1[k] = 0.0;
            } else if (fl[k] > nbm2[k]) {
                cell = nbm2[k];
                c0[k] = 1.0;
                c1[k] = 0.0;
            } else {
                cell = fl[k];
                c0[k] = u0[k] - (double)cell;
                c1[k] = du[k];
            }
            base += cell * strd[k];
        }
        if (base != loaded) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                int idx = base;
#pragma unroll
                for (int k = 0; k < DIM; ++k) idx += ((c >> k) & 1) ? off[k] : 0;
                cs[c] = g.sigt[idx];
            }
            loaded = base;
        }
        auto sig = [&](double t) {
            double v[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) v[c] = cs[c];
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                const double f = fma(t, c1[k], c0[k]);
                const int h = 1 << (DIM - 1 - k);
#pragma unroll
                for (int c = 0; c < h; ++c) v[c] = fma(f, v[2 * c + 1] - v[2 * c], v[2 * c]);
            }
            return v[0];
        };
        if (guard == 0) s0 = sig(t0);
        const double sm = sig(0.5 * (t0 + t1)), s1 = sig(t1);
        tau += (t1 - t0) * (1.0 / 6.0) * (s0 + 4.0 * sm + s1);
        // the crossings that end this piece
#pragma unroll
        for (int k = 0; k < DIM; ++k)
            if (tn[k] <= t1) {
                tn[k] += dt[k];
                fl[k] += st[k];
            }
        t0 = t1;
        s0 = s1;
    }
    return tau;
}

// The same march in FP32 for the reduced precisions (NEE only; the FP64
// mode keeps hg_optical_depth_tri).  The per-ray set-up (centre coordinate,
// first crossing, distance to the box) is formed in FP64 and rounded once;
// each crossing time is the first one plus an integer count of spacings (one
// FMA, no accumulated rounding), so the pieces stay within FP32 rounding of
// the planes (about 3e-5 of a wavelength at 500 wavelengths), where a shift
// changes the integral only to second order because sigma is continuous.
template <int DIM>
__device__ __forceinline__ float hg_optical_depth_tri_f32(const HGrid &g, const double *x, const double *dir, double nd)
{
    constexpr int NC = 1 << DIM;
    float tb[3], dt[3], u0[3], du[3];
    int fl[3], st[3], cnt[3], off[3], nbm2[3], strd[3];
    double tend_d = INFINITY;
    int stride = 1;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const double m = -dir[k];
        if (m > 0) tend_d = fmin(tend_d, (g.bmax[k] - x[k]) / m);
        else if (m < 0) tend_d = fmin(tend_d, (x[k] - g.bmin[k]) / -m);
        const double u = (x[k] - g.bmin[k]) * g.ibbin[k] - 0.5;
        u0[k] = (float)u;
        du[k] = (float)(m * g.ibbin[k]);
        if (m > 0) {
            tb[k] = (float)((floor(u) + 1.0 - u) * g.bbin[k] / m);
            dt[k] = (float)(g.bbin[k] / m);
            fl[k] = (int)floor(u);
            st[k] = 1;
        } else if (m < 0) {
            tb[k] = (float)((u - (ceil(u) - 1.0)) * g.bbin[k] / -m);
            dt[k] = (float)(g.bbin[k] / -m);
            fl[k] = (int)ceil(u) - 1;
            st[k] = -1;
        } else {
            tb[k] = INFINITY;
            dt[k] = 0.f;
            fl[k] = (int)floor(u);
            st[k] = 0;
        }
        cnt[k] = 0;
        nbm2[k] = g.nb[k] - 2;
        off[k] = g.nb[k] > 1 ? stride : 0;
        strd[k] = stride;
        stride *= g.nb[k];
    }
    const float tend = (float)fmax(fmin(tend_d, nd), 0.0);
    float cs[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) cs[c] = 0.f;
    int loaded = -1;
    float t0 = 0.f, s0 = 0.f, tau = 0.f;
    for (int guard = 0; guard < (1 << 22) && t0 < tend; ++guard) {
        float tn[3];
        float t1 = tend;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            tn[k] = st[k] ? fmaf((float)cnt[k], dt[k], tb[k]) : INFINITY;
            t1 = fminf(t1, tn[k]);
        }
        float c0[3], c1[3];
        int base = 0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            int cell;
            if (nbm2[k] < 0 || fl[k] < 0) {
                cell = 0;
                c0[k] = 0.f;
                c1[k] = 0.f;
            } else if (fl[k] > nbm2[k]) {
                cell = nbm2[k];
                c0[k] = 1.f;
                c1[k] = 0.f;
            } else {
                cell = fl[k];
                c0[k] = u0[k] - (float)cell;
                c1[k] = du[k];
            }
            base += cell * strd[k];
        }
        if (base != loaded) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                int idx = base;
#pragma unroll
                for (int k = 0; k < DIM; ++k) idx += ((c >> k) & 1) ? off[k] : 0;
                cs[c] = g.sigt_f[idx];
            }
            loaded = base;
        }
        auto sig = [&](float t) {
            float v[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) v[c] = cs[c];
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                const float f = fmaf(t, c1[k], c0[k]);
                const int h = 1 << (DIM - 1 - k);
#pragma unroll
                for (int c = 0; c < h; ++c) v[c] = fmaf(f, v[2 * c + 1] - v[2 * c], v[2 * c]);
            }
            return v[0];
        };
        if (guard == 0) s0 = sig(t0);
        const float sm = sig(0.5f * (t0 + t1)), s1 = sig(t1);
        tau = fmaf((t1 - t0) * (1.f / 6.f), s0 + 4.f * sm + s1, tau);
#pragma unroll
        for (int k = 0; k < DIM; ++k)
            if (tn[k] <= t1) {
                ++cnt[k];
                fl[k] += st[k];
            }
        t0 = t1;
        s0 = s1;
    }
    return tau;
}

}  // namespace scmc
