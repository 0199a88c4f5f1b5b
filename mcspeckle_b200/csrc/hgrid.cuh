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
__device__ __forceinline__ double hg_optical_depth(const HGrid &g, const double *x, const double *dir, double nd)
{
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

}  // namespace scmc
