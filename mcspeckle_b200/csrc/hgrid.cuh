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
// voxel is nudged by 1e-4 of the voxel size (cubeDist.m:13-16).
template <int DIM>
__device__ __forceinline__ double hg_optical_depth(const HGrid &g, const double *x, const double *dir, double nd)
{
    double m[3], nx[3], bmn[3], bmx[3];
    const double thr = 1.0000000000000004e-07;
#pragma unroll
    for (int k = 0; k < 3; ++k) { m[k] = -dir[k]; nx[k] = x[k]; bmn[k] = bmx[k] = 0.0; }
    double ep = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) ep = fmax(ep, fabs(g.bbin[k]));
    ep = 1.0000000000000002e-04 * ep;  // 0.1^4 as MATLAB evaluates it
    double bdv = 0.0, wbdv = 0.0;
    for (int guard = 0; guard < (1 << 22); ++guard) {
        const int64_t bi = hg_find_bin(g, nx, bmn, bmx);
        double d = INFINITY;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            const double den = fmax(fabs(m[j]), thr);
            const double bd = (m[j] <= 0) ? (nx[j] - bmn[j]) / den : (-nx[j] + bmx[j]) / den;
            d = fmin(d, bd);
        }
#pragma unroll
        for (int k = 0; k < DIM; ++k) nx[k] = nx[k] + (d + ep) * m[k];
        const double s = g.sigt[bi];
        bdv = bdv + d;
        wbdv = wbdv + d * s;
        if (bdv >= nd) {
            wbdv = wbdv - (bdv - nd) * s;
            break;
        }
        if (hg_outside(g, nx)) break;
    }
    return wbdv;
}

}  // namespace scmc
