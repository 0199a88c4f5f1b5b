// postprocess.cuh - SCMC's post-processing of rendered fields and covariances.
//
//  refocus (refocus.m:1-34): rU(p) = (sum_v conj(u_v) e^{-2 pi i/lambda v.p})
//      e^{2 pi i/lambda l.p} on an ndgrid of points.  One thread per grid
//      point; the views are staged in shared memory.  The phase is formed in
//      FP64; MIXED reduces it mod 2 pi in FP64 and evaluates sincos in FP32.
//
//  samples of a field from a covariance (samplingFromCovMatrix.m:47-64):
//      Sigma = 0.5 [Re C, -Im C; Im C, Re C] (2N x 2N), s = g chol(Sigma)
//      for rows g of standard normals, z = s(1:N) + i s(N+1:2N).  Blocked
//      right-looking Cholesky in FP64 (64-column blocks: diagonal block in
//      one CTA's shared memory, panel by forward substitution, trailing
//      update by a tiled FP64 product), then the triangular product with the
//      normals, which come from the per-sample Philox normal streams.
#pragma once

#include "nee.cuh"

namespace scmc {

struct RefocusGrid {
    int dim;
    int64_t n[3];
    double bmin[3], stp[3];
};

template <bool MIXED>
__global__ void __launch_bounds__(256)
refocus_kernel(RefocusGrid G, const double2 *__restrict__ u, const double *__restrict__ v, int64_t nv, double l0,
               double l1, double l2, double kw, int as_written, double2 *__restrict__ rU)
{
    __shared__ double sv[256][3];
    __shared__ double2 su[256];
    const int64_t N = G.n[0] * G.n[1] * G.n[2];
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double pos[3] = {0, 0, 0};
    {
        int64_t r = p;
        for (int d = 0; d < G.dim; ++d) {
            pos[d] = G.bmin[d] + (double)(r % G.n[d]) * G.stp[d];
            r /= G.n[d];
        }
    }
    double sx = 0.0, sy = 0.0;
    for (int64_t v0 = 0; v0 < nv; v0 += 256) {
        const int nc = (int)min((int64_t)256, nv - v0);
        __syncthreads();
        if ((int)threadIdx.x < nc) {
            for (int d = 0; d < 3; ++d) sv[threadIdx.x][d] = d < G.dim ? v[G.dim * (v0 + threadIdx.x) + d] : 0.0;
            su[threadIdx.x] = u[v0 + threadIdx.x];
        }
        __syncthreads();
        if (p < N) {
            for (int i = 0; i < nc; ++i) {
                const double ph = -kw * (sv[i][0] * pos[0] + sv[i][1] * pos[1] + sv[i][2] * pos[2]);
                double c, s;
                if (MIXED) {
                    float fs, fc;
                    __sincosf((float)reduce_2pi(ph), &fs, &fc);
                    s = fs;
                    c = fc;
                } else {
                    sincos(ph, &s, &c);
                }
                const double2 uu = su[i];  // conj(u) * e
                sx += uu.x * c + uu.y * s;
                sy += uu.x * s - uu.y * c;
            }
        }
    }
    if (p >= N) return;
    const double pl = kw * (l0 * pos[0] + l1 * pos[1] + l2 * pos[2]);
    double c, s;
    sincos(pl, &s, &c);
    rU[p] = (as_written && p == 0) ? make_double2(0.0, 0.0) : make_double2(sx * c - sy * s, sx * s + sy * c);
}

// Sigma (n = 2N, column-major) from C (N x N complex, column-major).
__global__ void sigma_build_kernel(const double2 *__restrict__ C, int64_t N, double *__restrict__ S)
{
    const int64_t n = 2 * N;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N * N; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q % N, j = q / N;
        const double2 c = C[q];
        S[i + n * j] = 0.5 * c.x;
        S[(i + N) + n * (j + N)] = 0.5 * c.x;
        S[i + n * (j + N)] = -0.5 * c.y;
        S[(i + N) + n * j] = 0.5 * c.y;
    }
}

constexpr int kCholNB = 64;

// Diagonal block [k0, k0 + nb) factorised in shared memory (lower, in place;
// the strictly upper part of the block is zeroed).  A pivot that is not
// positive sets *err and is replaced by 1 so the remaining steps stay finite.
__global__ void __launch_bounds__(256) chol_diag_kernel(double *__restrict__ S, int64_t n, int64_t k0, int nb,
                                                        int *__restrict__ err)
{
    __shared__ double a[kCholNB][kCholNB + 1];
    for (int q = threadIdx.x; q < nb * nb; q += blockDim.x) {
        const int i = q % nb, j = q / nb;
        a[i][j] = S[(k0 + i) + n * (k0 + j)];
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        if (threadIdx.x == 0) {
            double d = a[j][j];
            if (!(d > 0.0)) {
                atomicExch(err, 1);
                d = 1.0;
            }
            a[j][j] = sqrt(d);
        }
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < nb; i += blockDim.x) a[i][j] /= a[j][j];
        __syncthreads();
        const int m = nb - j - 1;
        for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
            const int i = j + 1 + q % m, c = j + 1 + q / m;
            if (c <= i) a[i][c] -= a[i][j] * a[c][j];
        }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < nb * nb; q += blockDim.x) {
        const int i = q % nb, j = q / nb;
        S[(k0 + i) + n * (k0 + j)] = i >= j ? a[i][j] : 0.0;
    }
}

// Panel rows [k0 + nb, n): L_ik = A_ik L_kk^{-T} by forward substitution, one
// thread per row.
__global__ void __launch_bounds__(128) chol_panel_kernel(double *__restrict__ S, int64_t n, int64_t k0, int nb)
{
    __shared__ double L[kCholNB][kCholNB + 1];
    for (int q = threadIdx.x; q < nb * nb; q += blockDim.x) {
        const int i = q % nb, j = q / nb;
        L[i][j] = S[(k0 + i) + n * (k0 + j)];
    }
    __syncthreads();
    const int64_t row = k0 + nb + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (row >= n) return;
    double x[kCholNB];
#pragma unroll 4
    for (int j = 0; j < nb; ++j) {
        double s = S[row + n * (k0 + j)];
        for (int c = 0; c < j; ++c) s -= x[c] * L[j][c];
        x[j] = s / L[j][j];
    }
    for (int j = 0; j < nb; ++j) S[row + n * (k0 + j)] = x[j];
}

// Trailing update A_ij -= sum_c L_ic L_jc over the panel columns [k0, k0+nb),
// for the lower-triangle 64 x 64 tiles of [k1, n) x [k1, n), k1 = k0 + nb.
// 256 threads, a 4 x 4 register tile each.
__global__ void __launch_bounds__(256) chol_update_kernel(double *__restrict__ S, int64_t n, int64_t k0, int nb)
{
    constexpr int KC = 32;  // panel columns staged per pass
    __shared__ double Li[kCholNB][KC + 1];  // [row in tile][panel column]
    __shared__ double Lj[kCholNB][KC + 1];
    const int64_t k1 = k0 + nb;
    const int64_t nt = (n - k1 + kCholNB - 1) / kCholNB;
    // blockIdx.x enumerates lower tiles (ti >= tj)
    int64_t t = blockIdx.x, ti = 0;
    while (t > ti) {
        t -= ti + 1;
        ++ti;
    }
    const int64_t tj = t;
    if (ti >= nt) return;
    const int64_t r0 = k1 + ti * kCholNB, c0 = k1 + tj * kCholNB;
    const int tr = (threadIdx.x % 16) * 4, tc = (threadIdx.x / 16) * 4;
    double acc[4][4] = {};
    for (int cb = 0; cb < nb; cb += KC) {
        const int kc = min(KC, nb - cb);
        __syncthreads();
        for (int q = threadIdx.x; q < kCholNB * KC; q += blockDim.x) {
            const int r = q % kCholNB, c = q / kCholNB;
            const bool in = c < kc;
            Li[r][c] = (in && r0 + r < n) ? S[(r0 + r) + n * (k0 + cb + c)] : 0.0;
            Lj[r][c] = (in && c0 + r < n) ? S[(c0 + r) + n * (k0 + cb + c)] : 0.0;
        }
        __syncthreads();
        for (int c = 0; c < kc; ++c) {
            double a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                a[q] = Li[tr + q][c];
                b[q] = Lj[tc + q][c];
            }
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] += a[p] * b[q];
        }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t i = r0 + tr + p, j = c0 + tc + q;
            if (i < n && j < n && j <= i) S[i + n * j] -= acc[p][q];
        }
}

// g[t][i]: the i-th value of the normal Philox stream of path t (2 per block).
__global__ void normals_kernel(uint32_t k0, uint32_t k1, int64_t T, int64_t n, double *__restrict__ g)
{
    const int64_t pairs = (n + 1) / 2;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < T * pairs; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = q / pairs, b = q % pairs;
        uint32_t o[4];
        philox4x32_10((uint32_t)b, 1u, (uint32_t)t, (uint32_t)((uint64_t)t >> 32), k0, k1, o);
        const double u1 = u52_to_unit(o[0], o[1]), u2 = u52_to_unit(o[2], o[3]);
        const double rad = sqrt(-2.0 * log(u1)), ang = (2.0 * SCMC_PI) * u2;
        g[t * n + 2 * b] = rad * cos(ang);
        if (2 * b + 1 < n) g[t * n + 2 * b + 1] = rad * sin(ang);
    }
}

// s_t = L g_t (row j: sum over i <= j), z_t = s(0:N) + i s(N:2N).
__global__ void sample_product_kernel(const double *__restrict__ S, int64_t N, int64_t T, const double *__restrict__ g,
                                      double2 *__restrict__ Z)
{
    const int64_t n = 2 * N;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N * T; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = q % N, t = q / N;
        const double *gt = g + t * n;
        double re = 0.0, im = 0.0;
        for (int64_t i = 0; i <= j; ++i) re += S[j + n * i] * gt[i];
        for (int64_t i = 0; i <= j + N; ++i) im += S[(j + N) + n * i] * gt[i];
        Z[j + N * t] = make_double2(re, im);
    }
}

// ---------------------------------------------------------------------------
// Memory-effect view of a covariance.  C(v1, v2, l1, l2) (v1 fastest, the
// scmc layout) with the views on an nvx x nvy grid and the lights on an
// nlx x nly grid (flat index x fastest) is reduced to the mean over all
// entries with the same view offset v1 - v2 and light offset l1 - l2:
//   R(dv, dl) = 1/(n(dv) n(dl)) sum_{v1 - v2 = dv, l1 - l2 = dl} C(v1, v2, l1, l2),
// n(d) = (nx - |dx|)(ny - |dy|) the number of pairs with offset d, stored
// with offset index (dx + nx - 1) + (2 nx - 1)(dy + ny - 1), view offset
// fastest, complex FP32.  examples/memoryEffectMeasurements/
// memoryEffectMeasurements.m:72-86 takes such means along diagonals of C.
// One CTA per light pair (l1, l2): its nv x nv block is contiguous, so the
// reads are coalesced; block sums per view offset collect in shared memory
// (FP64) and are added once into the FP64 sums of (view offset, light offset).
// Every element of C is read once: the kernel is HBM bound.
// ---------------------------------------------------------------------------
struct OffsetGrid {
    int nvx, nvy, nlx, nly;
};

__global__ void __launch_bounds__(256) offsets_sum_kernel(const double2 *__restrict__ C1,
                                                          const double2 *__restrict__ C2, OffsetGrid g,
                                                          double2 *__restrict__ sums)
{
    extern __shared__ double2 part[];  // one per view offset
    const int nv = g.nvx * g.nvy, nl = g.nlx * g.nly;
    const int ovx = 2 * g.nvx - 1, nvo = ovx * (2 * g.nvy - 1), olx = 2 * g.nlx - 1;
    for (int o = threadIdx.x; o < nvo; o += blockDim.x) part[o] = make_double2(0.0, 0.0);
    __syncthreads();
    const int l1 = blockIdx.x % nl, l2 = blockIdx.x / nl;
    const int64_t base = (int64_t)nv * nv * blockIdx.x;  // (l1, l2) block, l1 fastest
    for (int64_t k = threadIdx.x; k < (int64_t)nv * nv; k += blockDim.x) {
        const int v1 = (int)(k % nv), v2 = (int)(k / nv);
        double2 c = C1[base + k];
        if (C2) {
            const double2 d = C2[base + k];
            c.x += d.x;
            c.y += d.y;
        }
        const int dx = v1 % g.nvx - v2 % g.nvx, dy = v1 / g.nvx - v2 / g.nvx;
        const int o = (dx + g.nvx - 1) + ovx * (dy + g.nvy - 1);
        atomicAdd(&part[o].x, c.x);
        atomicAdd(&part[o].y, c.y);
    }
    __syncthreads();
    const int ldx = l1 % g.nlx - l2 % g.nlx, ldy = l1 / g.nlx - l2 / g.nlx;
    const int lo = (ldx + g.nlx - 1) + olx * (ldy + g.nly - 1);
    for (int o = threadIdx.x; o < nvo; o += blockDim.x) {
        atomicAdd(&sums[(int64_t)lo * nvo + o].x, part[o].x);
        atomicAdd(&sums[(int64_t)lo * nvo + o].y, part[o].y);
    }
}

__global__ void offsets_finalize_kernel(const double2 *__restrict__ sums, OffsetGrid g, float2 *__restrict__ R)
{
    const int ovx = 2 * g.nvx - 1, nvo = ovx * (2 * g.nvy - 1), olx = 2 * g.nlx - 1;
    const int64_t n = (int64_t)nvo * olx * (2 * g.nly - 1);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int o = (int)(k % nvo), lo = (int)(k / nvo);
        const int dvx = o % ovx - (g.nvx - 1), dvy = o / ovx - (g.nvy - 1);
        const int dlx = lo % olx - (g.nlx - 1), dly = lo / olx - (g.nly - 1);
        const double cnt = (double)(g.nvx - abs(dvx)) * (g.nvy - abs(dvy)) * (g.nlx - abs(dlx)) * (g.nly - abs(dly));
        R[k] = make_float2((float)(sums[k].x / cnt), (float)(sums[k].y / cnt));
    }
}

}  // namespace scmc
