// fq.cuh - MCfieldFourierQuad on the GPU (MCfieldFourierQuad.m:77-303).
//
// The reference records every vertex of an isotropic walk, sorts vertices
// by the depth of the view-side vertex, grids them per z plane on the
// lateral pixel grid and takes fftshift(fft2(ifftshift(.))) per plane and
// light, then flips, crops, multiplies by exp(zexp0 * tz) and sums planes.
// That FFT is the centred DFT
//     X[q] = sum_p x[p] exp(-2 pi i (q-c)(p-c)/M),   c = floor(M/2),
// evaluated only at the cropped, flipped outputs; here it is evaluated
// directly for each vertex: output (r1, r2) of plane P receives
//     c_e * T[r1][p1_e] * T[r2][p2_e],   T[r][p] = exp(-2 pi i m'(r) P(p) / M)
// with the same pixel indices p1, p2 (rounded positions) and bin indices
// m'(r) as the reference.  Vertices are bucketed by plane (counting sort),
// each CTA owns a 32 x 32 output tile of one light and one plane, stages the
// twiddle columns of a sub-batch of vertices in shared memory, and at the
// plane's end multiplies by exp(zexp0 * tz) before adding into the FP64 sum.
#pragma once

#include <cuda_fp16.h>

#include "accum.cuh"

namespace scmc {

struct FqParams {
    int nv0, nx, nz, nl, cbs;
    double box_stp, gx1, gy1;
    double kw;             // 2 pi / lambda
    double sigt_half;
    double bmin_z, bmax_z;
    double l_diratt, l_idiratt;
    const double *gz;      // nz plane boundaries
    const double *l;       // [nl][3]
    // phase conventions: MCfieldFourierQuad uses light phase +k l.x and
    // vertex phase -k (-z1 + tz); MCfieldFourierQuadOnWave uses vsign for both
    double lsign = 1.0, vsign_vertex = -1.0;
    // MCfieldFourierQuadOnWave: lights combined with weights wl (nl of them)
    // into one output light; null for MCfieldFourierQuad
    const double2 *wl = nullptr;
    // extension: l holds point-source positions and each vertex's light factor
    // is evalphaseatt.m:10-16's near-field term, evaluated through phaseatt
    // with the walk's (padded) box in `nf`
    int light_point = 0;
    NeeParams nf{};
};

// The light factor of an entry for output light j (MCfieldFourierQuad.m:272):
// exp(i k l_j.xl - sigt/2 * slab attenuation); for a point source at l_j
// (extension) the near-field evalphaseatt term; with weights
// (MCfieldFourierQuadOnWave.m:278-302) sum_j wl_j exp(i vsign k l_j.xl) times
// the same attenuation.  Phases are reduced mod 2 pi in FP64 outside P64.
template <int POL>
__device__ __forceinline__ typename cplx_t<typename std::conditional<POL == P64, double, float>::type>::type
fq_light_factor(const FqParams &F, int j, const double *xl)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    const double at = F.sigt_half * ((xl[2] - F.bmin_z) * F.l_diratt + (F.bmax_z - xl[2]) * F.l_idiratt);
    const int j0 = F.wl ? 0 : j, j1 = F.wl ? F.nl : j + 1;
    C sum = C{};
    if (F.light_point) {  // one point source per output light (the OnWave form has none)
        return phaseatt<3, POL>(xl, F.l + 3 * j, 0, F.nf);
    }
    for (int jj = j0; jj < j1; ++jj) {
        const double *lj = F.l + 3 * jj;
        const double ph = F.lsign * F.kw * (lj[0] * xl[0] + lj[1] * xl[1] + lj[2] * xl[2]);
        C e;
        if constexpr (POL == P64) {
            double s, co;
            sincos(ph, &s, &co);
            e = make_double2(co, s);
        } else {
            float s, co;
            sincosf((float)reduce_2pi(ph), &s, &co);
            e = make_float2(co, s);
        }
        if (F.wl) e = cmul(e, to_c<C>(F.wl[jj]));
        sum.x += e.x;
        sum.y += e.y;
    }
    if constexpr (POL == P64) {
        const double a = exp(-at);
        return make_double2(a * sum.x, a * sum.y);
    } else {
        const float a = expf(-(float)at);
        return make_float2(a * sum.x, a * sum.y);
    }
}

// One entry per (vertex, pass): pass 0 views from the first scatterer and
// lights from the vertex (MCfieldFourierQuad.m:224-232 tt = 1), pass 1 the
// reverse (tt = 2, CBS).
struct FqEntry {
    double xl[3];     // light-side position
    double2 c0;       // pxL * exp(-i k (tz - zv)), light independent
    int p1, p2;       // 0-based pixel indices of the view-side position
    int plane;
};

// With one output light (one light, or the weighted sum of MCfieldFourierQuadOnWave)
// and the CTA-pair form, an entry needs only its factor and pixels: 16 bytes
// instead of 56 through the plane sort.
struct FqEntryC {
    float2 sv;                 // c0 * light factor (FP32, as the operands use it)
    unsigned short p1, p2;     // pixel indices (< 65536, checked on the host)
    int plane;
};

__device__ __forceinline__ double fq_mround(double x) { return x < 0 ? -floor(-x + 0.5) : floor(x + 0.5); }

// Plane of a view-side depth: plane j holds gz[j] <= z < gz[j+1]; depths at
// or beyond the last boundary are in no plane (the reference's scan never
// reaches them).
__device__ __forceinline__ int fq_plane(const FqParams &F, double z)
{
    int lo = 0, hi = F.nz - 1;  // find the first boundary index b in [1, nz-1] with z < gz[b]
    if (!(z < F.gz[F.nz - 1])) return -1;
    lo = 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (z < F.gz[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo - 1;
}

// Build the entries of a batch: singles are paths 0..n_paths-1, multis
// follow.  counts[plane] is incremented for the counting sort.
template <bool COMPACT>
__global__ void fq_entries_kernel(const __grid_constant__ FqParams F, SingleRec S, int64_t scap, MultiRec M, int64_t mcap, int64_t n_paths,
                                  int64_t n_multi, void *__restrict__ out_v, int *__restrict__ counts)
{
    const int64_t nvert = n_paths + n_multi;
    const int passes = F.cbs ? 2 : 1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nvert * passes;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int pass = (int)(k / nvert);
        const int64_t v = k % nvert;
        double x[3], x1[3], wpx, xi;
        int pl;
        if (v < n_paths) {
            for (int d = 0; d < 3; ++d) x1[d] = x[d] = S.x1[d * scap + v];
            wpx = S.wpx[v];
            xi = S.xi[v];
            pl = 1;
        } else {
            const int64_t e = v - n_paths;
            const int64_t p = M.path[e];
            for (int d = 0; d < 3; ++d) {
                x[d] = M.x[d * mcap + e];
                x1[d] = S.x1[d * scap + p];
            }
            wpx = M.wpx[e];
            xi = M.xi[e];
            pl = M.plen[e];
        }
        const double *xv = pass == 0 ? x1 : x;
        const double *xl = pass == 0 ? x : x1;
        FqEntry en;
        for (int d = 0; d < 3; ++d) en.xl[d] = xl[d];
        en.plane = fq_plane(F, xv[2]);
        int p1 = (int)fq_mround((xv[0] - F.gx1) / F.box_stp);
        int p2 = (int)fq_mround((xv[1] - F.gy1) / F.box_stp);
        en.p1 = min(max(p1, 0), F.nx - 1);
        en.p2 = min(max(p2, 0), F.nx - 1);
        // pxL = sqrt(w/px) e^{2 pi i xi}, /sqrt(2) with CBS after the first event (lines 181-182)
        double s = sqrt(wpx);
        if (F.cbs && pl > 1) s = 1.0 / sqrt(2.0) * s;
        double sp, cp;
        sincos(2.0 * SCMC_PI * xi, &sp, &cp);
        double tz = 0.0;
        if (en.plane >= 0) tz = (F.gz[en.plane] + F.gz[en.plane + 1]) / 2;
        double sd, cd;
        // exp(-2 pi i/lambda (-z + tz)) (MCfieldFourierQuad.m:272; OnWave: vsign for -1)
        sincos(F.vsign_vertex * F.kw * (-xv[2] + tz), &sd, &cd);
        en.c0 = make_double2(s * (cp * cd - sp * sd), s * (cp * sd + sp * cd));
        if constexpr (COMPACT) {
            FqEntryC ec;
            ec.sv = cmul(to_c<float2>(en.c0), fq_light_factor<PMIX>(F, 0, en.xl));
            ec.p1 = (unsigned short)en.p1;
            ec.p2 = (unsigned short)en.p2;
            ec.plane = en.plane;
            reinterpret_cast<FqEntryC *>(out_v)[k] = ec;
        } else {
            reinterpret_cast<FqEntry *>(out_v)[k] = en;
        }
        if (en.plane >= 0) atomicAdd(&counts[en.plane], 1);
    }
}

template <typename E>
__global__ void fq_scatter_kernel(const E *__restrict__ in, int64_t n, const int *__restrict__ offsets,
                                  int *__restrict__ cursor, E *__restrict__ out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const E e = in[k];
        if (e.plane < 0) continue;
        const int pos = offsets[e.plane] + atomicAdd(&cursor[e.plane], 1);
        out[pos] = e;
    }
}

// T[r][p] = exp(-2 pi i m'(r) P(p) / M): the centred DFT's twiddles at the
// reference's cropped, flipped bins (see the file comment); stored [p][r]
// when transposed.
template <typename C>
__global__ void fq_twiddle_kernel(int nv0, int nx, double M, double nx_pad, double nv_pad, C *__restrict__ T,
                                  int transposed)
{
    const double c = floor(M / 2);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)nv0 * nx;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int r = transposed ? (int)(k % nv0) : (int)(k / nx), p = transposed ? (int)(k / nv0) : (int)(k % nx);
        const double m = (M - 1 - ((double)r + nv_pad)) - c;
        const double P = ((double)p + nx_pad) - c;
        const double t = fmod(m * P, M);
        double s, co;
        sincos(-2.0 * SCMC_PI * t / M, &s, &co);
        T[k] = to_c<C>(make_double2(co, s));
    }
}

constexpr int kFqTile = 32;
constexpr int kFqEB = 16;

// One CTA: a 32 x 32 tile of (r1, r2) for light j and plane planes[blockIdx.y].
template <int POL, typename AccT>
__global__ void __launch_bounds__(256)
fq_accum_kernel(const __grid_constant__ FqParams F, const FqEntry *__restrict__ E, const int *__restrict__ offsets,
                const int *__restrict__ planes, const typename cplx_t<typename std::conditional<POL == P64, double, float>::type>::type *__restrict__ T,
                const double2 *__restrict__ zexp0, AccT *__restrict__ U)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    __shared__ C t1[kFqEB][kFqTile];
    __shared__ C t2[kFqEB][kFqTile];
    __shared__ C sc[kFqEB];
    const int nvt = (F.nv0 + kFqTile - 1) / kFqTile;
    const int tile = blockIdx.x % (nvt * nvt);
    const int j = blockIdx.x / (nvt * nvt);
    const int r10 = (tile % nvt) * kFqTile, r20 = (tile / nvt) * kFqTile;
    const int plane = planes[blockIdx.y];
    const int e0 = offsets[plane], e1 = offsets[plane + 1];
    C acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = C{};
    for (int eb = e0; eb < e1; eb += kFqEB) {
        const int ne = min(kFqEB, e1 - eb);
        // per entry: the light factor exp(i k l.xl - sigt/2 * slab attenuation) (line 272)
        if (threadIdx.x < ne) {
            const FqEntry en = E[eb + threadIdx.x];
            sc[threadIdx.x] = cmul(to_c<C>(en.c0), fq_light_factor<POL>(F, j, en.xl));
        }
        for (int idx = threadIdx.x; idx < kFqEB * 2 * kFqTile; idx += blockDim.x) {
            const int k = idx / (2 * kFqTile), m = idx % (2 * kFqTile);
            C v = C{};
            if (k < ne) {
                const FqEntry &en = E[eb + k];
                if (m < kFqTile) {
                    const int r = r10 + m;
                    if (r < F.nv0) v = T[(int64_t)r * F.nx + en.p1];
                } else {
                    const int r = r20 + (m - kFqTile);
                    if (r < F.nv0) v = T[(int64_t)r * F.nx + en.p2];
                }
            }
            if (m < kFqTile) t1[k][m] = v;
            else t2[k][m - kFqTile] = v;
        }
        __syncthreads();
        for (int k = 0; k < ne; ++k) {
            const C s = sc[k];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int o = threadIdx.x + 256 * q;
                const int a = o % kFqTile, b = o / kFqTile;
                const C w = cmul(s, t2[k][b]);
                const C v = cmul(w, t1[k][a]);
                acc[q].x += v.x;
                acc[q].y += v.y;
            }
        }
        __syncthreads();
    }
    const int nv0 = F.nv0;
    const double tz = (F.gz[plane] + F.gz[plane + 1]) / 2;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int o = threadIdx.x + 256 * q;
        const int r1 = r10 + o % kFqTile, r2 = r20 + o / kFqTile;
        if (r1 < nv0 && r2 < nv0) {
            const double2 z = zexp0[r1 + (int64_t)nv0 * r2];
            // exp(zexp0 * tz) (line 281)
            const double mag = exp(z.x * tz);
            double s, co;
            sincos(z.y * tz, &s, &co);
            const double2 f = make_double2(mag * co, mag * s);
            const double2 a = make_double2((double)acc[q].x, (double)acc[q].y);
            const double2 v = cmul(f, a);
            const int64_t off = 2 * ((int64_t)r1 + (int64_t)nv0 * r2 + (int64_t)nv0 * nv0 * j);
            atomicAdd(&U[off], (AccT)v.x);
            atomicAdd(&U[off + 1], (AccT)v.y);
        }
    }
}

// ---------------------------------------------------------------------------
// Tensor-core form (MIXED / FP16).  Per plane P and light j the DFT sum is the
// complex product F_P = A_P B_P^T over the plane's entries e:
//     A_P[r1][e] = s_e(j) T[r1][p1_e],   B_P[r2][e] = T[r2][p2_e],
// with s_e(j) = c0_e * exp(i k l_j.xl_e - sigt/2 * slab attenuation).  The
// entries, sorted by plane, are laid out in blocks of 32 (a plane's last block
// zero-padded), in the real expansion of the tensor-core field path
//     A[2r1] = (Re a, -Im a), A[2r1+1] = (Im a, Re a), B[r2] = (Re b, Im b),
// two K columns per entry, so one 64-column K block never spans two planes.
// fq_planes_tc_kernel (herk_tc.cuh) computes F_P plane after plane for a
// range of planes per CTA, multiplies each by exp(zexp0 * tz_P) into a
// running sum in TMEM and adds that sum into the output once; the output of
// this form is stored [light][r1][r2] (r2 fastest) in FP32.
// ---------------------------------------------------------------------------
// The entry scales s_e(j) of a plane group can span many decades (a point
// source: 1/r and the attenuation), and FP16 keeps its relative precision
// only above 2^-14.  The group's operands are therefore scaled by a power of
// two 2^(13 - e), e the exponent of max |s_e| (exact in FP16 and FP32), which
// the plane loop undoes when it adds a chain into U (fq_scale_exponent,
// herk_tc.cuh).  fq_scale_kernel finds max |s_e| (as the ordered bits of a
// non-negative float).
__global__ void __launch_bounds__(256)
fq_scale_kernel(const __grid_constant__ FqParams F, const FqEntry *__restrict__ E, const int2 *__restrict__ blk,
                int64_t nblk, int bs, int light, unsigned *__restrict__ max_bits)
{
    float m = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nblk * bs; i += (int64_t)gridDim.x * blockDim.x) {
        const int2 bk = blk[i / bs];
        const int t = (int)(i % bs);
        if (t < bk.y) {
            const FqEntry en = E[bk.x + t];
            const float2 sv = cmul(to_c<float2>(en.c0), fq_light_factor<PMIX>(F, light, en.xl));
            m = fmaxf(m, fmaxf(fabsf(sv.x), fabsf(sv.y)));
        }
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && isfinite(m)) atomicMax(max_bits, __float_as_uint(m));
}

template <bool SPLIT>
__global__ void __launch_bounds__(256)
fq_tc_rows_kernel(const __grid_constant__ FqParams F, const FqEntry *__restrict__ E, const int2 *__restrict__ blk,
                  int light, const float2 *__restrict__ Tt, int64_t K, __half *__restrict__ Ahi,
                  __half *__restrict__ Alo, __half *__restrict__ Bm, const unsigned *__restrict__ max_bits)
{
    const float scale = ldexpf(1.f, fq_scale_exponent(max_bits));
    constexpr int RB = 64;  // twiddle rows staged per pass
    __shared__ float2 ss[32];
    __shared__ int sp1[32], sp2[32];
    __shared__ float2 ta[RB][33], tb[RB][33];  // [r - r0][entry]
    const int2 bk = blk[blockIdx.x];  // (first entry, entries in this block)
    if (threadIdx.x < 32) {
        float2 sv = make_float2(0.f, 0.f);
        int p1 = 0, p2 = 0;
        if ((int)threadIdx.x < bk.y) {
            const FqEntry en = E[bk.x + threadIdx.x];
            sv = cmul(to_c<float2>(en.c0), fq_light_factor<PMIX>(F, light, en.xl));
            sv.x *= scale;
            sv.y *= scale;
            p1 = en.p1;
            p2 = en.p2;
        }
        ss[threadIdx.x] = sv;
        sp1[threadIdx.x] = p1;
        sp2[threadIdx.x] = p2;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t col = 2 * ((int64_t)blockIdx.x * 32 + lane);
    for (int r0 = 0; r0 < F.nv0; r0 += RB) {
        __syncthreads();
        // the entries' twiddle columns T[r0 .. r0 + RB)[p], contiguous in Tt
        for (int idx = threadIdx.x; idx < 32 * RB; idx += blockDim.x) {
            const int e = idx / RB, rr = idx % RB, r = r0 + rr;
            const bool ok = e < bk.y && r < F.nv0;
            ta[rr][e] = ok ? Tt[(int64_t)sp1[e] * F.nv0 + r] : make_float2(0.f, 0.f);
            tb[rr][e] = ok ? Tt[(int64_t)sp2[e] * F.nv0 + r] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        const float2 sv = ss[lane];
        for (int rr = warp; rr < RB && r0 + rr < F.nv0; rr += 8) {
            const int r = r0 + rr;
            const float2 av = cmul(sv, ta[rr][lane]), bv = tb[rr][lane];
            const __half hr = __float2half_rn(av.x), hi = __float2half_rn(av.y);
            __half *e = Ahi + (int64_t)(2 * r) * K + col;
            *reinterpret_cast<__half2 *>(e) = __halves2half2(hr, __hneg(hi));
            *reinterpret_cast<__half2 *>(e + K) = __halves2half2(hi, hr);
            if (SPLIT) {
                const __half lr = __float2half_rn(av.x - __half2float(hr));
                const __half li = __float2half_rn(av.y - __half2float(hi));
                __half *o = Alo + (int64_t)(2 * r) * K + col;
                *reinterpret_cast<__half2 *>(o) = __halves2half2(lr, __hneg(li));
                *reinterpret_cast<__half2 *>(o + K) = __halves2half2(li, lr);
            }
            *reinterpret_cast<__half2 *>(Bm + (int64_t)r * K + col) =
                __halves2half2(__float2half_rn(bv.x), __float2half_rn(bv.y));
        }
    }
}

__device__ __forceinline__ uint32_t h2_bits(__half2 h)
{
    return *reinterpret_cast<const uint32_t *>(&h);
}

// The CTA-pair form's per-entry inputs in K-column order (block * 64 + t,
// a plane's last block zero-padded): sv = c0 * light factor (FP32, unscaled)
// and the pixel pair (p1, p2); also max |sv| for the group's operand scale.
__global__ void __launch_bounds__(256)
fq_pair_prep_kernel(const __grid_constant__ FqParams F, const FqEntry *__restrict__ E, const int2 *__restrict__ blk,
                    int64_t nblk, int light, float2 *__restrict__ svk, int2 *__restrict__ ppk,
                    unsigned *__restrict__ max_bits)
{
    float m = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nblk * 64; i += (int64_t)gridDim.x * blockDim.x) {
        const int2 bk = blk[i >> 6];
        const int t = (int)(i & 63);
        float2 sv = make_float2(0.f, 0.f);
        int2 pp = make_int2(0, 0);
        if (t < bk.y) {
            const FqEntry en = E[bk.x + t];
            sv = cmul(to_c<float2>(en.c0), fq_light_factor<PMIX>(F, light, en.xl));
            pp = make_int2(en.p1, en.p2);
            m = fmaxf(m, fmaxf(fabsf(sv.x), fabsf(sv.y)));
        }
        svk[i] = sv;
        ppk[i] = pp;
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && isfinite(m)) atomicMax(max_bits, __float_as_uint(m));
}

// The same from compact entries (factor already applied).
__global__ void __launch_bounds__(256)
fq_pair_prep_compact_kernel(const FqEntryC *__restrict__ E, const int2 *__restrict__ blk, int64_t nblk,
                            float2 *__restrict__ svk, int2 *__restrict__ ppk, unsigned *__restrict__ max_bits)
{
    float m = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nblk * 64; i += (int64_t)gridDim.x * blockDim.x) {
        const int2 bk = blk[i >> 6];
        const int t = (int)(i & 63);
        float2 sv = make_float2(0.f, 0.f);
        int2 pp = make_int2(0, 0);
        if (t < bk.y) {
            const FqEntryC en = E[bk.x + t];
            sv = en.sv;
            pp = make_int2(en.p1, en.p2);
            m = fmaxf(m, fmaxf(fabsf(sv.x), fabsf(sv.y)));
        }
        svk[i] = sv;
        ppk[i] = pp;
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && isfinite(m)) atomicMax(max_bits, __float_as_uint(m));
}

// Planar rows for the CTA-pair form (grids of at least 128 angles): one block
// of 64 K columns per CTA, written as the contiguous slab [row][64 entries] of
// each plane at blockIdx.x * nv0 * 64: A planes Re / Im of s_e(j) T[r1][p1_e]
// (with the low parts for hi+lo), B planes Re / Im of T[r2][p2_e].  Thread =
// (rows r = r0, r0 + 16, ..., 4 consecutive entries): one 8-byte store per
// plane and row, a warp's stores two consecutive rows (256 contiguous bytes).
// T[r][p] is linear in r in its phase (fq_twiddle_kernel: T[r + 1][p] =
// T[r][p] exp(2 pi i P / M)), so each thread reads the twiddles of its first
// two rows only and steps the rest with the ratio T[r0 + 16][p] conj(T[r0][p])
// in FP32 (at most nv0 / 16 - 1 steps, far below FP16's rounding).  No shared
// memory and no barrier: several CTAs per SM keep the stores streaming.
template <bool SPLIT>
__global__ void __launch_bounds__(256, 4)
fq_tc_rows_planar_kernel(int nv0, const float2 *__restrict__ svk, const int2 *__restrict__ ppk,
                         const float2 *__restrict__ Tt, __half *__restrict__ Are, __half *__restrict__ Aim,
                         __half *__restrict__ Alr, __half *__restrict__ Ali, __half *__restrict__ Bre,
                         __half *__restrict__ Bim, const unsigned *__restrict__ max_bits)
{
    const float scale = ldexpf(1.f, fq_scale_exponent(max_bits));
    const int e0 = (threadIdx.x & 15) * 4, rsub = threadIdx.x >> 4;
    const int64_t c0 = (int64_t)blockIdx.x * 64 + e0;
    float2 av[4], aw[4], bv[4], bw[4];  // current A, B values of the 4 entries and their 16-row ratios
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float2 sv = svk[c0 + j];  // zero in a block's padding
        sv.x *= scale;
        sv.y *= scale;
        const int2 pp = ppk[c0 + j];
        const int64_t o1 = (int64_t)pp.x * nv0 + rsub, o2 = (int64_t)pp.y * nv0 + rsub;
        const float2 t1 = Tt[o1], t2 = Tt[o2], u1 = Tt[o1 + 16], u2 = Tt[o2 + 16];  // nv0 >= 128
        av[j] = cmul(sv, t1);
        bv[j] = t2;
        aw[j] = cmul(u1, make_float2(t1.x, -t1.y));
        bw[j] = cmul(u2, make_float2(t2.x, -t2.y));
    }
    const int64_t slab = (int64_t)blockIdx.x * nv0 * 64;
    for (int r = rsub; r < nv0; r += 16) {
        const __half2 r01 = __floats2half2_rn(av[0].x, av[1].x), r23 = __floats2half2_rn(av[2].x, av[3].x);
        const __half2 i01 = __floats2half2_rn(av[0].y, av[1].y), i23 = __floats2half2_rn(av[2].y, av[3].y);
        const int64_t o = slab + (int64_t)r * 64 + e0;
        *reinterpret_cast<uint2 *>(Are + o) = make_uint2(h2_bits(r01), h2_bits(r23));
        *reinterpret_cast<uint2 *>(Aim + o) = make_uint2(h2_bits(i01), h2_bits(i23));
        if (SPLIT) {
            *reinterpret_cast<uint2 *>(Alr + o) = make_uint2(
                h2_bits(__floats2half2_rn(av[0].x - __low2float(r01), av[1].x - __high2float(r01))),
                h2_bits(__floats2half2_rn(av[2].x - __low2float(r23), av[3].x - __high2float(r23))));
            *reinterpret_cast<uint2 *>(Ali + o) = make_uint2(
                h2_bits(__floats2half2_rn(av[0].y - __low2float(i01), av[1].y - __high2float(i01))),
                h2_bits(__floats2half2_rn(av[2].y - __low2float(i23), av[3].y - __high2float(i23))));
        }
        *reinterpret_cast<uint2 *>(Bre + o) = make_uint2(h2_bits(__floats2half2_rn(bv[0].x, bv[1].x)),
                                                         h2_bits(__floats2half2_rn(bv[2].x, bv[3].x)));
        *reinterpret_cast<uint2 *>(Bim + o) = make_uint2(h2_bits(__floats2half2_rn(bv[0].y, bv[1].y)),
                                                         h2_bits(__floats2half2_rn(bv[2].y, bv[3].y)));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            av[j] = cmul(av[j], aw[j]);
            bv[j] = cmul(bv[j], bw[j]);
        }
    }
}

// u = norm * boxexp0 o U.  r2_fast: U is stored [light][r1][r2] (the
// tensor-core form) instead of u's [light][r2][r1].
template <typename AccT>
__global__ void fq_finalize_kernel(const AccT *__restrict__ U, const double2 *__restrict__ boxexp0, int nv0, int nl,
                                   double norm, double2 *__restrict__ u, int r2_fast = 0)
{
    const int64_t n = (int64_t)nv0 * nv0 * nl;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double2 b = boxexp0[k % ((int64_t)nv0 * nv0)];
        int64_t src = k;
        if (r2_fast) {
            const int64_t r1 = k % nv0, r2 = (k / nv0) % nv0, j = k / ((int64_t)nv0 * nv0);
            src = r2 + nv0 * (r1 + nv0 * j);
        }
        const double2 a = make_double2((double)U[2 * src], (double)U[2 * src + 1]);
        const double2 v = cmul(a, b);
        u[k] = make_double2(norm * v.x, norm * v.y);
    }
}

}  // namespace scmc
