// onwave.cuh - MCfieldOnWave (MCfieldOnWave.m:1-267): the field of all lights
// at once, combined with complex weights Wl (an incident wave made of the
// lights).  Per event the light side collapses to one number,
//   multiple scattering  B = sum_j b_j Wl_j  (and B2 = sum_j b2_j Wl_j, CBS),
//                        u_i += alpha (a_i B + a0_i B2)            (lines 177, 212, 223-226)
//   single scattering    u_i += alpha e_v0_i sum_j af_ij e_l0_j Wl_j   (line 221)
// so the work per multiple-scattering event is O(nv + nl) instead of the
// O(nv nl) of the full field.  One warp per event: lanes share the lights
// (warp-shuffle sums) and then the views; each CTA accumulates a chunk of
// views in shared memory (FP64) and adds it to the output once.
#pragma once

#include "accum.cuh"

namespace scmc {

constexpr int kOwWarps = 8;
constexpr int kOwMaxViews = 2048;  // views per CTA chunk (grid.y covers the rest)

template <typename C> __device__ __forceinline__ C warp_csum(C v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

inline size_t onwave_smem(int nvc, int nl, size_t csize)
{
    return sizeof(double2) * (size_t)nvc + csize * (size_t)kOwWarps * nl + 16;
}

template <int DIM, int POL, bool SINGLE>
__global__ void __launch_bounds__(kOwWarps * 32)
onwave_accum_kernel(const __grid_constant__ NeeParams Q, SingleRec S, int64_t scap, MultiRec M, int64_t mcap, int64_t n_events,
                    int64_t ev_per_cta, int nvc, const double2 *__restrict__ Wl, double2 *__restrict__ U)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *acc = reinterpret_cast<double2 *>(smem_raw);  // [nvc]
    C *cbuf = reinterpret_cast<C *>(acc + nvc);            // [warps][nl] (singles)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int v0 = blockIdx.y * nvc;
    const int nvt = min(nvc, Q.nv - v0);
    for (int i = threadIdx.x; i < nvt; i += blockDim.x) acc[i] = make_double2(0.0, 0.0);
    __syncthreads();
    const int64_t e_begin = (int64_t)blockIdx.x * ev_per_cta;
    const int64_t e_end = min(n_events, e_begin + ev_per_cta);
    C *cb = cbuf + (size_t)warp * Q.nl;
    for (int64_t e = e_begin + warp; e < e_end; e += kOwWarps) {
        EventView ev;
        load_event<DIM, SINGLE>(Q, S, scap, M, mcap, e, ev);
        double s = sqrt(ev.wpx);
        if (!SINGLE && Q.cbs) s *= 1.0 / sqrt(2.0);
        double sp, cp;
        sincos(2.0 * SCMC_PI * ev.xi, &sp, &cp);  // exp(2 pi i rand), MCfieldOnWave.m:231
        const double2 alpha = make_double2(s * cp, s * sp);
        if (SINGLE) {
            for (int j = lane; j < Q.nl; j += 32) {
                const C e0 = phaseatt<DIM, POL>(ev.x1, Q.l + 3 * j, Q.is_ff_l, Q);
                cb[j] = cmul(e0, to_c<C>(Wl[j]));
            }
            __syncwarp();
            for (int i = lane; i < nvt; i += 32) {
                const int vi = v0 + i;
                C sum = C{};
                for (int j = 0; j < Q.nl; ++j) {
                    const C af = to_c<C>(single_amp<DIM>(Q, vi, j, ev.x1));
                    const C t = cmul(af, cb[j]);
                    sum.x += t.x;
                    sum.y += t.y;
                }
                const C ev0 = phaseatt<DIM, POL>(ev.x1, Q.vs + 3 * vi, Q.is_ff_v, Q);
                const C t = cmul(ev0, sum);
                const double2 c = cmul(alpha, make_double2((double)t.x, (double)t.y));
                atomicAdd(&acc[i].x, c.x);
                atomicAdd(&acc[i].y, c.y);
            }
            __syncwarp();
        } else {
            C B = C{}, B2 = C{};
            for (int j = lane; j < Q.nl; j += 32) {
                C b, b2;
                nee_light<DIM, POL, C>(Q, j, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, b, b2);
                const C w = to_c<C>(Wl[j]);
                const C t = cmul(b, w), t2 = cmul(b2, w);
                B.x += t.x;
                B.y += t.y;
                B2.x += t2.x;
                B2.y += t2.y;
            }
            B = warp_csum(B);
            B2 = warp_csum(B2);
            for (int i = lane; i < nvt; i += 32) {
                C a, a0;
                nee_view<DIM, POL, C>(Q, v0 + i, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, a, a0);
                C t = cmul(a, B);
                if (Q.cbs) {
                    const C t2 = cmul(a0, B2);
                    t.x += t2.x;
                    t.y += t2.y;
                }
                const double2 c = cmul(alpha, make_double2((double)t.x, (double)t.y));
                atomicAdd(&acc[i].x, c.x);
                atomicAdd(&acc[i].y, c.y);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nvt; i += blockDim.x) {
        atomicAdd(&U[v0 + i].x, acc[i].x);
        atomicAdd(&U[v0 + i].y, acc[i].y);
    }
}

__global__ void onwave_finalize_kernel(const double2 *__restrict__ U, int nv, double norm, double2 *__restrict__ u)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
        u[i] = make_double2(norm * U[i].x, norm * U[i].y);
}

}  // namespace scmc
