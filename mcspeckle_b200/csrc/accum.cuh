// accum.cuh - field accumulation, covariance row generation and the CUDA-core
// Hermitian rank-k update.
//
// Field (MCfield.m:207-222): u[v,l] += sqrt(w/px) e^{2 pi i xi} t[v,l] with
//   single events  t = e_v0[v] e_l0[l]             (times af(v,l): applied per
//                                                   event for near-field
//                                                   sources, at finalisation for
//                                                   far-field ones)
//   multi events   t = a[v] b[l] (+ a0[v] b2[l]) / sqrt(2) with CBS.
// Each CTA owns a (view tile x light tile) block of u and a range of events;
// vectors for a sub-batch of events are staged in shared memory.
//
// Covariance (MCcov.m:232-263): every event is one Hermitian rank-1 update
// C += t t^H with t = sqrt(w/px) * (...) over the flattened index
// n = v + nv*l.  Rows t are generated per event, then contracted.
#pragma once

#include "nee.cuh"
#include "walk.cuh"

namespace scmc {

struct EventView {
    double x[3], ow[3], x1[3], w1[3];
    double wpx, xi, w0p;
};

// Load the data of event e (single: e is a path index).
template <int DIM, bool SINGLE>
__device__ __forceinline__ void load_event(const NeeParams &Q, const SingleRec &S, int64_t scap,
                                           const MultiRec &M, int64_t mcap, int64_t e, EventView &ev)
{
    int64_t p = SINGLE ? e : (int64_t)M.path[e];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ev.x1[k] = S.x1[k * scap + p];
        ev.w1[k] = S.w1[k * scap + p];
    }
    if (SINGLE) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { ev.x[k] = ev.x1[k]; ev.ow[k] = 0.0; }
        ev.wpx = S.wpx[p];
        ev.xi = S.xi[p];
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ev.x[k] = M.x[k * mcap + e];
            ev.ow[k] = M.ow[k * mcap + e];
        }
        ev.wpx = M.wpx[e];
        ev.xi = M.xi[e];
    }
    ev.w0p = first_dir_pdf<DIM>(Q, ev.w1);
}

// ---------------------------------------------------------------------------
// Field accumulation
// ---------------------------------------------------------------------------
constexpr int kFieldThreads = 256;
constexpr int kFieldEB = 8;       // events staged per sub-batch
constexpr int kFieldMaxTile = 1024;

template <typename A> struct acc_ptr;

// One CTA's share of the field sum: a tv x tl tile (`tile`) of views and
// lights over the events [e_begin, e_end) (path indices for singles, record
// indices for multiple scattering), added into U.
template <int DIM, int POL, bool SINGLE, typename AccT>
__device__ __forceinline__ void field_accum_body(const NeeParams &Q, const SingleRec &S, int64_t scap, const MultiRec &M,
                                                 int64_t mcap, int64_t e_begin, int64_t e_end, int tile, int tv, int tl,
                                                 int n_vtiles, AccT *__restrict__ U, int field_phase, int mean_mode)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sa = reinterpret_cast<C *>(smem_raw);          // [EB][tv]
    C *sa0 = sa + kFieldEB * tv;                        // [EB][tv]
    C *sb = sa0 + kFieldEB * tv;                        // [EB][tl]
    C *sb2 = sb + kFieldEB * tl;                        // [EB][tl]
    C *ssc = sb2 + kFieldEB * tl;                       // [EB] scale
    EventView *sev = reinterpret_cast<EventView *>(ssc + kFieldEB);  // [EB]

    const int v0 = (tile % n_vtiles) * tv;
    const int l0 = (tile / n_vtiles) * tl;
    const int nvt = min(tv, Q.nv - v0);
    const int nlt = min(tl, Q.nl - l0);
    const int nq = tv * tl;
    const int near_single = SINGLE && !(Q.is_ff_l && Q.is_ff_v);

    C acc[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[r] = C{};

    for (int64_t eb = e_begin; eb < e_end; eb += kFieldEB) {
        const int ne = (int)min((int64_t)kFieldEB, e_end - eb);
        if (threadIdx.x < ne) {
            EventView ev;
            load_event<DIM, SINGLE>(Q, S, scap, M, mcap, eb + threadIdx.x, ev);
            sev[threadIdx.x] = ev;
            double s = mean_mode ? ev.wpx : sqrt(ev.wpx);
            if (!SINGLE && Q.cbs) s *= 1.0 / sqrt(2.0);
            double2 rot = make_double2(1.0, 0.0);
            if (field_phase) {
                double sp, cp;
                sincos(2.0 * SCMC_PI * ev.xi, &sp, &cp);
                rot = make_double2(cp, sp);
            }
            ssc[threadIdx.x] = to_c<C>(make_double2(s * rot.x, s * rot.y));
        }
        __syncthreads();
        const int per = tv + tl;
        for (int idx = threadIdx.x; idx < kFieldEB * per; idx += kFieldThreads) {
            int k = idx / per, m = idx % per;
            if (k >= ne) continue;
            const EventView &ev = sev[k];
            if (m < tv) {
                int i = v0 + m;
                C a = C{}, a0 = C{};
                if (i < Q.nv) {
                    if (SINGLE) a = phaseatt<DIM, POL>(ev.x1, Q.vs + 3 * i, Q.is_ff_v, Q);
                    else nee_view<DIM, POL, C>(Q, i, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, a, a0);
                }
                sa[k * tv + m] = a;
                sa0[k * tv + m] = a0;
            } else {
                int j = l0 + (m - tv);
                C b = C{}, b2 = C{};
                if (j < Q.nl) {
                    if (SINGLE && mean_mode) b = phase_plain<DIM, POL>(ev.x1, Q.l + 3 * j, Q.is_ff_l, Q);
                    else if (SINGLE) b = phaseatt<DIM, POL>(ev.x1, Q.l + 3 * j, Q.is_ff_l, Q);
                    else nee_light<DIM, POL, C>(Q, j, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, b, b2);
                }
                sb[k * tl + (m - tv)] = b;
                sb2[k * tl + (m - tv)] = b2;
            }
        }
        __syncthreads();
        for (int k = 0; k < ne; ++k) {
            const C sc = ssc[k];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                int q = threadIdx.x + r * kFieldThreads;
                if (q >= nq) break;
                int vi = q % tv, lj = q / tv;
                C t = cmul(sa[k * tv + vi], sb[k * tl + lj]);
                if (!SINGLE && Q.cbs) {
                    C t2 = cmul(sa0[k * tv + vi], sb2[k * tl + lj]);
                    t.x += t2.x; t.y += t2.y;
                }
                if (near_single && vi < nvt && lj < nlt) {
                    double2 af = single_amp<DIM>(Q, v0 + vi, l0 + lj, sev[k].x1);
                    t = cmul(t, to_c<C>(af));
                }
                C c = cmul(sc, t);
                acc[r].x += c.x;
                acc[r].y += c.y;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        int q = threadIdx.x + r * kFieldThreads;
        if (q >= nq) break;
        int vi = q % tv, lj = q / tv;
        if (vi < nvt && lj < nlt) {
            int64_t o = 2 * ((int64_t)(v0 + vi) + (int64_t)Q.nv * (l0 + lj));
            atomicAdd(&U[o], (AccT)acc[r].x);
            atomicAdd(&U[o + 1], (AccT)acc[r].y);
        }
    }
}

template <int DIM, int POL, bool SINGLE, typename AccT>
__global__ void __launch_bounds__(kFieldThreads)
field_accum_kernel(const __grid_constant__ NeeParams Q, SingleRec S, int64_t scap, MultiRec M, int64_t mcap, int64_t n_events,
                   int tv, int tl, int n_vtiles, int64_t ev_per_cta, AccT *__restrict__ U, int field_phase,
                   int mean_mode = 0)
{
    const int64_t e_begin = (int64_t)blockIdx.y * ev_per_cta;
    const int64_t e_end = min(n_events, e_begin + ev_per_cta);
    field_accum_body<DIM, POL, SINGLE, AccT>(Q, S, scap, M, mcap, e_begin, e_end, (int)blockIdx.x, tv, tl, n_vtiles, U,
                                             field_phase, mean_mode);
}

// Many field requests in one launch (the request server's packs): CTA b
// takes job jobs[b] - request, tile, event range, singles or multiple
// scattering - with that request's NEE parameters and accumulators.
struct PackJob {
    int req, tile, single, pad;
    int64_t e_begin, e_end;
};
struct PackTiling {
    int tv, tl, n_vtiles, pad;
    int64_t acc_s, acc_m;  // offsets (AccT units) of the request's accumulators in the pack's arena
};

template <int DIM, int POL, typename AccT>
__global__ void __launch_bounds__(kFieldThreads)
field_accum_packed_kernel(const NeeParams *__restrict__ Qs, const PackTiling *__restrict__ tiling,
                          const PackJob *__restrict__ jobs, SingleRec S, int64_t scap, MultiRec M, int64_t mcap,
                          AccT *__restrict__ arena)
{
    const PackJob j = jobs[blockIdx.x];
    const PackTiling t = tiling[j.req];
    const NeeParams &Q = Qs[j.req];
    if (j.single)
        field_accum_body<DIM, POL, true, AccT>(Q, S, scap, M, mcap, j.e_begin, j.e_end, j.tile, t.tv, t.tl, t.n_vtiles,
                                               arena + t.acc_s, 1, 0);
    else
        field_accum_body<DIM, POL, false, AccT>(Q, S, scap, M, mcap, j.e_begin, j.e_end, j.tile, t.tv, t.tl,
                                                t.n_vtiles, arena + t.acc_m, 1, 0);
}

// u = norm * (A o Us + Um), A = af(l.v) for far-field singles, else 1.
template <int DIM, typename AccT>
__device__ __forceinline__ void field_finalize_at(const NeeParams &Q, const AccT *__restrict__ Us,
                                                  const AccT *__restrict__ Um, double norm, double2 *__restrict__ u,
                                                  int64_t q)
{
    int i = (int)(q % Q.nv), j = (int)(q / Q.nv);
    double2 s = make_double2((double)Us[2 * q], (double)Us[2 * q + 1]);
    if (Q.is_ff_l && Q.is_ff_v) {
        double2 af = evalampfunc<DIM>(dot3<DIM>(Q.l + 3 * j, Q.v + 3 * i), Q.pf);
        s = cmul(af, s);
    }
    u[q] = make_double2(norm * (s.x + (double)Um[2 * q]), norm * (s.y + (double)Um[2 * q + 1]));
}

template <int DIM, typename AccT>
__global__ void field_finalize_kernel(const __grid_constant__ NeeParams Q, const AccT *__restrict__ Us, const AccT *__restrict__ Um,
                                      double norm, double2 *__restrict__ u)
{
    int64_t n = (int64_t)Q.nv * Q.nl;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        field_finalize_at<DIM, AccT>(Q, Us, Um, norm, u, q);
}

// The finalisation of a pack: blockIdx.y = request, its output at outs[r].
template <int DIM, typename AccT>
__global__ void field_finalize_packed_kernel(const NeeParams *__restrict__ Qs, const PackTiling *__restrict__ tiling,
                                             const AccT *__restrict__ arena, const double *__restrict__ norms,
                                             double2 *const *__restrict__ outs)
{
    const int r = blockIdx.y;
    const NeeParams &Q = Qs[r];
    const PackTiling t = tiling[r];
    const int64_t n = (int64_t)Q.nv * Q.nl;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        field_finalize_at<DIM, AccT>(Q, arena + t.acc_s, arena + t.acc_m, norms[r], outs[r], q);
}

// ---------------------------------------------------------------------------
// Covariance: per-event rows t (flattened n = v + nv*l), row-major [E][N]
// ---------------------------------------------------------------------------
template <int DIM, int POL, bool SINGLE>
__global__ void __launch_bounds__(256)
cov_rows_kernel(const __grid_constant__ NeeParams Q, SingleRec S, int64_t scap, MultiRec M, int64_t mcap, int64_t e_begin,
                int64_t n_ev, int eb, typename cplx_t<typename std::conditional<POL == P64, double, float>::type>::type *__restrict__ T)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nv = Q.nv, nl = Q.nl;
    C *sa = reinterpret_cast<C *>(smem_raw);  // [eb][nv]
    C *sa0 = sa + eb * nv;
    C *sb = sa0 + eb * nv;                    // [eb][nl]
    C *sb2 = sb + eb * nl;
    double *ssc = reinterpret_cast<double *>(sb2 + eb * nl);   // [eb]
    EventView *sev = reinterpret_cast<EventView *>(ssc + eb + (eb & 1));

    const int64_t r0 = (int64_t)blockIdx.x * eb;
    const int ne = (int)min((int64_t)eb, n_ev - r0);
    if (ne <= 0) return;
    if (threadIdx.x < ne) {
        EventView ev;
        load_event<DIM, SINGLE>(Q, S, scap, M, mcap, e_begin + r0 + threadIdx.x, ev);
        sev[threadIdx.x] = ev;
        ssc[threadIdx.x] = sqrt(ev.wpx);
    }
    __syncthreads();
    const int per = nv + nl;
    for (int idx = threadIdx.x; idx < ne * per; idx += blockDim.x) {
        int k = idx / per, m = idx % per;
        const EventView &ev = sev[k];
        if (m < nv) {
            C a = C{}, a0 = C{};
            if (SINGLE) a = phaseatt<DIM, POL>(ev.x1, Q.vs + 3 * m, Q.is_ff_v, Q);
            else nee_view<DIM, POL, C>(Q, m, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, a, a0);
            sa[k * nv + m] = a;
            sa0[k * nv + m] = a0;
        } else {
            int j = m - nv;
            C b = C{}, b2 = C{};
            if (SINGLE) b = phaseatt<DIM, POL>(ev.x1, Q.l + 3 * j, Q.is_ff_l, Q);
            else nee_light<DIM, POL, C>(Q, j, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, b, b2);
            sb[k * nl + j] = b;
            sb2[k * nl + j] = b2;
        }
    }
    __syncthreads();
    const int64_t N = (int64_t)nv * nl;
    for (int k = 0; k < ne; ++k) {
        const double sc = ssc[k];
        C *row = T + (r0 + k) * N;
        for (int64_t q = threadIdx.x; q < N; q += blockDim.x) {
            int vi = (int)(q % nv), lj = (int)(q / nv);
            C t = cmul(sa[k * nv + vi], sb[k * nl + lj]);
            if (!SINGLE && Q.cbs) {
                C t2 = cmul(sa0[k * nv + vi], sb2[k * nl + lj]);
                t.x += t2.x; t.y += t2.y;
            }
            if (SINGLE) t = cmul(t, to_c<C>(single_amp<DIM>(Q, vi, lj, sev[k].x1)));
            row[q] = cscale<C>(t, sc);
        }
    }
}

// C[i][j] += sum_e T[e][i] conj(T[e][j]) over the upper-triangular tile list.
// 256 threads as 16 x 16, each owning RPT x RPT entries strided by 16.
template <typename R, typename A, int RPT, int BK>
__global__ void __launch_bounds__(256)
herk_cc_kernel(const typename cplx_t<R>::type *__restrict__ T, int64_t n_ev, int N,
               const int2 *__restrict__ tiles, typename cplx_t<A>::type *__restrict__ Cacc)
{
    using Cx = typename cplx_t<R>::type;
    constexpr int TILE = 16 * RPT;
    __shared__ Cx As[BK][TILE];
    __shared__ Cx Bs[BK][TILE];
    const int2 t = tiles[blockIdx.x];
    const int i0 = t.x * TILE, j0 = t.y * TILE;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    Cx acc[RPT][RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int c = 0; c < RPT; ++c) acc[r][c] = Cx{};

    for (int64_t e0 = 0; e0 < n_ev; e0 += BK) {
        for (int idx = threadIdx.x; idx < BK * TILE; idx += 256) {
            int k = idx / TILE, c = idx % TILE;
            int64_t e = e0 + k;
            Cx a = Cx{}, b = Cx{};
            if (e < n_ev) {
                if (i0 + c < N) a = T[e * N + i0 + c];
                if (j0 + c < N) b = T[e * N + j0 + c];
            }
            As[k][c] = a;
            Bs[k][c] = b;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            Cx a[RPT], b[RPT];
#pragma unroll
            for (int r = 0; r < RPT; ++r) a[r] = As[k][ty + 16 * r];
#pragma unroll
            for (int c = 0; c < RPT; ++c) b[c] = Bs[k][tx + 16 * c];
#pragma unroll
            for (int r = 0; r < RPT; ++r)
#pragma unroll
                for (int c = 0; c < RPT; ++c) {
                    // a * conj(b)
                    acc[r][c].x += a[r].x * b[c].x + a[r].y * b[c].y;
                    acc[r][c].y += a[r].y * b[c].x - a[r].x * b[c].y;
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int c = 0; c < RPT; ++c) {
            int i = i0 + ty + 16 * r, j = j0 + tx + 16 * c;
            if (i < N && j < N) {
                auto &o = Cacc[(int64_t)i * N + j];
                o.x += (A)acc[r][c].x;
                o.y += (A)acc[r][c].y;
            }
        }
}

// Full nv x nv x nl x nl output from the Hermitian accumulator.
// layout 0: C[i][j] complex row-major; layout 1: real-expanded D[2i+p][j].
template <typename A>
__global__ void cov_finalize_kernel(const A *__restrict__ Cacc, const A *__restrict__ Cacc2, int layout, int nv, int nl,
                                    double scale, double2 *__restrict__ out)
{
    // Cacc2 (may be null): a second partial accumulator of the same layout, added in.
    const int64_t N = (int64_t)nv * nl;
    const int64_t total = N * N;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        int64_t v1 = q % nv, r = q / nv;
        int64_t v2 = r % nv; r /= nv;
        int64_t l1 = r % nl, l2 = r / nl;
        int64_t i1 = v1 + nv * l1, i2 = v2 + nv * l2;
        bool flip = i1 > i2;
        int64_t a = flip ? i2 : i1, b = flip ? i1 : i2;
        double re, im;
        const int64_t ore = layout == 0 ? 2 * (a * N + b) : (2 * a) * N + b;
        const int64_t oim = layout == 0 ? ore + 1 : ore + N;
        re = (double)Cacc[ore];
        im = (double)Cacc[oim];
        if (Cacc2) {
            re += (double)Cacc2[ore];
            im += (double)Cacc2[oim];
        }
        if (flip) im = -im;
        if (i1 == i2) im = 0.0;  // sum of |t_i|^2: real, as the reference's products give
        out[q] = make_double2(scale * re, scale * im);
    }
}

}  // namespace scmc
