// field_tc.cuh - the field accumulation of MCfield.m:207-222 on tcgen05.
//
// u[v,l] = sum_e alpha_e (a_e[v] b_e[l] + a0_e[v] b2_e[l])   (CBS: /sqrt2 in alpha)
// is a complex GEMM over events.  With K = 2 real columns per term:
//   A[2v]   = ( Re t, -Im t),  A[2v+1] = ( Im t, Re t ),   t = alpha * a[v]
//   B[l]    = ( Re b,  Im b)
//   D = A B^T:  D[2v][l] = Re u,  D[2v+1][l] = Im u.
// Single-scattering events of far-field lights and views are the rank-1
// terms alpha e_v0[v] e_l0[l]; their amplitude af(l.v) multiplies the sum at
// finalisation.  The GEMM is herk_tc_kernel with a separate B operand and the
// full tile list.
#pragma once

#include "herk_tc.cuh"

namespace scmc {

struct FieldTcPlan {
    int nv, nl, terms;       // terms per event: 1, or 2 with CBS (multiple scattering)
    bool split;
    int ksplit;              // K slices per output tile (D holds ksplit partial sums)
    int64_t events_per_chunk, K;
    std::vector<int2> tiles;
};

struct FieldTcOps {
    __half *ahi, *alo, *b;
    int2 *tiles;
    int *err;
    CUtensorMap m_ahi, m_alo, m_b;
    int n_tiles;
};

// sms: multiprocessors; the K split fills them when the output has few tiles.
// chunk_bytes bounds the operand memory of one chunk of events.
inline FieldTcPlan field_tc_plan(int nv, int nl, int terms, bool split, int sms, size_t chunk_bytes = (size_t)1 << 30,
                                 int ksplit = 0)
{
    FieldTcPlan p;
    p.nv = nv;
    p.nl = nl;
    p.terms = terms;
    p.split = split;
    // bytes per event: A (hi [+ lo]) 2nv rows and B nl rows, 2 fp16 per term
    const int64_t per = (int64_t)terms * 4 * ((split ? 2 : 1) * 2 * (int64_t)nv + nl);
    int64_t e = (int64_t)chunk_bytes / std::max<int64_t>(per, 1);
    e = std::max<int64_t>(32, std::min<int64_t>(e, (int64_t)1 << 18));
    e = (e / 32) * 32;
    p.events_per_chunk = e;
    p.K = 2 * (int64_t)terms * e;
    const int n_tm = (2 * nv + TC_BM - 1) / TC_BM, n_tn = (nl + TC_BN - 1) / TC_BN;
    for (int tn = 0; tn < n_tn; ++tn)
        for (int tm = 0; tm < n_tm; ++tm) p.tiles.push_back(make_int2(tm, tn));
    const int nt = (int)p.tiles.size();
    p.ksplit = std::max(1, std::min(sms / std::max(nt, 1), (int)(p.K / TC_BK / 8)));
    if (ksplit > 0) p.ksplit = std::max(1, std::min(ksplit, (int)(p.K / TC_BK)));
    return p;
}

inline size_t field_tc_bytes(const FieldTcPlan &p)
{
    const size_t a = tc_align((size_t)2 * p.nv * p.K * sizeof(__half));
    const size_t b = tc_align((size_t)p.nl * p.K * sizeof(__half));
    return (p.split ? 2 : 1) * a + b + tc_align(p.tiles.size() * sizeof(int2)) + 1024;
}

inline FieldTcOps field_tc_ops(const FieldTcPlan &p, void *mem, cudaStream_t st)
{
    FieldTcOps o{};
    char *base = reinterpret_cast<char *>(mem);
    const size_t a = tc_align((size_t)2 * p.nv * p.K * sizeof(__half));
    const size_t b = tc_align((size_t)p.nl * p.K * sizeof(__half));
    o.ahi = reinterpret_cast<__half *>(base);
    o.alo = p.split ? reinterpret_cast<__half *>(base + a) : o.ahi;
    char *q = base + (p.split ? 2 : 1) * a;
    o.b = reinterpret_cast<__half *>(q);
    o.tiles = reinterpret_cast<int2 *>(q + b);
    o.err = reinterpret_cast<int *>(q + b + tc_align(p.tiles.size() * sizeof(int2)));
    o.n_tiles = (int)p.tiles.size();
    if (cudaMemcpyAsync(o.tiles, p.tiles.data(), p.tiles.size() * sizeof(int2), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemsetAsync(o.err, 0, sizeof(int), st) != cudaSuccess)
        throw std::runtime_error("field tensor-core operand set-up failed");
    const uint64_t K = (uint64_t)p.K;
    o.m_ahi = tc_map(o.ahi, K, 2 * (uint64_t)p.nv, K * 2, TC_BM);
    o.m_alo = tc_map(o.alo, K, 2 * (uint64_t)p.nv, K * 2, TC_BM);
    o.m_b = tc_map(o.b, K, (uint64_t)p.nl, K * 2, TC_BN);
    return o;
}

constexpr int kFtRows = 128;  // phase rows (views then lights) staged per pass

inline size_t field_tc_rows_smem()
{
    return sizeof(float2) * (2 * kFtRows * 33 + 32) + sizeof(EventView) * 32 + 16;
}

// Operand rows of one chunk: one CTA per 32 events (lane = event when
// writing, so a row segment is 32 consecutive 4- or 8-byte words).  Rows are
// produced kFtRows at a time: m < nv are views (scaled by alpha), m >= nv
// lights.  SINGLE is used only for far-field lights and views.
template <int DIM, bool SINGLE, bool SPLIT>
__global__ void __launch_bounds__(256)
field_tc_rows_kernel(const __grid_constant__ NeeParams Q, SingleRec S, int64_t scap, MultiRec M, int64_t mcap, int64_t e0, int64_t n_ev,
                     int terms, int64_t K, __half *__restrict__ Ahi, __half *__restrict__ Alo,
                     __half *__restrict__ Bm, int field_phase)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nv = Q.nv, nl = Q.nl;
    float2 *sp = reinterpret_cast<float2 *>(smem_raw);   // [kFtRows][33]
    float2 *sq = sp + kFtRows * 33;                        // [kFtRows][33]
    float2 *salpha = sq + kFtRows * 33;                    // [32]
    EventView *sev = reinterpret_cast<EventView *>(salpha + 32);

    const int64_t g0 = (int64_t)blockIdx.x * 32;
    const int ne = (int)max((int64_t)0, min((int64_t)32, n_ev - g0));
    if (threadIdx.x < 32) {
        EventView ev{};
        float2 al = make_float2(0.f, 0.f);
        if (threadIdx.x < ne) {
            load_event<DIM, SINGLE>(Q, S, scap, M, mcap, e0 + g0 + threadIdx.x, ev);
            double s = sqrt(ev.wpx);
            if (!SINGLE && Q.cbs) s *= 1.0 / sqrt(2.0);
            double sn = 0.0, cs = 1.0;
            if (field_phase) sincos(2.0 * SCMC_PI * ev.xi, &sn, &cs);
            al = make_float2((float)(s * cs), (float)(s * sn));
        }
        sev[threadIdx.x] = ev;
        salpha[threadIdx.x] = al;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t col = 2 * (int64_t)terms * (g0 + lane);
    const int total = nv + nl;
    for (int m0 = 0; m0 < total; m0 += kFtRows) {
        const int mc = min(kFtRows, total - m0);
        // lanes take consecutive directions of one event (converged marches
        // in a heterogeneous medium: one event's rays have similar lengths)
        for (int idx = threadIdx.x; idx < 32 * mc; idx += blockDim.x) {
            const int k = idx / mc, r = idx - k * mc, m = m0 + r;
            float2 p = make_float2(0.f, 0.f), q = make_float2(0.f, 0.f);
            if (k < ne) {
                const EventView &ev = sev[k];
                if (m < nv) {
                    if (SINGLE) p = phaseatt<DIM, PMIX>(ev.x1, Q.vs + 3 * m, Q.is_ff_v, Q);
                    else nee_view<DIM, PMIX, float2>(Q, m, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, p, q);
                    p = cmul(p, salpha[k]);
                    q = cmul(q, salpha[k]);
                } else {
                    const int j = m - nv;
                    if (SINGLE) p = phaseatt<DIM, PMIX>(ev.x1, Q.l + 3 * j, Q.is_ff_l, Q);
                    else nee_light<DIM, PMIX, float2>(Q, j, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, p, q);
                }
            }
            sp[r * 33 + k] = p;
            sq[r * 33 + k] = q;
        }
        __syncthreads();
        for (int r = warp; r < mc; r += 8) {
            const int m = m0 + r;
            const float2 v0 = sp[r * 33 + lane], v1 = sq[r * 33 + lane];
            if (m < nv) {
                const __half h0r = __float2half_rn(v0.x), h0i = __float2half_rn(v0.y);
                const __half h1r = __float2half_rn(v1.x), h1i = __float2half_rn(v1.y);
                __half *e = Ahi + (int64_t)(2 * m) * K + col, *o = e + K;
                if (terms == 2) {
                    __half2 ev2[2] = {__halves2half2(h0r, __hneg(h0i)), __halves2half2(h1r, __hneg(h1i))};
                    __half2 od2[2] = {__halves2half2(h0i, h0r), __halves2half2(h1i, h1r)};
                    *reinterpret_cast<uint2 *>(e) = *reinterpret_cast<uint2 *>(ev2);
                    *reinterpret_cast<uint2 *>(o) = *reinterpret_cast<uint2 *>(od2);
                } else {
                    *reinterpret_cast<__half2 *>(e) = __halves2half2(h0r, __hneg(h0i));
                    *reinterpret_cast<__half2 *>(o) = __halves2half2(h0i, h0r);
                }
                if (SPLIT) {
                    const __half l0r = __float2half_rn(v0.x - __half2float(h0r));
                    const __half l0i = __float2half_rn(v0.y - __half2float(h0i));
                    const __half l1r = __float2half_rn(v1.x - __half2float(h1r));
                    const __half l1i = __float2half_rn(v1.y - __half2float(h1i));
                    __half *le = Alo + (int64_t)(2 * m) * K + col, *lo = le + K;
                    if (terms == 2) {
                        __half2 ev2[2] = {__halves2half2(l0r, __hneg(l0i)), __halves2half2(l1r, __hneg(l1i))};
                        __half2 od2[2] = {__halves2half2(l0i, l0r), __halves2half2(l1i, l1r)};
                        *reinterpret_cast<uint2 *>(le) = *reinterpret_cast<uint2 *>(ev2);
                        *reinterpret_cast<uint2 *>(lo) = *reinterpret_cast<uint2 *>(od2);
                    } else {
                        *reinterpret_cast<__half2 *>(le) = __halves2half2(l0r, __hneg(l0i));
                        *reinterpret_cast<__half2 *>(lo) = __halves2half2(l0i, l0r);
                    }
                }
            } else {
                __half *b = Bm + (int64_t)(m - nv) * K + col;
                const __half2 b0 = __halves2half2(__float2half_rn(v0.x), __float2half_rn(v0.y));
                if (terms == 2) {
                    __half2 bb[2] = {b0, __halves2half2(__float2half_rn(v1.x), __float2half_rn(v1.y))};
                    *reinterpret_cast<uint2 *>(b) = *reinterpret_cast<uint2 *>(bb);
                } else {
                    *reinterpret_cast<__half2 *>(b) = b0;
                }
            }
        }
        __syncthreads();
    }
}

// u = norm * (Ds' + Dm), summing the K slices of the real-expanded
// accumulators D[ks][2v+p][l] in slice order.  ds_slices > 0: the singles are
// far-field tensor-core sums, multiplied here by af(l.v); ds_slices == 0: the
// singles are CUDA-core sums in complex layout (index 2(v + nv l)).
template <int DIM>
__global__ void field_tc_finalize_kernel(const __grid_constant__ NeeParams Q, const double *__restrict__ Ds, int ds_slices,
                                         const double *__restrict__ Dm, int dm_slices, double norm,
                                         double2 *__restrict__ u)
{
    const int64_t n = (int64_t)Q.nv * Q.nl, slice = 2 * n;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % Q.nv), j = (int)(q / Q.nv);
        const int64_t re = (int64_t)(2 * i) * Q.nl + j, im = re + Q.nl;
        double2 s = make_double2(0.0, 0.0), m = make_double2(0.0, 0.0);
        if (ds_slices > 0) {
            for (int k = 0; k < ds_slices; ++k) {
                s.x += Ds[k * slice + re];
                s.y += Ds[k * slice + im];
            }
            s = cmul(evalampfunc<DIM>(dot3<DIM>(Q.l + 3 * j, Q.v + 3 * i), Q.pf), s);
        } else {
            s = make_double2(Ds[2 * q], Ds[2 * q + 1]);
        }
        for (int k = 0; k < dm_slices; ++k) {
            m.x += Dm[k * slice + re];
            m.y += Dm[k * slice + im];
        }
        u[q] = make_double2(norm * (s.x + m.x), norm * (s.y + m.y));
    }
}

}  // namespace scmc
