// walk.cuh - the random walk of MCfield.m:112-250 / MCcov.m:112-290.
//
// One lane walks one path at a time and takes the next path as soon as its
// current one leaves the box or is killed, so every lane stays busy until
// the batch runs out (a flattened event loop: all lanes run the same loop
// body).  The walk is FP64 in every precision mode, so the three modes see
// identical paths for the same seed.
//
// Two passes share the walk: the count pass stores the number of events of
// every path; after an exclusive scan the record pass re-walks each path
// (Philox makes it identical) and writes its events at fixed offsets, in
// path order.  The first event of a path goes to the single-scattering
// record (index = path), the others to the multiple-scattering records.
#pragma once

#include "common.cuh"
#include "hgrid.cuh"

namespace scmc {

// Single-scattering records: one per path (SoA, stride = cap).
struct SingleRec {
    double *x1;   // 3*cap: first scatterer
    double *w1;   // 3*cap: first outgoing direction
    double *wpx;  // weight/px at the first event
    double *xi;   // random-phase uniform of the first event (field)
    int32_t *nev; // events of the path
};

// Multiple-scattering records (SoA, stride = cap).
struct MultiRec {
    double *x;     // 3*cap: event position
    double *ow;    // 3*cap: incoming direction
    double *wpx;   // weight/px
    double *xi;    // random-phase uniform (field)
    int32_t *path; // path index within the batch
    int32_t *plen; // pL (>= 2)
};

struct WalkState {
    double x[3], w[3], ow[3];
    double px, weight;
    int pL;
    bool dead;   // dropped before its first event (voxel-medium plane launch missed)
};

// smpWoodcock.m:1-15: delta tracking against max(sigt) along v from x.
template <int DIM>
__device__ __forceinline__ double hg_woodcock(const HGrid &g, const double *x, const double *v, PathRng &r)
{
    double d = 0.0, nx[3] = {0, 0, 0};
    for (int guard = 0; guard < (1 << 24); ++guard) {
        d = d - log(1 - r.rand()) / g.sigt_max;
#pragma unroll
        for (int k = 0; k < DIM; ++k) nx[k] = x[k] + d * v[k];
        if (hg_outside(g, nx)) break;
        const double sg = g.trilinear ? hg_sigma_tri<DIM>(g, nx) : g.sigt[hg_find_bin(g, nx, nullptr, nullptr)];
        if (r.rand() <= (sg / g.sigt_max)) break;
    }
    return d;
}

// First scatterer in the voxel medium (MCCovHetro.m:90-115).  Returns false
// when the path is dropped (plane launch missing the box).
template <int DIM>
__device__ __forceinline__ bool hg_first_scatter(const WalkParams &P, PathRng &r, WalkState &s)
{
    const HGrid &g = P.hg;
    if (P.smp_flg == 1) {
        // smpicdf.m over invCDFvec.m: voxel = count of cdf values below the
        // upper edge of hist bin i, i = ceil(rand * N)
        int64_t i = (int64_t)ceil(r.rand() * (double)g.n_icdf);
        i = i < 1 ? 1 : i;
        int64_t cnt;
        if (g.n_vox == 1 || i >= g.n_icdf) {
            cnt = g.n_vox;
        } else {
            const double edge = g.cdf_lo + (double)i * g.cdf_step;
            int64_t lo = 0, hi = g.n_vox;  // first k with cdf[k] >= edge
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (g.cdf[mid] < edge) lo = mid + 1;
                else hi = mid;
            }
            cnt = lo;
        }
        int64_t rem = (cnt < 1 ? 1 : cnt) - 1;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            const int64_t ii = rem % g.nb[k];
            rem /= g.nb[k];
            const double bmn = g.bmin[k] + g.bbin[k] * (double)ii;
            s.x[k] = r.rand() * g.bbin[k] + bmn;
        }
        s.px = g.inv_V;
        if (g.trilinear) {
            // the voxel pick samples sigma_nearest(x) / V; the medium is
            // sigma_trilinear: px carries their ratio (a zero trilinear
            // sigma gives px = inf, a weight of 0)
            s.px = g.inv_V * g.sigt[hg_find_bin(g, s.x, nullptr, nullptr)] / hg_sigma_tri<DIM>(g, s.x);
        }
        return !hg_outside(g, s.x);
    }
    // expSmpXHetro.m:1-31: launch from a plane across meanl, enter the box,
    // one Woodcock flight; px = |transmittance|^2 / lrad^(dim-1)
    double mx = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) mx = fmax(mx, fmax(fabs(g.bmax[k]), fabs(g.bmin[k])));
    double q[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < DIM - 1; ++k) q[k] = (r.rand() - 0.5) * g.lrad;
    double x0[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        double a = 0.0;
#pragma unroll
        for (int c = 0; c < DIM - 1; ++c) a += g.basis[k + DIM * c] * q[c];
        x0[k] = a - P.meanl[k] * mx * DIM;
    }
    // cubeProj.m:1-18
    const double thr = 1.0000000000000004e-07;
    double d = -INFINITY;
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
        const double den = fmax(fabs(P.meanl[j]), thr);
        const double bd = (P.meanl[j] <= 0) ? (x0[j] - g.bmax[j]) / den : (-x0[j] + g.bmin[j]) / den;
        d = fmax(d, bd);
    }
    if (!(d >= 0)) return false;
    double ep = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) ep = fmax(ep, fabs(g.bmax[k] - g.bmin[k]));
    ep = 1.0000000000000002e-04 * ep;
#pragma unroll
    for (int k = 0; k < DIM; ++k) s.x[k] = x0[k] + (d + ep) * P.meanl[k];
    if (hg_outside(g, s.x)) return false;
    const double dw = hg_woodcock<DIM>(g, s.x, P.meanl, r);
#pragma unroll
    for (int k = 0; k < DIM; ++k) s.x[k] = s.x[k] + dw * P.meanl[k];
    if (hg_outside(g, s.x)) return false;
    const double wbdv = hg_optical_depth<DIM>(g, s.x, P.meanl, 1.0e12);
    const double e = exp(-(1.0 / 2.0 * wbdv));
    s.px = e * e / pow(g.lrad, (double)(DIM - 1));
    return true;
}

// Initialise a path: first scatterer (MCfield.m:118-125) and first
// direction (MCfield.m:149-155).  Returns false for a dropped path (voxel
// medium only), which the walk records as one event of zero weight.
template <int DIM>
__device__ __forceinline__ bool path_init(const WalkParams &P, PathRng &r, WalkState &s)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) { s.x[k] = 0.0; s.w[k] = 0.0; s.ow[k] = 0.0; }
    s.dead = false;
    if (P.hetero) {
        const bool ok = hg_first_scatter<DIM>(P, r, s);
        s.dead = !ok;
        if (!ok) {
#pragma unroll
            for (int k = 0; k < 3; ++k) { s.x[k] = k < DIM ? 0.5 * (P.box_min[k] + P.box_max[k]) : 0.0; s.w[k] = P.meanl[k]; }
            s.px = 1.0;
            s.pL = 0;
            s.weight = 0.0;
            return false;
        }
        if (!P.has_pf0) randn_dir<DIM>(s.w, r);
        else smpampfunc_general<DIM>(P.meanl, P.pf0, s.w, r);
        s.pL = 0;
        s.weight = hg_albedo(P.hg, s.x);
        return true;
    }
    if (P.smp_flg == 1) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) s.x[k] = r.rand() * P.box_w[k] + P.box_min[k];
        s.px = 1.0;
    } else {
        exp_smp_x<DIM>(P, s.x, &s.px, r);
    }
    if (!P.has_pf0) randn_dir<DIM>(s.w, r);
    else smpampfunc_general<DIM>(P.meanl, P.pf0, s.w, r);
    s.pL = 0;
    s.weight = P.albedo;
    return true;
}

// After the event at s.x has been recorded: free flight, box exit, roulette
// and the next direction (MCfield.m:225-246).  Returns false when the path
// ends.
template <int DIM>
__device__ __forceinline__ bool path_advance(const WalkParams &P, PathRng &r, WalkState &s)
{
    if (s.dead) return false;  // a dropped path is one zero-weight event
    if (P.hetero) {
        // MCCovHetro.m:238-254: Woodcock flight, voxel albedo
        const double d = hg_woodcock<DIM>(P.hg, s.x, s.w, r);
#pragma unroll
        for (int k = 0; k < DIM; ++k) s.x[k] = s.x[k] + d * s.w[k];
        if (hg_outside(P.hg, s.x)) return false;
        if (s.weight < kKillThr) {
            if (r.rand() > hg_albedo(P.hg, s.x)) return false;
        } else {
            s.weight = s.weight * hg_albedo(P.hg, s.x);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) s.ow[k] = s.w[k];
        smpampfunc_general<DIM>(s.ow, P.pf, s.w, r);
        return true;
    }
    double d = -log(-r.rand() + 1.0) / P.sigt;
    bool out = false;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        s.x[k] = s.x[k] + d * s.w[k];
        out |= (s.x[k] > P.box_max[k]) || (s.x[k] < P.box_min[k]);
    }
    if (out) return false;
    if (s.weight < kKillThr) {
        if (r.rand() > P.albedo) return false;
    } else {
        s.weight = s.weight * P.albedo;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) s.ow[k] = s.w[k];
    smpampfunc_general<DIM>(s.ow, P.pf, s.w, r);
    return true;
}

// Pass 1: events per path.
template <int DIM>
__global__ void __launch_bounds__(128) walk_count_kernel(const __grid_constant__ WalkParams P, int32_t *__restrict__ counts,
                                                         unsigned long long *__restrict__ next_path,
                                                         int *__restrict__ err)
{
    PathRng r;
    WalkState s;
    int64_t p = -1;
    int n = 0;
    for (;;) {
        if (p < 0) {
            p = (int64_t)atomicAdd(next_path, 1ull);
            if (p >= P.n_paths) break;
            r.init(P.key0, P.key1, P.path_base + (uint64_t)p);
            path_init<DIM>(P, r, s);
            n = 0;
        }
        ++n;
        if (P.want_phase) (void)r.rand();  // MCfield.m:220
        bool alive = path_advance<DIM>(P, r, s);
        if (alive && P.max_events > 0 && n >= P.max_events) {
            atomicExch(err, 1);
            alive = false;
        }
        if (!alive) {
            counts[p] = n;
            p = -1;
        }
    }
}

// Pass 2: records.  moff[p] = index of the first multiple-scattering record
// of path p (exclusive scan of counts[p] - 1).
template <int DIM>
__global__ void __launch_bounds__(128) walk_record_kernel(const __grid_constant__ WalkParams P, const int64_t *__restrict__ moff,
                                                          SingleRec S, int64_t scap, MultiRec M,
                                                          int64_t mcap, unsigned long long *__restrict__ next_path)
{
    PathRng r;
    WalkState s;
    int64_t p = -1;
    int64_t mo = 0;
    for (;;) {
        if (p < 0) {
            p = (int64_t)atomicAdd(next_path, 1ull);
            if (p >= P.n_paths) break;
            r.init(P.key0, P.key1, P.path_base + (uint64_t)p);
            path_init<DIM>(P, r, s);
            mo = moff[p];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                S.x1[k * scap + p] = s.x[k];
                S.w1[k * scap + p] = s.w[k];
            }
        }
        ++s.pL;
        double xi = P.want_phase ? r.rand() : 0.0;
        double wpx = s.weight / s.px;
        if (s.pL == 1) {
            S.wpx[p] = wpx;
            S.xi[p] = xi;
        } else {
            int64_t e = mo + (s.pL - 2);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                M.x[k * mcap + e] = s.x[k];
                M.ow[k * mcap + e] = s.ow[k];
            }
            M.wpx[e] = wpx;
            M.xi[e] = xi;
            M.path[e] = (int32_t)p;
            M.plen[e] = s.pL;
        }
        bool alive = path_advance<DIM>(P, r, s);
        if (alive && P.max_events > 0 && s.pL >= P.max_events) alive = false;
        if (!alive) {
            S.nev[p] = s.pL;
            p = -1;
        }
    }
}

// One pass for the reduced-precision modes: each lane walks paths taken from
// an atomic counter and writes its records as it goes.  A path's single
// record sits at its own index; the multiple-scattering records of a warp's
// lanes at one step get consecutive slots from one atomicAdd by the warp
// (ballot, popc), so the records are in no fixed order (every consumer reads
// an event's path from M.path).  slots[0] counts paths handed out, slots[1]
// the multiple-scattering events; records past mcap are counted but not
// written, and the host then walks the batch again with room for all of
// them (Philox regenerates the same paths).
template <int DIM>
__global__ void __launch_bounds__(128) walk_onepass_kernel(const __grid_constant__ WalkParams P, SingleRec S,
                                                           int64_t scap, MultiRec M, int64_t mcap,
                                                           unsigned long long *__restrict__ slots,
                                                           int *__restrict__ err)
{
    PathRng r;
    WalkState s;
    int64_t p = -1;
    bool active = true;
    const int lane = threadIdx.x & 31;
    for (;;) {
        if (active && p < 0) {
            p = (int64_t)atomicAdd(&slots[0], 1ull);
            if (p >= P.n_paths) {
                active = false;
                p = -1;
            } else {
                r.init(P.key0, P.key1, P.path_base + (uint64_t)p);
                path_init<DIM>(P, r, s);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    S.x1[k * scap + p] = s.x[k];
                    S.w1[k * scap + p] = s.w[k];
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        bool multi = false;
        double xi = 0.0, wpx = 0.0;
        if (active) {
            ++s.pL;
            xi = P.want_phase ? r.rand() : 0.0;
            wpx = s.weight / s.px;
            if (s.pL == 1) {
                S.wpx[p] = wpx;
                S.xi[p] = xi;
            } else {
                multi = true;
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, multi);
        if (mask) {
            const int leader = __ffs(mask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&slots[1], (unsigned long long)__popc(mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (multi) {
                const int64_t e = (int64_t)base + __popc(mask & ((1u << lane) - 1u));
                if (e < mcap) {
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        M.x[k * mcap + e] = s.x[k];
                        M.ow[k * mcap + e] = s.ow[k];
                    }
                    M.wpx[e] = wpx;
                    M.xi[e] = xi;
                    M.path[e] = (int32_t)p;
                    M.plen[e] = s.pL;
                }
            }
        }
        if (active) {
            bool alive = path_advance<DIM>(P, r, s);
            if (alive && P.max_events > 0 && s.pL >= P.max_events) {
                atomicExch(err, 1);
                alive = false;
            }
            if (!alive) {
                S.nev[p] = s.pL;
                p = -1;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Packs of requests (the request server): the paths of n requests are one
// index range, request r owning [prefix[r], prefix[r + 1]); path g of request
// r is that request's path path_base + g - prefix[r] under its own Philox key
// and medium.  Two passes as for one request, so each request's records are
// contiguous (its multiple-scattering records follow moff[prefix[r]]).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pack_request(const int64_t *__restrict__ prefix, int n, int64_t g)
{
    int lo = 0, hi = n - 1;  // the last r with prefix[r] <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int DIM>
__global__ void __launch_bounds__(128) walk_count_packed_kernel(const WalkParams *__restrict__ Ps,
                                                                const int64_t *__restrict__ prefix, int n_req,
                                                                int64_t n_paths, int32_t *__restrict__ counts,
                                                                unsigned long long *__restrict__ next_path,
                                                                int *__restrict__ err)
{
    PathRng r;
    WalkState s;
    int64_t p = -1;
    const WalkParams *P = Ps;
    int n = 0;
    for (;;) {
        if (p < 0) {
            p = (int64_t)atomicAdd(next_path, 1ull);
            if (p >= n_paths) break;
            const int q = pack_request(prefix, n_req, p);
            P = Ps + q;
            r.init(P->key0, P->key1, P->path_base + (uint64_t)(p - prefix[q]));
            path_init<DIM>(*P, r, s);
            n = 0;
        }
        ++n;
        if (P->want_phase) (void)r.rand();
        bool alive = path_advance<DIM>(*P, r, s);
        if (alive && P->max_events > 0 && n >= P->max_events) {
            atomicExch(err, 1);
            alive = false;
        }
        if (!alive) {
            counts[p] = n;
            p = -1;
        }
    }
}

template <int DIM>
__global__ void __launch_bounds__(128) walk_record_packed_kernel(const WalkParams *__restrict__ Ps,
                                                                 const int64_t *__restrict__ prefix, int n_req,
                                                                 int64_t n_paths, const int64_t *__restrict__ moff,
                                                                 SingleRec S, int64_t scap, MultiRec M, int64_t mcap,
                                                                 unsigned long long *__restrict__ next_path)
{
    PathRng r;
    WalkState s;
    int64_t p = -1, mo = 0;
    const WalkParams *P = Ps;
    for (;;) {
        if (p < 0) {
            p = (int64_t)atomicAdd(next_path, 1ull);
            if (p >= n_paths) break;
            const int q = pack_request(prefix, n_req, p);
            P = Ps + q;
            r.init(P->key0, P->key1, P->path_base + (uint64_t)(p - prefix[q]));
            path_init<DIM>(*P, r, s);
            mo = moff[p];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                S.x1[k * scap + p] = s.x[k];
                S.w1[k * scap + p] = s.w[k];
            }
        }
        ++s.pL;
        const double xi = P->want_phase ? r.rand() : 0.0;
        const double wpx = s.weight / s.px;
        if (s.pL == 1) {
            S.wpx[p] = wpx;
            S.xi[p] = xi;
        } else {
            const int64_t e = mo + (s.pL - 2);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                M.x[k * mcap + e] = s.x[k];
                M.ow[k * mcap + e] = s.ow[k];
            }
            M.wpx[e] = wpx;
            M.xi[e] = xi;
            M.path[e] = (int32_t)p;
            M.plen[e] = s.pL;
        }
        bool alive = path_advance<DIM>(*P, r, s);
        if (alive && P->max_events > 0 && s.pL >= P->max_events) alive = false;
        if (!alive) {
            S.nev[p] = s.pL;
            p = -1;
        }
    }
}

}  // namespace scmc
