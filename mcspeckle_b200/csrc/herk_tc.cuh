// herk_tc.cuh - covariance contraction on tcgen05 tensor cores (sm_100a).
//
// Every event contributes one Hermitian rank-1 update C += t t^H
// (MCcov.m:232-263), t in C^N with N = nv*nl.  A chunk of E events is the
// complex rank-E update C += T^T conj(T), done as one real GEMM:
//
//   K  = 2E (column 2e holds Re, 2e+1 holds Im of event e)
//   A  = [2N x K]  row 2i   = ( Re t_i,  Im t_i)  per event
//                  row 2i+1 = ( Im t_i, -Re t_i)
//   B  = [N  x K]  row j    = ( Re t_j,  Im t_j)  (= the even rows of A)
//   D  = A B^T     D[2i][j] = Re C[i][j],  D[2i+1][j] = Im C[i][j]
//
// Precision: A is split into FP16 hi + lo parts (A = hi + lo to ~2^-22).
// This single-CTA kernel (and the field and FourierQuad forms) computes
// D = (A_hi + A_lo) B_hi^T, compensating A's rounding only; the CTA-pair
// covariance kernel (herk_tc2_kernel) adds a second sweep A_hi B_lo^T, so
// only A_lo B_lo^T is left out.  Products accumulate in FP32 in TMEM; after
// the chunk the tile is added into an FP64 accumulator, which carries the sum
// across chunks.
//
// Kernel shape: one CTA per 128 x 256 output tile of the upper triangle
// (complex rows 64*tm .. 64*tm+63 against complex columns 256*tn ..).
// Warp 0 issues TMA loads (128B swizzle, no multicast), warp 1 issues
// tcgen05.mma (M=128, N=256, K=16, kind::f16) from one lane, all four warps
// drain TMEM in the epilogue.  3-stage smem ring of 64 KB.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <stdexcept>
#include <vector>

#include "accum.cuh"

namespace scmc {

constexpr int TC_BM = 128;
constexpr int TC_BN = 256;
constexpr int TC_BK = 64;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 2;
constexpr int TC_B_BYTES = TC_BN * TC_BK * 2;
constexpr int TC_TMEM_COLS = 256;
// SPLIT: A_hi + A_lo + B per stage (64 KB, 3 stages); otherwise A + B (48 KB, 4 stages)
template <bool SPLIT> struct TcCfg {
    static constexpr int STAGE_BYTES = (SPLIT ? 2 : 1) * TC_A_BYTES + TC_B_BYTES;
    static constexpr int STAGES = SPLIT ? 3 : 4;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
    static constexpr int B_OFF = (SPLIT ? 2 : 1) * TC_A_BYTES;
};
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;  // 2 s bound on every wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after `limit` ns (TC_WAIT_NS by default) without the
// phase completing.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned long long limit = TC_WAIT_NS)
{
    if (mbar_try_wait(bar, parity)) return true;
    unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_ns() - t0 > limit) return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, rows of 128 B,
// 8-row groups 1024 B apart (SBO), LBO unused (1), sm_100 version bits.
__device__ __forceinline__ uint64_t umma_desc_sw128(const void *smem_tile)
{
    uint64_t a = (uint64_t)((smem_u32(smem_tile) & 0x3FFFF) >> 4);
    return a | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// kind::f16 instruction descriptor: D F32, A/B F16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int M, int N)
{
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// The FourierQuad plane data of fq_planes_tc_kernel.  zexp0 and rr are
// stored r1-fastest ([r2][r1]): a warp's lanes hold 16 consecutive rows r1 at
// one column, so its loads are contiguous.  U is stored [r1][r2].
struct PlaneEpi {
    const double2 *zexp0;  // [r2][r1]: the plane factor is exp(zexp0 * tz)
    const float2 *rr;      // [r2][r1]: exp(zexp0 * 2 z_bin), the factor between planes P and P - 2
    const double *gz;      // plane boundaries
    const int *planes;     // plane of each plane slot
    double *U;             // [r1][r2] complex interleaved FP64, this light (the sum across planes and batches)
    int nv0;
    int n_uniform;         // planes 0 .. n_uniform-1 have centres bmin_z + (P + 1/2) z_bin
    const unsigned *max_bits;  // the group's operand scale (fq_scale_exponent); the flush undoes it
};

// The exponent of the power-of-two operand scale of a FourierQuad plane
// group: max |s_e| maps into [2^13, 2^14), well inside FP16's normal range.
__device__ __forceinline__ int fq_scale_exponent(const unsigned *max_bits)
{
    const float m = __uint_as_float(*max_bits);
    return m > 0.f ? 13 - ilogbf(m) : 0;
}

// Bounded waits can be made to run out on purpose (scmc_test_wait_fault):
// the producer then issues no copy and the consumers wait only this long, so
// the abort path runs with nothing in flight.
constexpr unsigned long long TC_TEST_WAIT_NS = 1000000ull;  // 1 ms
inline std::atomic<int> &tc_test_fault()
{
    static std::atomic<int> on{0};
    return on;
}

// One 128 x 256 tile of D += (A_hi [+ A_lo]) B^T over num_kb K-blocks of 64.
template <bool SPLIT>
__global__ void __launch_bounds__(128, 1)
herk_tc_kernel(const __grid_constant__ CUtensorMap tm_ahi, const __grid_constant__ CUtensorMap tm_alo,
               const __grid_constant__ CUtensorMap tm_b, const int2 *__restrict__ tiles, int num_kb, int kb_per_split,
               int Mr, int N, double *__restrict__ D, int *__restrict__ err, int test_fault)
{
    // split-K: blockIdx.y takes K-blocks [kb0, kb0 + nkb) and owns the slice
    // D + blockIdx.y * Mr * N; the host makes every slice non-empty.
    const int kb0 = (int)blockIdx.y * kb_per_split;
    const int nkb = min(num_kb, kb0 + kb_per_split) - kb0;
    if (nkb <= 0) return;
    D += (int64_t)blockIdx.y * Mr * N;
    extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + TcCfg<SPLIT>::STAGES * TcCfg<SPLIT>::STAGE_BYTES);
    uint64_t *empty = full + TcCfg<SPLIT>::STAGES;
    uint64_t *done = empty + TcCfg<SPLIT>::STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
    int *issued = abort_flag + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 tile = tiles[blockIdx.x];
    const int row0 = tile.x * TC_BM;
    const int col0 = tile.y * TC_BN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TcCfg<SPLIT>::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        *issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const unsigned long long wait_ns = test_fault ? TC_TEST_WAIT_NS : TC_WAIT_NS;
    if (warp == 0 && lane == 0) {
        // TMA producer (none in a fault test)
        for (int kb = 0; kb < (test_fault ? 0 : nkb); ++kb) {
            const int s = kb % TcCfg<SPLIT>::STAGES;
            if (kb >= TcCfg<SPLIT>::STAGES && !mbar_wait(&empty[s], ((kb / TcCfg<SPLIT>::STAGES) - 1) & 1)) {
                atomicExch(abort_flag, 1);
                break;
            }
            if (*(volatile int *)abort_flag) break;
            uint8_t *st = base + s * TcCfg<SPLIT>::STAGE_BYTES;
            mbar_expect_tx(&full[s], TcCfg<SPLIT>::STAGE_BYTES);
            const int kx = (kb0 + kb) * TC_BK;
            tma_load_2d(st, &tm_ahi, kx, row0, &full[s]);
            if (SPLIT) tma_load_2d(st + TC_A_BYTES, &tm_alo, kx, row0, &full[s]);
            tma_load_2d(st + TcCfg<SPLIT>::B_OFF, &tm_b, kx, col0, &full[s]);
            *(volatile int *)issued = kb + 1;
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        constexpr uint32_t idesc = umma_idesc_f16(TC_BM, TC_BN);
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % TcCfg<SPLIT>::STAGES;
            if (!mbar_wait(&full[s], (kb / TcCfg<SPLIT>::STAGES) & 1, wait_ns)) {
                atomicExch(abort_flag, 1);
                break;
            }
            tc_fence_after();
            uint8_t *st = base + s * TcCfg<SPLIT>::STAGE_BYTES;
            const uint64_t dh = umma_desc_sw128(st);
            const uint64_t dl = umma_desc_sw128(st + TC_A_BYTES);
            const uint64_t db = umma_desc_sw128(st + TcCfg<SPLIT>::B_OFF);
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; ++kk) {
                const uint64_t adv = (uint64_t)(kk * 32) >> 4;  // 16 fp16 = 32 B along K
                umma_f16(tmem, dh + adv, db + adv, idesc, (kb | kk) != 0);
                if (SPLIT) umma_f16(tmem, dl + adv, db + adv, idesc, 1u);
            }
            umma_commit(&empty[s]);
        }
        umma_commit(done);  // fires once every issued MMA has completed
    }
    __syncwarp();

    const bool ok = mbar_wait(done, 0);
    tc_fence_after();
    __syncthreads();
    if (!ok || *(volatile int *)abort_flag) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            // wait (bounded) for TMA copies this CTA still has in flight
            const int n_issued = *(volatile int *)issued;
            for (int kb = (n_issued > TcCfg<SPLIT>::STAGES ? n_issued - TcCfg<SPLIT>::STAGES : 0); kb < n_issued; ++kb)
                (void)mbar_wait(&full[kb % TcCfg<SPLIT>::STAGES], (kb / TcCfg<SPLIT>::STAGES) & 1);
        }
    } else {
        // Epilogue: TMEM -> registers -> smem transpose -> coalesced FP64 RMW.
        float *ep = reinterpret_cast<float *>(base) + warp * 32 * 33;
        const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < TC_BN; c0 += 32) {
            uint32_t r[32];
            tmem_ld32(tbase + c0, r);
#pragma unroll
            for (int j = 0; j < 32; ++j) ep[lane * 33 + j] = __uint_as_float(r[j]);
            __syncwarp();
            const int n = col0 + c0 + lane;
            // all 32 loads of the chunk in flight before the adds and stores
            double *p = D + (int64_t)(row0 + warp * 32) * N + n;
            const int rows = min(32, Mr - (row0 + warp * 32));
            double v[32];
#pragma unroll
            for (int rr = 0; rr < 32; ++rr) v[rr] = (rr < rows && n < N) ? p[(int64_t)rr * N] : 0.0;
#pragma unroll
            for (int rr = 0; rr < 32; ++rr)
                if (rr < rows && n < N) p[(int64_t)rr * N] = v[rr] + (double)ep[rr * 33 + lane];
            __syncwarp();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
        "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
        "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}

// 16 columns of this warp's 32 TMEM lanes, without waiting (tmem_wait_ld).
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

// ---------------------------------------------------------------------------
// The FourierQuad per-plane sums with the plane loop inside the CTA.
//
// A CTA owns one 128 x 256 tile (64 complex rows r1 as Re / Im real rows,
// 256 columns r2) and a contiguous range of plane slots of a group
// (pranges[y]: first slot, slot count; kranges[slot]: the plane's K blocks,
// contiguous across slots).  It needs  sum_P exp(zexp0 tz_P) F_P  over its
// planes, F_P the plane's product A_P B_P^T.  The planes are walked from the
// deepest down, alternately into two accumulators of 256 TMEM columns
// (chain 0: slots 0, 2, 4, ... of the walk; chain 1: slots 1, 3, ...), each
// summed Horner-wise: after plane P's MMAs, when the chain's next plane is
// P - 2 (uniform planes, planes are 2 z_bin apart), the epilogue multiplies
// the accumulator in place by rr = exp(zexp0 2 z_bin) in FP32 and the next
// plane's MMAs add on top, so the chain holds sum_k rr^(m-k) F_(P_k).  When
// the chain's next plane is not P - 2 (an empty plane, the last,
// non-uniform plane, the end of the range) or the segment reached
// kFqSegMax planes, the epilogue adds exp(zexp0 tz_P) times the
// accumulator into U (factor with the phase product and reduction in FP64,
// sincos and exp in FP32; the sum across planes and batches is FP64) and the
// chain's next MMA starts it afresh.  While
// the epilogue works on one chain the MMAs of the other run.
// Warp 0 issues the TMA loads of every K block in walk order through the
// ring, warp 1 the MMAs, warps 4-7 (one TMEM lane quarter each) the
// epilogue.  Every wait is bounded.
// ---------------------------------------------------------------------------
constexpr int kFqSegMax = 64;  // chain steps between FP64-seeded flushes

// Whether a chain continues from plane p_hi (segment of seg_len planes so
// far) to the chain's next plane p_lo.
__device__ __forceinline__ bool fq_chain_continues(int p_hi, int p_lo, int seg_len, int n_uniform)
{
    return p_hi - p_lo == 2 && p_hi < n_uniform && seg_len < kFqSegMax;
}

template <bool SPLIT>
__global__ void __launch_bounds__(256, 1)
fq_planes_tc_kernel(const __grid_constant__ CUtensorMap tm_ahi, const __grid_constant__ CUtensorMap tm_alo,
                    const __grid_constant__ CUtensorMap tm_b, const int2 *__restrict__ tiles,
                    const int2 *__restrict__ kranges, const int2 *__restrict__ pranges, int Mr, int N,
                    const __grid_constant__ PlaneEpi pe, int *__restrict__ err, int test_fault)
{
    using Cfg = TcCfg<SPLIT>;
    constexpr int S = Cfg::STAGES;
    extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + S * Cfg::STAGE_BYTES);
    uint64_t *empty = full + S;
    uint64_t *acc_full = empty + S;   // [2], one per chain
    uint64_t *acc_empty = acc_full + 2;
    uint64_t *done = acc_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
    int *issued = abort_flag + 1;
    int *ep_fail = issued + 1;  // written only by the epilogue warps

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 tile = tiles[blockIdx.x];
    const int row0 = tile.x * TC_BM;
    const int col0 = tile.y * TC_BN;
    const int2 pr = pranges[blockIdx.y];  // the host makes every range non-empty
    const int last = pr.x + pr.y - 1;     // the walk goes from slot `last` down to pr.x
    const unsigned long long wait_ns = test_fault ? TC_TEST_WAIT_NS : TC_WAIT_NS;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int c = 0; c < 2; ++c) {
            mbar_init(&acc_full[c], 1);
            mbar_init(&acc_empty[c], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        *issued = 0;
        *ep_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // TMA producer: the K blocks of every plane, deepest plane first
        int kb = 0;
        bool stop = test_fault != 0;  // fault test: no copy is ever issued
        for (int i = 0; i < pr.y && !stop; ++i) {
            const int2 kr = kranges[last - i];
            for (int j = 0; j < kr.y; ++j, ++kb) {
                const int s = kb % S;
                if (kb >= S && !mbar_wait(&empty[s], ((kb / S) - 1) & 1)) {
                    atomicExch(abort_flag, 1);
                    stop = true;
                    break;
                }
                if (*(volatile int *)abort_flag) {
                    stop = true;
                    break;
                }
                uint8_t *st = base + s * Cfg::STAGE_BYTES;
                mbar_expect_tx(&full[s], Cfg::STAGE_BYTES);
                const int kx = (kr.x + j) * TC_BK;
                tma_load_2d(st, &tm_ahi, kx, row0, &full[s]);
                if (SPLIT) tma_load_2d(st + TC_A_BYTES, &tm_alo, kx, row0, &full[s]);
                tma_load_2d(st + Cfg::B_OFF, &tm_b, kx, col0, &full[s]);
                *(volatile int *)issued = kb + 1;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: plane slot i of the walk into chain i & 1
        constexpr uint32_t idesc = umma_idesc_f16(TC_BM, TC_BN);
        int kb = 0;
        bool ok = true;
        int prev[2] = {0, 0}, seg[2] = {0, 0};
        for (int i = 0; i < pr.y && ok; ++i) {
            const int c = i & 1;
            const int slot = last - i;
            const int P = pe.planes[slot];
            const bool start = i < 2 || !fq_chain_continues(prev[c], P, seg[c], pe.n_uniform);
            seg[c] = start ? 1 : seg[c] + 1;
            prev[c] = P;
            if (i >= 2) {  // the epilogue has released this chain's accumulator
                if (!mbar_wait(&acc_empty[c], ((i >> 1) - 1) & 1, wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
            }
            const uint32_t tacc = tmem + (uint32_t)(c * TC_TMEM_COLS);
            const int nk = kranges[slot].y;
            for (int j = 0; j < nk; ++j, ++kb) {
                const int s = kb % S;
                if (!mbar_wait(&full[s], (kb / S) & 1, wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                uint8_t *st = base + s * Cfg::STAGE_BYTES;
                const uint64_t dh = umma_desc_sw128(st);
                const uint64_t dl = umma_desc_sw128(st + TC_A_BYTES);
                const uint64_t db = umma_desc_sw128(st + Cfg::B_OFF);
#pragma unroll
                for (int kk = 0; kk < TC_BK / 16; ++kk) {
                    const uint64_t adv = (uint64_t)(kk * 32) >> 4;
                    umma_f16(tacc, dh + adv, db + adv, idesc, (start && j == 0 && kk == 0) ? 0u : 1u);
                    if (SPLIT) umma_f16(tacc, dl + adv, db + adv, idesc, 1u);
                }
                umma_commit(&empty[s]);
            }
            if (ok) umma_commit(&acc_full[c]);
        }
        if (!ok) atomicExch(abort_flag, 1);
        umma_commit(done);  // fires once every issued MMA has completed
    } else if (warp >= 4) {
        // epilogue: TMEM lane = real row row0 + 32 q + lane (Re rows even, Im
        // rows odd).  The lane pair (2i, 2i + 1) shares complex row r1: the
        // even lane produces columns t, the odd lane columns 16 + t of each
        // 32-column chunk, and they swap halves so each stores its own row.
        const int q = warp - 4;
        const int R = row0 + q * 32 + lane;
        const int r1 = R >> 1;
        const bool odd = lane & 1, row_ok = R < Mr;
        const int jb = odd ? 16 : 0;
        int prev[2] = {0, 0}, seg[2] = {0, 0};
        for (int i = 0; i < pr.y; ++i) {
            const int c = i & 1;
            const int slot = last - i;
            const int P = pe.planes[slot];
            const bool start = i < 2 || !fq_chain_continues(prev[c], P, seg[c], pe.n_uniform);
            seg[c] = start ? 1 : seg[c] + 1;
            prev[c] = P;
            const bool cont = i + 2 < pr.y && fq_chain_continues(P, pe.planes[slot - 2], seg[c], pe.n_uniform);
            // the four warps agree on a timeout before leaving the loop, so
            // that every named barrier below is reached by all of them
            if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[c], (i >> 1) & 1, wait_ns)) && lane == 0)
                atomicExch(ep_fail, 1);
            asm volatile("bar.sync 1, 128;" ::: "memory");
            if (*(volatile int *)ep_fail) {
                atomicExch(abort_flag, 1);
                break;
            }
            tc_fence_after();
            const uint32_t tacc = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(c * TC_TMEM_COLS);
            const double tz = (pe.gz[P] + pe.gz[P + 1]) / 2;
            const float unscale = ldexpf(1.f, -fq_scale_exponent(pe.max_bits));
            for (int c0 = 0; c0 < TC_BN; c0 += 32) {
                uint32_t a[32];
                tmem_ld32(tacc + c0, a);
                // this lane's column n = col0 + c0 + jb + t: its own value and
                // the partner's (Re, Im) of the same complex element
                float fx[16], fy[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    const int n = col0 + c0 + jb + t;
                    const bool ok = row_ok && n < N;
                    if (cont) {
                        const float2 f = ok ? pe.rr[(int64_t)n * pe.nv0 + r1] : make_float2(0.f, 0.f);
                        fx[t] = f.x;
                        fy[t] = f.y;
                    } else {
                        const double2 z = ok ? pe.zexp0[(int64_t)n * pe.nv0 + r1] : make_double2(0.0, 0.0);
                        float sn, cs;
                        __sincosf((float)reduce_2pi(z.y * tz), &sn, &cs);
                        const float mag = ok ? expf((float)(z.x * tz)) * unscale : 0.f;
                        fx[t] = mag * cs;
                        fy[t] = mag * sn;
                    }
                }
                uint32_t out[32];
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    // even lane: element (r1, t) = (a[t], partner's a[t]);
                    // odd lane: element (r1, 16 + t) = (partner's a[16 + t], a[16 + t])
                    const float mine = __uint_as_float(odd ? a[16 + t] : a[t]);
                    const float give = __uint_as_float(odd ? a[t] : a[16 + t]);
                    const float got = __shfl_xor_sync(0xffffffffu, give, 1);
                    const float re = odd ? got : mine, im = odd ? mine : got;
                    const float vr = fx[t] * re - fy[t] * im, vi = fx[t] * im + fy[t] * re;
                    if (cont) {
                        // the chain continues: store back, even lane keeps the Re row, odd the Im row
                        const float send = odd ? vr : vi;
                        const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
                        out[t] = __float_as_uint(odd ? recv : vr);       // column t of this lane's row
                        out[16 + t] = __float_as_uint(odd ? vi : recv);  // column 16 + t
                    } else {
                        const int n = col0 + c0 + jb + t;
                        if (row_ok && n < N) {
                            double *u = pe.U + 2 * ((int64_t)r1 * pe.nv0 + n);
                            atomicAdd(u, (double)vr);
                            atomicAdd(u + 1, (double)vi);
                        }
                    }
                }
                if (cont) tmem_st32(tacc + c0, out);
            }
            if (cont) asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            asm volatile("bar.sync 1, 128;" ::: "memory");
            if (q == 0 && lane == 0) mbar_arrive(&acc_empty[c]);
        }
    }
    __syncwarp();

    const bool ok = mbar_wait(done, 0);
    tc_fence_after();
    __syncthreads();
    const bool failed = !ok || *(volatile int *)abort_flag;
    if (failed && threadIdx.x == 0) {
        atomicExch(err, 1);
        // wait (bounded) for TMA copies this CTA still has in flight
        const int n_issued = *(volatile int *)issued;
        for (int kb = (n_issued > S ? n_issued - S : 0); kb < n_issued; ++kb)
            (void)mbar_wait(&full[kb % S], (kb / S) & 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_TMEM_COLS)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// The covariance product on a CTA pair (cluster of 2, tcgen05 cta_group::2),
// from split-complex ("planar") operands.
//
// The rows are stored as two planes, Re T and Im T (N rows x K events each,
// FP16, plus the low parts for hi+lo), half the bytes of the real-expanded
// layout.  For complex rows i and columns j
//     Re C_ij = Re t_i . Re t_j + Im t_i . Im t_j
//     Im C_ij = Im t_i . Re t_j - Re t_i . Im t_j
// so a pair that owns 256 complex rows x 256 complex columns keeps two
// accumulators in TMEM (columns 0-255: Re C, 256-511: Im C) and issues four
// M=256 N=256 K=16 MMAs per 16 events from four tiles of shared memory; the
// minus sign is the MMA's negate-A bit.  CTA r loads the 128 A rows
// crow0 + 128 r of both planes and B rows col0 + 128 r of both planes: 64 KB
// per stage (96 KB hi+lo) for 4 x 128 x 256 x 64 multiply-adds per SM, twice
// the work per loaded byte of a real-expanded tile.  The loads are plain (no
// multicast); their completion is counted on the leader's barrier.  The
// leader's MMA commits arrive on both CTAs' barriers (commit multicast).
// Every wait is bounded as in herk_tc_kernel.
// ---------------------------------------------------------------------------
// Two 64 KB stages (FP16) leave room on the SM for a row-generation CTA of
// the next chunk (about 72 KB at 64 x 64); three (FP16 only: 193 KB) are the
// autotuner's alternative.
constexpr int TC2_TMEM_COLS = 512;  // Re C and Im C, 256 columns each
template <bool SPLIT, int NSTAGES = 2> struct Tc2Cfg {
    static constexpr int TILE = 128 * TC_BK * 2;  // 128 rows x 64 events of one plane
    static constexpr int NA = SPLIT ? 4 : 2;      // A tiles: Re, Im (hi), Re, Im (lo)
    static constexpr int STAGE_BYTES = (NA + 2) * TILE;
    static constexpr int STAGES = NSTAGES;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
    static constexpr int B_OFF = NA * TILE;  // then Re B, Im B
};

__device__ __forceinline__ uint32_t cluster_ctarank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Address of the same shared-memory offset in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ uint32_t ld_shared_cluster_u32(uint32_t addr)
{
    uint32_t v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// TMA load into this CTA's shared memory whose completion is counted on a
// barrier of either CTA of the pair (cluster address).  No multicast.
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map, int x, int y, uint32_t bar_cluster)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster)
        : "memory");
}

// The same for a 3-D map (K-block-major operands: x = entry in the block, y = row, z = block).
__device__ __forceinline__ void tma_load_3d_pair(void *dst, const CUtensorMap *map, int x, int y, int z,
                                                 uint32_t bar_cluster)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar_cluster)
        : "memory");
}

__device__ __forceinline__ void umma_f16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// Arrive on the barrier at this offset in both CTAs once the leader's issued
// MMAs have completed.
__device__ __forceinline__ void umma_commit_pair(uint64_t *bar)
{
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(mask)
        : "memory");
}

template <bool SPLIT, int NSTAGES>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(128, 1)
herk_tc2_kernel(const __grid_constant__ CUtensorMap tm_re, const __grid_constant__ CUtensorMap tm_im,
                const __grid_constant__ CUtensorMap tm_re_lo, const __grid_constant__ CUtensorMap tm_im_lo,
                const int2 *__restrict__ tiles, int num_kb, int kb_per_split, int N, double *__restrict__ D,
                int *__restrict__ err, int test_fault)
{
    using Cfg = Tc2Cfg<SPLIT, NSTAGES>;
    extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + Cfg::STAGES * Cfg::STAGE_BYTES);
    uint64_t *empty = full + Cfg::STAGES;
    uint64_t *done = empty + Cfg::STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
    int *issued = abort_flag + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    // The split-K range is the same for both CTAs of a pair (same blockIdx.y),
    // so either both return here or neither does.
    const int kb0 = (int)blockIdx.y * kb_per_split;
    const int nkb = min(num_kb, kb0 + kb_per_split) - kb0;
    if (nkb <= 0) return;
    // hi+lo: a first sweep of (A hi + A lo) B hi over the K blocks and a
    // second of A hi B lo, so both operands' FP16 rounding is compensated
    // (only A lo B lo, about 2^-22 relative, is left out)
    const int nk_all = SPLIT ? 2 * nkb : nkb;
    const int Mr = 2 * N;
    D += (int64_t)blockIdx.y * Mr * N;
    const int2 tile = tiles[blockIdx.x >> 1];
    const int crow0 = tile.x * 256 + (int)rank * 128;  // this CTA's complex rows
    const int col0 = tile.y * 256;                     // the pair's complex columns
    const int brow0 = col0 + (int)rank * 128;          // this CTA's B rows

    if (threadIdx.x == 0) {
        for (int s = 0; s < Cfg::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        *issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC2_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    cluster_sync_all();  // both CTAs' barriers exist before any load or commit reaches them
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const unsigned long long wait_ns = test_fault ? TC_TEST_WAIT_NS : TC_WAIT_NS;
    if (warp == 0 && lane == 0) {
        // TMA producer (both CTAs; none in a fault test); completion counted on the leader's full[s]
        const uint32_t full0 = mapa_shared(smem_u32(&full[0]), 0);
        for (int kb = 0; kb < (test_fault ? 0 : nk_all); ++kb) {
            const int s = kb % Cfg::STAGES;
            if (kb >= Cfg::STAGES && !mbar_wait(&empty[s], ((kb / Cfg::STAGES) - 1) & 1)) {
                atomicExch(abort_flag, 1);
                break;
            }
            if (*(volatile int *)abort_flag) break;
            uint8_t *st = base + s * Cfg::STAGE_BYTES;
            const bool sweep2 = SPLIT && kb >= nkb;  // A hi x B lo
            if (rank == 0) mbar_expect_tx(&full[s], sweep2 ? 2 * 4 * Cfg::TILE : 2 * Cfg::STAGE_BYTES);
            const uint32_t fb = full0 + (uint32_t)(s * sizeof(uint64_t));
            const int kx = (kb0 + (sweep2 ? kb - nkb : kb)) * TC_BK;
            tma_load_2d_pair(st, &tm_re, kx, crow0, fb);
            tma_load_2d_pair(st + Cfg::TILE, &tm_im, kx, crow0, fb);
            if (sweep2) {
                tma_load_2d_pair(st + Cfg::B_OFF, &tm_re_lo, kx, brow0, fb);
                tma_load_2d_pair(st + Cfg::B_OFF + Cfg::TILE, &tm_im_lo, kx, brow0, fb);
            } else {
                if (SPLIT) {
                    tma_load_2d_pair(st + 2 * Cfg::TILE, &tm_re_lo, kx, crow0, fb);
                    tma_load_2d_pair(st + 3 * Cfg::TILE, &tm_im_lo, kx, crow0, fb);
                }
                tma_load_2d_pair(st + Cfg::B_OFF, &tm_re, kx, brow0, fb);
                tma_load_2d_pair(st + Cfg::B_OFF + Cfg::TILE, &tm_im, kx, brow0, fb);
            }
            *(volatile int *)issued = kb + 1;
        }
    } else if (warp == 1 && lane == 0 && rank == 0) {
        // MMA issuer (leader only)
        constexpr uint32_t idesc = umma_idesc_f16(256, 256);
        constexpr uint32_t idesc_neg = idesc | (1u << 13);  // negate A
        const uint32_t t_re = tmem, t_im = tmem + 256;
        for (int kb = 0; kb < nk_all; ++kb) {
            const int s = kb % Cfg::STAGES;
            if (!mbar_wait(&full[s], (kb / Cfg::STAGES) & 1, wait_ns)) {
                atomicExch(abort_flag, 1);
                break;
            }
            tc_fence_after();
            const bool sweep2 = SPLIT && kb >= nkb;  // the stage holds A hi and B lo
            uint8_t *st = base + s * Cfg::STAGE_BYTES;
            const uint64_t ar = umma_desc_sw128(st), ai = umma_desc_sw128(st + Cfg::TILE);
            const uint64_t br = umma_desc_sw128(st + Cfg::B_OFF), bi = umma_desc_sw128(st + Cfg::B_OFF + Cfg::TILE);
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; ++kk) {
                const uint64_t adv = (uint64_t)(kk * 32) >> 4;
                const uint32_t first = (kb | kk) != 0;
                umma_f16_pair(t_re, ar + adv, br + adv, idesc, first);
                umma_f16_pair(t_im, ai + adv, br + adv, idesc, first);
                umma_f16_pair(t_re, ai + adv, bi + adv, idesc, 1u);
                umma_f16_pair(t_im, ar + adv, bi + adv, idesc_neg, 1u);
                if (SPLIT && !sweep2) {
                    const uint64_t lr = umma_desc_sw128(st + 2 * Cfg::TILE) + adv;
                    const uint64_t li = umma_desc_sw128(st + 3 * Cfg::TILE) + adv;
                    umma_f16_pair(t_re, lr, br + adv, idesc, 1u);
                    umma_f16_pair(t_im, li, br + adv, idesc, 1u);
                    umma_f16_pair(t_re, li, bi + adv, idesc, 1u);
                    umma_f16_pair(t_im, lr, bi + adv, idesc_neg, 1u);
                }
            }
            umma_commit_pair(&empty[s]);
        }
        umma_commit_pair(done);  // both CTAs' done[] once every issued MMA has completed
    }
    __syncwarp();

    const bool ok = mbar_wait(done, 0);
    tc_fence_after();
    __syncthreads();
    const bool failed = !ok || *(volatile int *)abort_flag;
    if (!failed) {
        // Epilogue: TMEM lane L = complex row crow0 + L; columns 0-255 -> D row
        // 2 (crow0 + L) (Re), 256-511 -> row 2 (crow0 + L) + 1 (Im); smem
        // transpose -> coalesced FP64 read-modify-write.
        float *ep = reinterpret_cast<float *>(base) + warp * 32 * 33;
        const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < 512; c0 += 32) {
            uint32_t r[32];
            tmem_ld32(tbase + c0, r);
#pragma unroll
            for (int j = 0; j < 32; ++j) ep[lane * 33 + j] = __uint_as_float(r[j]);
            __syncwarp();
            const int part = c0 >> 8;
            const int n = col0 + (c0 & 255) + lane;
            // all 32 loads of the chunk in flight before the adds and stores
            double *p = D + (int64_t)(2 * (crow0 + warp * 32) + part) * N + n;
            const int rows = min(32, N - (crow0 + warp * 32));
            double v[32];
#pragma unroll
            for (int rr = 0; rr < 32; ++rr) v[rr] = (rr < rows && n < N) ? p[(int64_t)2 * rr * N] : 0.0;
#pragma unroll
            for (int rr = 0; rr < 32; ++rr)
                if (rr < rows && n < N) p[(int64_t)2 * rr * N] = v[rr] + (double)ep[rr * 33 + lane];
            __syncwarp();
        }
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();
    if (threadIdx.x == 0) {
        // After a failure anywhere in the pair, the leader waits (bounded) for
        // the pair's copies still in flight, which are counted on its
        // barriers, before the pair exits.
        const int peer_abort = (int)ld_shared_cluster_u32(mapa_shared(smem_u32(abort_flag), rank ^ 1u));
        if (failed || peer_abort) {
            atomicExch(err, 1);
            if (rank == 0) {
                const int mine = *(volatile int *)issued;
                const int peer = (int)ld_shared_cluster_u32(mapa_shared(smem_u32(issued), 1));
                const int n_issued = max(mine, peer);
                for (int kb = (n_issued > Cfg::STAGES ? n_issued - Cfg::STAGES : 0); kb < n_issued; ++kb)
                    (void)mbar_wait(&full[kb % Cfg::STAGES], (kb / Cfg::STAGES) & 1);
            }
        }
    }
    cluster_sync_all();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC2_TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------------------
// The FourierQuad per-plane sums on a CTA pair from planar operands.
//
// For grids of at least 128 angles: A planes (Re, Im of s_e T[r1][p1_e]) and
// B planes (Re, Im of T[r2][p2_e]), FP16 (plus the low parts of A for hi+lo),
// K-block-major: per block of 64 entries (a plane's last block zero-padded) a
// contiguous nv0 x 64 slab, so a tile load is one contiguous 16 KB read.  A
// pair owns 256 rows r1 x 256 columns r2 (at nv0 = 256 the
// whole output, so every operand byte is read once per launch) with Re F and
// Im F in TMEM columns 0-255 and 256-511 of both CTAs (each CTA 128 rows):
//     Re F += Re A Re B - Im A Im B,   Im F += Im A Re B + Re A Im B
// (the minus is the MMA's negate-A bit), four M=256 N=256 K=16 MMAs per 16
// entries, issued by the leader.  The planes of the pair's range are walked
// from the deepest down in one Horner chain: after plane P's MMAs, when the
// next plane is P - 1 (uniform planes), the epilogue warps of both CTAs
// multiply their rows in place by r = exp(zexp0 z_bin) (FP32) and the next
// plane's MMAs add on top; otherwise (an empty plane, the last non-uniform
// plane, the range's end, or kFqSegMax steps) they add exp(zexp0 tz_P) times
// the chain into the FP64 output (factor: phase product and reduction in
// FP64, sincos and exp in FP32) and the next MMA starts afresh.  Each
// epilogue thread holds one row r1 with its Re and Im columns, so the complex
// products need no shuffles; 8 warps per CTA (two per TMEM lane quarter, half
// the columns each) keep the per-plane step short, since the MMAs wait for
// it.  The epilogues of both CTAs arrive on the leader's acc_empty (count 2)
// before the next plane's MMAs.  Warp 0 lane 0 issues the loads, warp 1 lane
// 0 the MMAs (leader), warps 2-3 only wait.  Loads are plain
// (no multicast), counted on the leader's full barrier; every wait is bounded.
// ---------------------------------------------------------------------------
struct PlaneEpi2 {
    const double2 *zexp0;  // [r2][r1]
    const float2 *r1step;  // [r2][r1]: exp(zexp0 * z_bin), planes P and P - 1
    const double *gz;      // plane boundaries
    const int *planes;     // plane of each plane slot
    double *U;             // [r2][r1] complex FP64, this light (a warp's rows are consecutive)
    int nv0;
    int n_uniform;
    const unsigned *max_bits;  // the group's operand scale (fq_scale_exponent)
};

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster_addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster_addr) : "memory");
}

__device__ __forceinline__ bool fq_chain1_continues(int p_hi, int p_lo, int seg_len, int n_uniform)
{
    return p_hi - p_lo == 1 && p_hi < n_uniform && seg_len < kFqSegMax;
}

template <bool SPLIT, int NSTAGES>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(384, 1)
fq_pair_planes_kernel(const __grid_constant__ CUtensorMap tm_are, const __grid_constant__ CUtensorMap tm_aim,
                      const __grid_constant__ CUtensorMap tm_are_lo, const __grid_constant__ CUtensorMap tm_aim_lo,
                      const __grid_constant__ CUtensorMap tm_bre, const __grid_constant__ CUtensorMap tm_bim,
                      const int2 *__restrict__ tiles, const int2 *__restrict__ kranges, const int2 *__restrict__ pranges,
                      const __grid_constant__ PlaneEpi2 pe, int *__restrict__ err, int test_fault)
{
    using Cfg = Tc2Cfg<SPLIT, NSTAGES>;
    constexpr int S = Cfg::STAGES;
    extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + S * Cfg::STAGE_BYTES);
    uint64_t *empty = full + S;
    uint64_t *acc_full = empty + S;
    uint64_t *acc_empty = acc_full + 1;  // the leader's counts both CTAs' epilogues
    uint64_t *done = acc_empty + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
    int *issued = abort_flag + 1;
    int *ep_fail = issued + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int2 tile = tiles[blockIdx.x >> 1];
    const int arow0 = tile.x * 256 + (int)rank * 128;  // this CTA's A rows (r1)
    const int col0 = tile.y * 256;                     // the pair's columns (r2)
    const int brow0 = col0 + (int)rank * 128;          // this CTA's B rows
    const int2 pr = pranges[blockIdx.y];               // the host makes every range non-empty
    const int last = pr.x + pr.y - 1;
    const unsigned long long wait_ns = test_fault ? TC_TEST_WAIT_NS : TC_WAIT_NS;
    const int N = pe.nv0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, 2);
        mbar_init(done, 1);
        *abort_flag = 0;
        *issued = 0;
        *ep_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC2_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    cluster_sync_all();  // both CTAs' barriers exist before any load, commit or remote arrive
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // TMA producer (both CTAs): K blocks of every plane, deepest first,
        // completion counted on the leader's full[s]
        const uint32_t full0 = mapa_shared(smem_u32(&full[0]), 0);
        int kb = 0;
        bool stop = test_fault != 0;  // fault test: no copy is ever issued
        for (int i = 0; i < pr.y && !stop; ++i) {
            const int2 kr = kranges[last - i];
            for (int j = 0; j < kr.y; ++j, ++kb) {
                const int s = kb % S;
                if (kb >= S && !mbar_wait(&empty[s], ((kb / S) - 1) & 1)) {
                    atomicExch(abort_flag, 1);
                    stop = true;
                    break;
                }
                if (*(volatile int *)abort_flag) {
                    stop = true;
                    break;
                }
                uint8_t *st = base + s * Cfg::STAGE_BYTES;
                if (rank == 0) mbar_expect_tx(&full[s], 2 * Cfg::STAGE_BYTES);
                const uint32_t fb = full0 + (uint32_t)(s * sizeof(uint64_t));
                const int kz = kr.x + j;  // the K block (64 entries, one contiguous nv0 x 64 slab per plane)
                tma_load_3d_pair(st, &tm_are, 0, arow0, kz, fb);
                tma_load_3d_pair(st + Cfg::TILE, &tm_aim, 0, arow0, kz, fb);
                if (SPLIT) {
                    tma_load_3d_pair(st + 2 * Cfg::TILE, &tm_are_lo, 0, arow0, kz, fb);
                    tma_load_3d_pair(st + 3 * Cfg::TILE, &tm_aim_lo, 0, arow0, kz, fb);
                }
                tma_load_3d_pair(st + Cfg::B_OFF, &tm_bre, 0, brow0, kz, fb);
                tma_load_3d_pair(st + Cfg::B_OFF + Cfg::TILE, &tm_bim, 0, brow0, kz, fb);
                *(volatile int *)issued = kb + 1;
            }
        }
    } else if (warp == 1 && lane == 0 && rank == 0) {
        // MMA issuer (leader only): plane slot i of the walk into the chain
        constexpr uint32_t idesc = umma_idesc_f16(256, 256);
        constexpr uint32_t idesc_neg = idesc | (1u << 13);  // negate A
        const uint32_t t_re = tmem, t_im = tmem + 256;
        int kb = 0, prev = 0, seg = 0;
        bool ok = true;
        for (int i = 0; i < pr.y && ok; ++i) {
            const int slot = last - i;
            const int P = pe.planes[slot];
            const bool start = i == 0 || !fq_chain1_continues(prev, P, seg, pe.n_uniform);
            seg = start ? 1 : seg + 1;
            prev = P;
            if (i >= 1) {  // both CTAs' epilogues have released the chain
                if (!mbar_wait(acc_empty, (i - 1) & 1, wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
            }
            const int nk = kranges[slot].y;
            for (int j = 0; j < nk; ++j, ++kb) {
                const int s = kb % S;
                if (!mbar_wait(&full[s], (kb / S) & 1, wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                uint8_t *st = base + s * Cfg::STAGE_BYTES;
                const uint64_t ar = umma_desc_sw128(st), ai = umma_desc_sw128(st + Cfg::TILE);
                const uint64_t br = umma_desc_sw128(st + Cfg::B_OFF), bi = umma_desc_sw128(st + Cfg::B_OFF + Cfg::TILE);
#pragma unroll
                for (int kk = 0; kk < TC_BK / 16; ++kk) {
                    const uint64_t adv = (uint64_t)(kk * 32) >> 4;
                    const uint32_t acc = (start && j == 0 && kk == 0) ? 0u : 1u;
                    umma_f16_pair(t_re, ar + adv, br + adv, idesc, acc);
                    umma_f16_pair(t_im, ai + adv, br + adv, idesc, acc);
                    umma_f16_pair(t_re, ai + adv, bi + adv, idesc_neg, 1u);
                    umma_f16_pair(t_im, ar + adv, bi + adv, idesc, 1u);
                    if (SPLIT) {
                        const uint64_t lr = umma_desc_sw128(st + 2 * Cfg::TILE) + adv;
                        const uint64_t li = umma_desc_sw128(st + 3 * Cfg::TILE) + adv;
                        umma_f16_pair(t_re, lr, br + adv, idesc, 1u);
                        umma_f16_pair(t_im, li, br + adv, idesc, 1u);
                        umma_f16_pair(t_re, li, bi + adv, idesc_neg, 1u);
                        umma_f16_pair(t_im, lr, bi + adv, idesc, 1u);
                    }
                }
                umma_commit_pair(&empty[s]);
            }
            if (ok) umma_commit_pair(acc_full);
        }
        if (!ok) atomicExch(abort_flag, 1);
        umma_commit_pair(done);  // both CTAs' done once every issued MMA has completed
    } else if (warp >= 4) {
        // epilogue (both CTAs, 8 warps): TMEM lane = row r1 = arow0 + 32 q +
        // lane (q = warp mod 4, the warp's lane quarter); warps 4-7 take
        // columns 0-127, warps 8-11 columns 128-255 (Re F in TMEM column c,
        // Im F in 256 + c).  The ratio table is read in chunks of 16 columns,
        // the next chunk's loads issued before this chunk's arithmetic, every
        // address valid (clamped to the grid) so the loads need no branches.
        const int q = warp & 3;
        const int cb = ((warp - 4) >> 2) * 128;
        const int r1 = arow0 + q * 32 + lane;
        const bool row_ok = r1 < N;
        const int64_t r1c = row_ok ? r1 : N - 1;
        const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
        const uint32_t empty0 = mapa_shared(smem_u32(acc_empty), 0);
        const float unscale = ldexpf(1.f, -fq_scale_exponent(pe.max_bits));
        auto col_idx = [&](int c) -> int64_t { return (int64_t)min(col0 + cb + c, N - 1) * pe.nv0 + r1c; };
        int prev = 0, seg = 0;
        for (int i = 0; i < pr.y; ++i) {
            const int slot = last - i;
            const int P = pe.planes[slot];
            const bool start = i == 0 || !fq_chain1_continues(prev, P, seg, pe.n_uniform);
            seg = start ? 1 : seg + 1;
            prev = P;
            const bool cont = i + 1 < pr.y && fq_chain1_continues(P, pe.planes[slot - 1], seg, pe.n_uniform);
            if (!__all_sync(0xffffffffu, mbar_wait(acc_full, i & 1, wait_ns)) && lane == 0) atomicExch(ep_fail, 1);
            asm volatile("bar.sync 1, 256;" ::: "memory");
            if (*(volatile int *)ep_fail) {
                atomicExch(abort_flag, 1);
                break;
            }
            tc_fence_after();
            if (cont) {
                // the chain continues: F <- r F in place (FP32)
                float2 f[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) f[t] = __ldg(&pe.r1step[col_idx(t)]);
#pragma unroll
                for (int c0 = 0; c0 < 128; c0 += 16) {
                    float2 g[16];
                    if (c0 + 16 < 128) {
#pragma unroll
                        for (int t = 0; t < 16; ++t) g[t] = __ldg(&pe.r1step[col_idx(c0 + 16 + t)]);
                    }
                    uint32_t re[16], im[16];
                    tmem_ld16_async(trow + cb + c0, re);
                    tmem_ld16_async(trow + 256 + cb + c0, im);
                    tmem_wait_ld();
#pragma unroll
                    for (int t = 0; t < 16; ++t) {
                        const float a = __uint_as_float(re[t]), b = __uint_as_float(im[t]);
                        re[t] = __float_as_uint(f[t].x * a - f[t].y * b);
                        im[t] = __float_as_uint(f[t].x * b + f[t].y * a);
                    }
                    tmem_st16(trow + cb + c0, re);
                    tmem_st16(trow + 256 + cb + c0, im);
                    if (c0 + 16 < 128) {
#pragma unroll
                        for (int t = 0; t < 16; ++t) f[t] = g[t];
                    }
                }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            } else {
                // the chain ends here: U += exp(zexp0 tz_P) F (factor in FP32
                // from FP64 phase and reduction; sum in FP64)
                const double tz = (pe.gz[P] + pe.gz[P + 1]) / 2;
#pragma unroll 1
                for (int c0 = 0; c0 < 128; c0 += 16) {
                    double2 z[16];
#pragma unroll
                    for (int t = 0; t < 16; ++t) z[t] = __ldg(&pe.zexp0[col_idx(c0 + t)]);
                    uint32_t re[16], im[16];
                    tmem_ld16_async(trow + cb + c0, re);
                    tmem_ld16_async(trow + 256 + cb + c0, im);
                    tmem_wait_ld();
#pragma unroll
                    for (int t = 0; t < 16; ++t) {
                        const int n = col0 + cb + c0 + t;
                        float sn, cs;
                        __sincosf((float)reduce_2pi(z[t].y * tz), &sn, &cs);
                        const float mag = expf((float)(z[t].x * tz)) * unscale;
                        const float a = __uint_as_float(re[t]), b = __uint_as_float(im[t]);
                        const float fx = mag * cs, fy = mag * sn;
                        if (row_ok && n < N) {
                            double *u = pe.U + 2 * ((int64_t)n * pe.nv0 + r1);
                            atomicAdd(u, (double)(fx * a - fy * b));
                            atomicAdd(u + 1, (double)(fx * b + fy * a));
                        }
                    }
                }
            }
            tc_fence_before();
            asm volatile("bar.sync 1, 256;" ::: "memory");
            if (q == 0 && cb == 0 && lane == 0) mbar_arrive_cluster(empty0);
        }
    }
    __syncwarp();

    const bool ok = mbar_wait(done, 0);
    tc_fence_after();
    __syncthreads();
    const bool failed = !ok || *(volatile int *)abort_flag;
    tc_fence_before();
    cluster_sync_all();
    if (threadIdx.x == 0) {
        // after a failure anywhere in the pair the leader waits (bounded) for
        // the pair's copies still in flight, which are counted on its barriers
        const int peer_abort = (int)ld_shared_cluster_u32(mapa_shared(smem_u32(abort_flag), rank ^ 1u));
        if (failed || peer_abort) {
            atomicExch(err, 1);
            if (rank == 0) {
                const int mine = *(volatile int *)issued;
                const int peer = (int)ld_shared_cluster_u32(mapa_shared(smem_u32(issued), 1));
                const int n_issued = max(mine, peer);
                for (int kb = (n_issued > S ? n_issued - S : 0); kb < n_issued; ++kb)
                    (void)mbar_wait(&full[kb % S], (kb / S) & 1);
            }
        }
    }
    cluster_sync_all();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC2_TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Rows of one chunk in FP16 K-major layouts, one CTA per group of 32 events:
// real-expanded rows (single-CTA kernel; lane = event, each row write is 32
// consecutive half2, 128 B) or planar rows (CTA pair).
// ---------------------------------------------------------------------------
// The per-event factors of 32 events (lane = event) in shared memory with row
// stride `ld` float2: views a (sa) and a0 (sa0, CBS), lights b (sb) and b2
// (sb2), the event scale sqrt(weight / px) (ssc) and the events (sev).
template <int DIM, bool SINGLE>
__device__ __forceinline__ void tc_rows_terms(const NeeParams &Q, const SingleRec &S, int64_t scap, const MultiRec &M,
                                              int64_t mcap, int64_t e0, int64_t g0, int ne, int ld, float2 *sa,
                                              float2 *sa0, float2 *sb, float2 *sb2, float *ssc, EventView *sev)
{
    const int nv = Q.nv, nl = Q.nl;
    if (threadIdx.x < 32) {
        EventView ev;
        if (threadIdx.x < ne) {
            load_event<DIM, SINGLE>(Q, S, scap, M, mcap, e0 + g0 + threadIdx.x, ev);
            ssc[threadIdx.x] = (float)sqrt(ev.wpx);
        } else {
            ssc[threadIdx.x] = 0.f;
            ev = EventView{};
        }
        sev[threadIdx.x] = ev;
    }
    __syncthreads();
    // lanes take consecutive directions of one event: the rays of one event to
    // nearby views (or lights) have about the same length, so a warp's
    // attenuation marches (heterogeneous medium) stay converged
    const int per = nv + nl;
    for (int idx = threadIdx.x; idx < 32 * per; idx += blockDim.x) {
        const int k = idx / per, m = idx - k * per;
        float2 p = make_float2(0.f, 0.f), q = make_float2(0.f, 0.f);
        if (k < ne) {
            const EventView &ev = sev[k];
            if (m < nv) {
                if (SINGLE) p = phaseatt<DIM, PMIX>(ev.x1, Q.vs + 3 * m, Q.is_ff_v, Q);
                else nee_view<DIM, PMIX, float2>(Q, m, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, p, q);
            } else {
                const int j = m - nv;
                if (SINGLE) p = phaseatt<DIM, PMIX>(ev.x1, Q.l + 3 * j, Q.is_ff_l, Q);
                else nee_light<DIM, PMIX, float2>(Q, j, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, p, q);
            }
        }
        if (m < nv) {
            sa[m * ld + k] = p;
            sa0[m * ld + k] = q;
        } else {
            sb[(m - nv) * ld + k] = p;
            sb2[(m - nv) * ld + k] = q;
        }
    }
    __syncthreads();
}

template <int DIM, bool SINGLE, bool SPLIT>
__global__ void __launch_bounds__(256)
tc_rows_kernel(const __grid_constant__ NeeParams Q, SingleRec S, int64_t scap, MultiRec M, int64_t mcap, int64_t e0, int64_t n_ev,
               int64_t K, __half *__restrict__ Ahi, __half *__restrict__ Alo, const float2 *__restrict__ af_tab)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nv = Q.nv, nl = Q.nl;
    float2 *sa = reinterpret_cast<float2 *>(smem_raw);  // [nv][33]
    float2 *sa0 = sa + nv * 33;
    float2 *sb = sa0 + nv * 33;                           // [nl][33]
    float2 *sb2 = sb + nl * 33;
    float *ssc = reinterpret_cast<float *>(sb2 + nl * 33);  // [32]
    EventView *sev = reinterpret_cast<EventView *>(ssc + 32);

    const int64_t g0 = (int64_t)blockIdx.x * 32;
    const int ne = (int)max((int64_t)0, min((int64_t)32, n_ev - g0));
    tc_rows_terms<DIM, SINGLE>(Q, S, scap, M, mcap, e0, g0, ne, 33, sa, sa0, sb, sb2, ssc, sev);
    // t_i, i = v + nv*l: light-outer, view-inner, so the light factor (times
    // the event scale) is loaded once per light and rows advance by pointer
    // increments (no integer division per entry).
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float sc = ssc[lane];
    const int64_t col = 2 * (g0 + lane);
    const int64_t step = 16 * K;  // 8 views = 16 real rows
    const bool cbs = !SINGLE && Q.cbs;
    for (int lj = 0; lj < nl; ++lj) {
        float2 bl = sb[lj * 33 + lane], bl2 = sb2[lj * 33 + lane];
        bl.x *= sc;
        bl.y *= sc;
        bl2.x *= sc;
        bl2.y *= sc;
        const int64_t i0 = (int64_t)nv * lj + warp;
        __half *ph = Ahi + 2 * i0 * K + col;
        __half *pl = Alo + 2 * i0 * K + col;
        for (int vi = warp; vi < nv; vi += 8, ph += step, pl += step) {
            float2 t = cmul(sa[vi * 33 + lane], bl);
            if (SINGLE) {
                const float2 af =
                    af_tab ? af_tab[vi + nv * lj] : to_c<float2>(single_amp<DIM>(Q, vi, lj, sev[lane].x1));
                t = cmul(t, af);
            } else if (cbs) {
                const float2 t2 = cmul(sa0[vi * 33 + lane], bl2);
                t.x += t2.x;
                t.y += t2.y;
            }
            const __half hr = __float2half_rn(t.x), hi = __float2half_rn(t.y);
            *reinterpret_cast<__half2 *>(ph) = __halves2half2(hr, hi);
            *reinterpret_cast<__half2 *>(ph + K) = __halves2half2(hi, __hneg(hr));
            if (SPLIT) {
                const __half lr = __float2half_rn(t.x - __half2float(hr));
                const __half li = __float2half_rn(t.y - __half2float(hi));
                *reinterpret_cast<__half2 *>(pl) = __halves2half2(lr, li);
                *reinterpret_cast<__half2 *>(pl + K) = __halves2half2(li, __hneg(lr));
            }
        }
    }
}

// NEE terms of the block's events toward directions m_lo .. m_lo + cnt - 1
// (views below nv, then lights) into p[(m - m_lo) * ld + k] and q[...]; lanes
// take consecutive directions of one event (converged heterogeneous marches).
template <int DIM, bool SINGLE>
__device__ __forceinline__ void tc_rows_dirs(const NeeParams &Q, const EventView *sev, int ne, int m_lo, int cnt,
                                             int ld, float2 *p_out, float2 *q_out)
{
    const int nv = Q.nv;
    for (int idx = threadIdx.x; idx < 32 * cnt; idx += blockDim.x) {
        const int k = idx / cnt, mm = idx - k * cnt, m = m_lo + mm;
        float2 p = make_float2(0.f, 0.f), q = make_float2(0.f, 0.f);
        if (k < ne) {
            const EventView &ev = sev[k];
            if (m < nv) {
                if (SINGLE) p = phaseatt<DIM, PMIX>(ev.x1, Q.vs + 3 * m, Q.is_ff_v, Q);
                else nee_view<DIM, PMIX, float2>(Q, m, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, p, q);
            } else {
                const int j = m - nv;
                if (SINGLE) p = phaseatt<DIM, PMIX>(ev.x1, Q.l + 3 * j, Q.is_ff_l, Q);
                else nee_light<DIM, PMIX, float2>(Q, j, ev.x, ev.ow, ev.x1, ev.w1, ev.w0p, p, q);
            }
        }
        p_out[mm * ld + k] = p;
        q_out[mm * ld + k] = q;
    }
}

// Shared memory of the planar rows kernel: view terms for vc views, light
// terms for all lights, 32 events each, plus the events.
inline size_t tc_rows_planar_smem(int vc, int nl)
{
    return sizeof(float2) * 32 * 2 * (size_t)(vc + nl) + 32 * sizeof(float) + 32 * sizeof(EventView) + 64;
}

// Planar rows (CTA-pair kernel): Re t_i and Im t_i in separate planes, rows of
// K events; Rhi / Rlo the Re planes, Ihi / Ilo the Im planes.  Lane = a pair
// of adjacent events and half-warp = a view, so each thread reads both
// events' factors with one 16-byte shared load, rounds them with one packed
// conversion and writes one half2 per plane.  The light terms are computed
// once; the view terms in chunks of vc views (all of them when they fit), so
// that with many views two CTAs still share an SM.
template <int DIM, bool SINGLE, bool SPLIT>
__global__ void __launch_bounds__(256)
tc_rows_planar_kernel(const __grid_constant__ NeeParams Q, SingleRec S, int64_t scap, MultiRec M, int64_t mcap, int64_t e0, int64_t n_ev,
                      int64_t K, __half *__restrict__ Rhi, __half *__restrict__ Rlo, __half *__restrict__ Ihi,
                      __half *__restrict__ Ilo, const float2 *__restrict__ af_tab, int vc)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nv = Q.nv, nl = Q.nl;
    float2 *sa = reinterpret_cast<float2 *>(smem_raw);  // [vc][32]
    float2 *sa0 = sa + vc * 32;
    float2 *sb = sa0 + vc * 32;  // [nl][32]
    float2 *sb2 = sb + nl * 32;
    float *ssc = reinterpret_cast<float *>(sb2 + nl * 32);  // [32]
    EventView *sev = reinterpret_cast<EventView *>(ssc + 32);

    const int64_t g0 = (int64_t)blockIdx.x * 32;
    const int ne = (int)max((int64_t)0, min((int64_t)32, n_ev - g0));
    if (threadIdx.x < 32) {
        EventView ev;
        if ((int)threadIdx.x < ne) {
            load_event<DIM, SINGLE>(Q, S, scap, M, mcap, e0 + g0 + threadIdx.x, ev);
            ssc[threadIdx.x] = (float)sqrt(ev.wpx);
        } else {
            ssc[threadIdx.x] = 0.f;
            ev = EventView{};
        }
        sev[threadIdx.x] = ev;
    }
    __syncthreads();
    tc_rows_dirs<DIM, SINGLE>(Q, sev, ne, nv, nl, 32, sb, sb2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h = lane >> 4, kp = lane & 15;  // view parity, event pair (events 2 kp, 2 kp + 1)
    const float s0 = ssc[2 * kp], s1 = ssc[2 * kp + 1];
    const float4 *sa4 = reinterpret_cast<const float4 *>(sa), *sa04 = reinterpret_cast<const float4 *>(sa0);
    const float4 *sb4 = reinterpret_cast<const float4 *>(sb), *sb24 = reinterpret_cast<const float4 *>(sb2);
    const int64_t col = g0 + 2 * kp;
    const int64_t step = 16 * K;  // 16 views
    const bool cbs = !SINGLE && Q.cbs;
    for (int vc0 = 0; vc0 < nv; vc0 += vc) {
        const int cnt = min(vc, nv - vc0);
        if (vc0 > 0) __syncthreads();  // the previous chunk's products have read sa / sa0
        tc_rows_dirs<DIM, SINGLE>(Q, sev, ne, vc0, cnt, 32, sa, sa0);
        __syncthreads();
        for (int lj = 0; lj < nl; ++lj) {
            float4 b = sb4[lj * 16 + kp], b2 = sb24[lj * 16 + kp];
            b = make_float4(b.x * s0, b.y * s0, b.z * s1, b.w * s1);
            b2 = make_float4(b2.x * s0, b2.y * s0, b2.z * s1, b2.w * s1);
            const int v0 = vc0 + 2 * warp + h;
            const int64_t o0 = ((int64_t)nv * lj + v0) * K + col;
            __half *pr = Rhi + o0, *pi = Ihi + o0, *qr = Rlo + o0, *qi = Ilo + o0;
            for (int vi = v0; vi < vc0 + cnt; vi += 16, pr += step, pi += step, qr += step, qi += step) {
                const float4 a = sa4[(vi - vc0) * 16 + kp];
                float2 t0 = cmul(make_float2(a.x, a.y), make_float2(b.x, b.y));
                float2 t1 = cmul(make_float2(a.z, a.w), make_float2(b.z, b.w));
                if (SINGLE) {
                    float2 f0, f1;
                    if (af_tab) {
                        f0 = f1 = af_tab[vi + nv * lj];
                    } else {
                        f0 = to_c<float2>(single_amp<DIM>(Q, vi, lj, sev[2 * kp].x1));
                        f1 = to_c<float2>(single_amp<DIM>(Q, vi, lj, sev[2 * kp + 1].x1));
                    }
                    t0 = cmul(t0, f0);
                    t1 = cmul(t1, f1);
                } else if (cbs) {
                    const float4 a0 = sa04[(vi - vc0) * 16 + kp];
                    const float2 u0 = cmul(make_float2(a0.x, a0.y), make_float2(b2.x, b2.y));
                    const float2 u1 = cmul(make_float2(a0.z, a0.w), make_float2(b2.z, b2.w));
                    t0.x += u0.x;
                    t0.y += u0.y;
                    t1.x += u1.x;
                    t1.y += u1.y;
                }
                const __half2 re = __floats2half2_rn(t0.x, t1.x), im = __floats2half2_rn(t0.y, t1.y);
                *reinterpret_cast<__half2 *>(pr) = re;
                *reinterpret_cast<__half2 *>(pi) = im;
                if (SPLIT) {
                    const float2 fr = __half22float2(re), fi = __half22float2(im);
                    *reinterpret_cast<__half2 *>(qr) = __floats2half2_rn(t0.x - fr.x, t1.x - fr.y);
                    *reinterpret_cast<__half2 *>(qi) = __floats2half2_rn(t0.y - fi.x, t1.y - fi.y);
                }
            }
        }
    }
}

// af(l_j . v_i) table for far-field single scattering, flattened i = v + nv*l.
template <int DIM>
__global__ void af_table_kernel(const __grid_constant__ NeeParams Q, float2 *__restrict__ tab)
{
    const int N = Q.nv * Q.nl;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int vi = i % Q.nv, lj = i / Q.nv;
        tab[i] = to_c<float2>(evalampfunc<DIM>(dot3<DIM>(Q.l + 3 * lj, Q.v + 3 * vi), Q.pf));
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct TcPlan {
    int N;
    bool split;
    // CTA-pair kernel on planar operands (256 x 256 complex tiles) instead of
    // the single-CTA kernel on real-expanded rows (128 real x 256 complex)
    bool pair;
    int64_t events_per_chunk;
    int64_t K;  // halves per operand row: 2 x events (real-expanded), events (planar)
    std::vector<int2> tiles;
    int stages = 2;  // pipeline stages of the CTA-pair kernel
};

struct TcOperands {
    __half *ahi, *alo;  // real-expanded rows; planar: the Re planes
    __half *ihi, *ilo;  // planar: the Im planes
    int2 *tiles;
    int *err;
    float2 *af;
    CUtensorMap m_ahi, m_alo, m_b;  // planar: m_ahi / m_alo / m_ihi / m_ilo are 128-row boxes of the planes
    CUtensorMap m_ihi, m_ilo;
    int n_tiles;
};

inline TcPlan tc_plan(int N, bool split, size_t chunk_bytes = (size_t)1 << 30, int64_t chunk_events = 0,
                      int stages = 0)
{
    TcPlan p;
    p.N = N;
    p.split = split;
    p.stages = (!split && stages == 3) ? 3 : 2;
    // The pair kernel pays off once its 256 complex rows are mostly real rows.
    p.pair = N >= 256;
    // Operand bytes per event: 8N (16N hi+lo) real-expanded, 4N (8N) planar;
    // keep a chunk's operands near chunk_bytes.  K blocks are 64 halves:
    // 32 events real-expanded, 64 planar.
    const int64_t per_event = (p.pair ? 4 : 8) * (split ? 2 : 1) * (int64_t)N;
    const int64_t eb = p.pair ? 64 : 32;
    // The error of the FP32 sums in TMEM grows in proportion to the chunk's
    // events (hi+lo on the 64 x 64 covariance, 1e5 paths: 2.0e-5 at 2048,
    // 4.0e-5 at 4096, 7.6e-5 at 8192, 2.6e-4 at 32768, at 0.88, 0.99, 1.05 and
    // 1.08e6 paths/s); once both operands are compensated it is the hi+lo
    // mode's only error of note, so that mode takes 4096-event chunks by
    // default (tunable up to 32768).  FP16 keeps 65536 (4.2e-4 in all, its
    // operands' rounding included).
    const int64_t e_max = split ? 32768 : 65536;
    int64_t e = chunk_events > 0 ? chunk_events : split ? 4096 : (int64_t)chunk_bytes / per_event;
    e = std::max<int64_t>(eb, std::min<int64_t>(e, e_max));
    e = (e / eb) * eb;
    p.events_per_chunk = e;
    p.K = p.pair ? e : 2 * e;
    const int bm_rows = p.pair ? 512 : TC_BM;  // real-expanded rows per tile
    const int n_tm = (2 * N + bm_rows - 1) / bm_rows;
    const int n_tn = (N + TC_BN - 1) / TC_BN;
    // Upper-triangle tiles (complex rows bm_rows/2 * tm .. against columns
    // TC_BN * tn ..) in blocks of GM x GN, so the CTAs of one wave share A row
    // blocks and B column blocks in L2 while they stream K.
    const int GM = p.pair ? 8 : 16, GN = 8;
    for (int bn = 0; bn < n_tn; bn += GN)
        for (int bm = 0; bm < n_tm; bm += GM)
            for (int tn = bn; tn < std::min(n_tn, bn + GN); ++tn)
                for (int tm = bm; tm < std::min(n_tm, bm + GM); ++tm)
                    if ((int64_t)(bm_rows / 2) * tm <= (int64_t)TC_BN * tn + TC_BN - 1) p.tiles.push_back(make_int2(tm, tn));
    return p;
}

inline size_t tc_align(size_t x) { return (x + 1023) & ~(size_t)1023; }

// Bytes of one operand part: 2N real-expanded rows, or one N-row plane.
inline size_t tc_part_bytes(const TcPlan &p)
{
    return tc_align((size_t)(p.pair ? 1 : 2) * p.N * p.K * sizeof(__half));
}

inline int tc_parts(const TcPlan &p) { return (p.split ? 2 : 1) * (p.pair ? 2 : 1); }

inline size_t tc_operand_bytes(const TcPlan &p)
{
    return tc_parts(p) * tc_part_bytes(p) + tc_align(p.tiles.size() * sizeof(int2)) + 1024 +
           tc_align((size_t)p.N * sizeof(float2));
}

inline PFN_cuTensorMapEncodeTiled_v12000 tc_encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            throw std::runtime_error("cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

inline CUtensorMap tc_map(const void *base, uint64_t cols, uint64_t rows, uint64_t row_stride_bytes, uint32_t box_rows)
{
    CUtensorMap m;
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {row_stride_bytes};
    cuuint32_t box[2] = {(cuuint32_t)TC_BK, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = tc_encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void *>(base), dims, strides, box,
                                estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed");
    return m;
}

// A K-block-major operand plane: [nblk][rows][64] FP16, boxes of 64 x 128 x 1.
inline CUtensorMap tc_map_kblocks(const void *base, uint64_t rows, uint64_t nblk)
{
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)TC_BK, rows, nblk};
    cuuint64_t strides[2] = {(cuuint64_t)TC_BK * 2, rows * TC_BK * 2};
    cuuint32_t box[3] = {(cuuint32_t)TC_BK, 128, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = tc_encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void *>(base), dims, strides, box,
                                estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed");
    return m;
}

inline TcOperands tc_make_operands(const TcPlan &p, void *mem, cudaStream_t st)
{
    TcOperands o{};
    char *b = reinterpret_cast<char *>(mem);
    const size_t a = tc_part_bytes(p);
    const size_t na = (size_t)tc_parts(p);
    // parts: Re hi [, Re lo] (real-expanded: A hi [, A lo]), then planar Im hi [, Im lo]
    o.ahi = reinterpret_cast<__half *>(b);
    o.alo = p.split ? reinterpret_cast<__half *>(b + a) : o.ahi;
    o.ihi = p.pair ? reinterpret_cast<__half *>(b + (p.split ? 2 : 1) * a) : nullptr;
    o.ilo = p.pair ? (p.split ? reinterpret_cast<__half *>(b + 3 * a) : o.ihi) : nullptr;
    o.tiles = reinterpret_cast<int2 *>(b + na * a);
    o.err = reinterpret_cast<int *>(b + na * a + tc_align(p.tiles.size() * sizeof(int2)));
    o.af = reinterpret_cast<float2 *>(reinterpret_cast<char *>(o.err) + 1024);
    o.n_tiles = (int)p.tiles.size();
    if (cudaMemcpyAsync(o.tiles, p.tiles.data(), p.tiles.size() * sizeof(int2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(o.err, 0, sizeof(int), st) != cudaSuccess)
        throw std::runtime_error("tcgen05 operand set-up failed");
    const uint64_t K = (uint64_t)p.K;
    if (p.pair) {
        o.m_ahi = tc_map(o.ahi, K, (uint64_t)p.N, K * 2, 128);
        o.m_alo = tc_map(o.alo, K, (uint64_t)p.N, K * 2, 128);
        o.m_ihi = tc_map(o.ihi, K, (uint64_t)p.N, K * 2, 128);
        o.m_ilo = tc_map(o.ilo, K, (uint64_t)p.N, K * 2, 128);
    } else {
        o.m_ahi = tc_map(o.ahi, K, 2 * (uint64_t)p.N, K * 2, TC_BM);
        o.m_alo = tc_map(o.alo, K, 2 * (uint64_t)p.N, K * 2, TC_BM);
        o.m_b = tc_map(o.ahi, K, (uint64_t)p.N, 2 * K * 2, TC_BN);
    }
    return o;
}

template <int DIM, bool SINGLE, bool SPLIT>
inline void tc_rows(const TcPlan &p, const TcOperands &o, const NeeParams &Q, const SingleRec &S, int64_t scap,
                    const MultiRec &M, int64_t mcap, int64_t e0, int64_t n, bool use_af_table, cudaStream_t st)
{
    const size_t smem = sizeof(float2) * 33 * 2 * (size_t)(Q.nv + Q.nl) + 32 * sizeof(float) +
                        32 * sizeof(EventView) + 64;
    const float2 *af = use_af_table ? o.af : nullptr;
    if (p.pair) {
        auto kern = tc_rows_planar_kernel<DIM, SINGLE, SPLIT>;
        // all views at once when two CTAs fit on an SM; else chunks of a multiple of 16 views
        constexpr size_t kTwoPerSm = 110 * 1024;
        int vc = Q.nv;
        while (vc > 16 && tc_rows_planar_smem(vc, Q.nl) > kTwoPerSm) vc = ((vc + 1) / 2 + 15) / 16 * 16;
        const size_t psmem = tc_rows_planar_smem(vc, Q.nl);
        if (psmem > 48 * 1024 &&
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem) != cudaSuccess)
            throw std::runtime_error("too many lights/views for the tensor-core row kernel");
        // every column of the 64-event blocks the product reads is written (zeros past n)
        const int grid = (int)((n + 63) / 64 * 2);
        kern<<<grid, 256, psmem, st>>>(Q, S, scap, M, mcap, e0, n, p.K, o.ahi, o.alo, o.ihi, o.ilo, af, vc);
    } else {
        auto kern = tc_rows_kernel<DIM, SINGLE, SPLIT>;
        if (smem > 48 * 1024 && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            throw std::runtime_error("too many lights/views for the tensor-core row kernel");
        const int grid = (int)((n + 31) / 32);
        kern<<<grid, 256, smem, st>>>(Q, S, scap, M, mcap, e0, n, p.K, o.ahi, o.alo, af);
    }
}

// D[ks][Mr][N] += A B^T over num_kb K-blocks, split ksplit ways along K.
template <bool SPLIT>
inline void tc_gemm_launch(const CUtensorMap &m_ahi, const CUtensorMap &m_alo, const CUtensorMap &m_b,
                           const int2 *tiles, int n_tiles, int num_kb, int ksplit, int Mr, int N, double *D, int *err,
                           cudaStream_t st)
{
    static std::atomic<uint64_t> attr_set{0};  // one bit per device ordinal
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cudaGetDevice failed");
    if (dev >= 64 || !((attr_set.load() >> dev) & 1)) {
        if (cudaFuncSetAttribute(herk_tc_kernel<SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcCfg<SPLIT>::SMEM_BYTES) != cudaSuccess)
            throw std::runtime_error("cannot reserve shared memory for the tensor-core kernel");
        if (dev < 64) attr_set.fetch_or((uint64_t)1 << dev);
    }
    const int kb_per = (num_kb + ksplit - 1) / ksplit;
    const int ks = (num_kb + kb_per - 1) / kb_per;  // every slice non-empty
    herk_tc_kernel<SPLIT><<<dim3((unsigned)n_tiles, (unsigned)ks), 128, TcCfg<SPLIT>::SMEM_BYTES, st>>>(
        m_ahi, m_alo, m_b, tiles, num_kb, kb_per, Mr, N, D, err, tc_test_fault().load());
}

// The plane-loop form: grid (tiles, plane ranges); pranges (device) holds
// n_ranges (first plane slot, plane count) pairs, kranges the K blocks of
// every plane slot, pe.planes the plane of every slot.
template <bool SPLIT>
inline void tc_gemm_plane_loop_launch(const CUtensorMap &m_ahi, const CUtensorMap &m_alo, const CUtensorMap &m_b,
                                      const int2 *tiles, int n_tiles, const int2 *kranges, const int2 *pranges,
                                      int n_ranges, int Mr, int N, const PlaneEpi &pe, int *err, cudaStream_t st)
// slots of one range must be in increasing plane order; the kernel walks them from the last
{
    static std::atomic<uint64_t> attr_set{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cudaGetDevice failed");
    if (dev >= 64 || !((attr_set.load() >> dev) & 1)) {
        if (cudaFuncSetAttribute(fq_planes_tc_kernel<SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcCfg<SPLIT>::SMEM_BYTES) != cudaSuccess)
            throw std::runtime_error("cannot reserve shared memory for the plane-loop tensor-core kernel");
        if (dev < 64) attr_set.fetch_or((uint64_t)1 << dev);
    }
    fq_planes_tc_kernel<SPLIT><<<dim3((unsigned)n_tiles, (unsigned)n_ranges), 256, TcCfg<SPLIT>::SMEM_BYTES, st>>>(
        m_ahi, m_alo, m_b, tiles, kranges, pranges, Mr, N, pe, err, tc_test_fault().load());
}

// The pair plane loop: grid (2 x tiles, plane ranges), clusters of 2.
template <bool SPLIT>
inline void fq_pair_planes_launch(const CUtensorMap *maps, const int2 *tiles, int n_tiles, const int2 *kranges,
                                  const int2 *pranges, int n_ranges, const PlaneEpi2 &pe, int *err, cudaStream_t st)
{
    constexpr int NS = SPLIT ? 2 : 3;
    using Cfg = Tc2Cfg<SPLIT, NS>;
    static std::atomic<uint64_t> attr_set{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cudaGetDevice failed");
    if (dev >= 64 || !((attr_set.load() >> dev) & 1)) {
        if (cudaFuncSetAttribute(fq_pair_planes_kernel<SPLIT, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Cfg::SMEM_BYTES) != cudaSuccess)
            throw std::runtime_error("cannot reserve shared memory for the FourierQuad pair kernel");
        if (dev < 64) attr_set.fetch_or((uint64_t)1 << dev);
    }
    fq_pair_planes_kernel<SPLIT, NS><<<dim3(2u * (unsigned)n_tiles, (unsigned)n_ranges), 384, Cfg::SMEM_BYTES, st>>>(
        maps[0], maps[1], maps[2], maps[3], maps[4], maps[5], tiles, kranges, pranges, pe, err,
        tc_test_fault().load());
}

// D[ks][2N][N] += the planar pair product (Re C in even rows, Im C in odd
// rows) over num_kb blocks of 64 events, split ksplit ways; tiles are 256 x 256
// complex rows x columns.
template <bool SPLIT, int NSTAGES>
inline void tc_gemm2_launch_stages(const TcOperands &o, int num_kb, int ksplit, int N, double *D, cudaStream_t st)
{
    using Cfg = Tc2Cfg<SPLIT, NSTAGES>;
    static std::atomic<uint64_t> attr_set{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cudaGetDevice failed");
    if (dev >= 64 || !((attr_set.load() >> dev) & 1)) {
        if (cudaFuncSetAttribute(herk_tc2_kernel<SPLIT, NSTAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Cfg::SMEM_BYTES) != cudaSuccess)
            throw std::runtime_error("cannot reserve shared memory for the CTA-pair tensor-core kernel");
        if (dev < 64) attr_set.fetch_or((uint64_t)1 << dev);
    }
    const int kb_per = (num_kb + ksplit - 1) / ksplit;
    const int ks = (num_kb + kb_per - 1) / kb_per;
    herk_tc2_kernel<SPLIT, NSTAGES><<<dim3(2u * (unsigned)o.n_tiles, (unsigned)ks), 128, Cfg::SMEM_BYTES, st>>>(
        o.m_ahi, o.m_ihi, o.m_alo, o.m_ilo, o.tiles, num_kb, kb_per, N, D, o.err, tc_test_fault().load());
}

// D[ks][2N][N] += the planar pair product (Re C in even rows, Im C in odd
// rows) over num_kb blocks of 64 events, split ksplit ways; tiles are 256 x 256
// complex rows x columns.  stages: 2, or 3 for the FP16 product.
template <bool SPLIT>
inline void tc_gemm2_launch(const TcOperands &o, int num_kb, int ksplit, int N, double *D, cudaStream_t st,
                            int stages = 2)
{
    if (!SPLIT && stages == 3) tc_gemm2_launch_stages<false, 3>(o, num_kb, ksplit, N, D, st);
    else tc_gemm2_launch_stages<SPLIT, 2>(o, num_kb, ksplit, N, D, st);
}

template <bool SPLIT>
inline void tc_herk_launch(const TcPlan &p, const TcOperands &o, int64_t n, double *D, cudaStream_t st)
{
    if (p.pair) {
        const int num_kb = (int)((n + TC_BK - 1) / TC_BK);  // 64 events per block
        tc_gemm2_launch<SPLIT>(o, num_kb, 1, p.N, D, st, p.stages);
    } else {
        const int num_kb = (int)((2 * n + TC_BK - 1) / TC_BK);
        tc_gemm_launch<SPLIT>(o.m_ahi, o.m_alo, o.m_b, o.tiles, o.n_tiles, num_kb, 1, 2 * p.N, p.N, D, o.err, st);
    }
}

inline void tc_herk(const TcPlan &p, const TcOperands &o, int64_t n, double *D, cudaStream_t st)
{
    if (p.split) tc_herk_launch<true>(p, o, n, D, st);
    else tc_herk_launch<false>(p, o, n, D, st);
}

}  // namespace scmc
