/*
 * scmc_oracle.h - CPU FP64 restatement of SCMC's Monte Carlo path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; nothing in the product links it.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.
 *
 * Parity pin: tests/golden/ holds outputs of the reference's own .m files
 * (code/MCfield.m, code/MCcov.m, code/MCfieldFourierQuad.m and the
 * coreFunctions they call) executed unmodified by a MATLAB-subset
 * interpreter with rand/randn served from recorded tapes.  In tape mode this
 * oracle consumes the same tapes in the same order and must reproduce those
 * outputs; in Philox mode it consumes the per-path counter-based streams the
 * GPU walk uses.
 */
#ifndef SCMC_ORACLE_H
#define SCMC_ORACLE_H

#include "../include/scmc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_RNG_TAPE = 0, ORACLE_RNG_PHILOX = 1 };

typedef struct {
    int32_t mode;
    const double *utape; int64_t un;   /* rand() tape (mode TAPE) */
    const double *ntape; int64_t nn;   /* randn() tape (mode TAPE) */
    int64_t used_u, used_n;            /* out: draws consumed */
} oracle_rng_spec;

/* MCfield.m:1-254.  u: 2*nv*nl doubles.  Returns 0, or -1 when a tape ran out. */
int oracle_field(const scmc_mc_args *a, oracle_rng_spec *rs, double *u);

/* MCfieldOnWave.m:1-267: the field of the lights combined with complex
 * weights Wl (2*nl doubles, interleaved).  u: 2*nv doubles. */
int oracle_field_onwave(const scmc_mc_args *a, const double *Wl, oracle_rng_spec *rs, double *u);

/* MCcov.m:1-299.  Ms, Mm: 2*nv*nv*nl*nl doubles.  threads<=1: serial. */
int oracle_cov(const scmc_mc_args *a, oracle_rng_spec *rs, double *Ms, double *Mm, int threads);

/* Walk only, writing records in the layout of scmc_export_records. */
int oracle_records(const scmc_mc_args *a, oracle_rng_spec *rs, int32_t want_phase,
                   int64_t capacity, double *x, double *ow, double *x1, double *w1,
                   double *wpx, double *xi, int32_t *plen, int64_t *path, int64_t *n_events);

/* Accumulate records (from any walk) with MCfield's / MCcov's NEE and update
 * rules, then normalise by a->norm_itr (or a->max_itr). */
int oracle_field_from_records(const scmc_mc_args *a, int64_t n, const double *x,
                              const double *ow, const double *x1, const double *w1,
                              const double *wpx, const double *xi, const int32_t *plen,
                              double *u);
int oracle_cov_from_records(const scmc_mc_args *a, int64_t n, const double *x,
                            const double *ow, const double *x1, const double *w1,
                            const double *wpx, const int32_t *plen,
                            double *Ms, double *Mm, int threads);

/* MCfieldFourierQuad.m:1-304 (isotropic walk, z-plane quadrature, lateral
 * gridding and a 2-D DFT per plane and light).  u: 2*nv0*nv0*nl doubles. */
int oracle_field_fourier_quad(const scmc_fq_args *a, oracle_rng_spec *rs, double *u);
/* MCfieldFourierQuadOnWave.m:1-337: the lights combined with weights Wl
 * (2*nl doubles, interleaved) into one output.  u: 2*nv0*nv0 doubles.
 * as_written = 1: the light weight of a plane's j3-th vertex is evaluated at
 * the j3-th vertex of the whole depth-sorted list, as lines 282-292 do;
 * 0: at the vertex itself (line 279's formula, the GPU's). */
int oracle_field_fourier_quad_onwave(const scmc_fq_args *a, const double *Wl, int32_t as_written,
                                     oracle_rng_spec *rs, double *u);

/* MCCovHetro.m:1-276 (Ms, Mm, mean1) and MCsampleHetro.m:1-227 (u). */
int oracle_cov_hetero(const scmc_hetero_args *a, oracle_rng_spec *rs, double *Ms, double *Mm, double *mean1,
                      int threads);
int oracle_field_hetero(const scmc_hetero_args *a, oracle_rng_spec *rs, double *u);

/* refocus.m:1-34: rU (2*N doubles, N grid points, x fastest).  v: dim x nv
 * column-major directions, l: dim, u: 2*nv doubles.  as_written = 1 leaves
 * the first grid point at 0, as the reference's chunk indices do. */
int64_t oracle_refocus_grid(int32_t dim, const double *box_min, const double *box_max, const double *box_stp,
                            int64_t *dims);
int oracle_refocus(const double *u, const double *v, int64_t nv, int32_t dim, const double *l,
                   const double *box_min, const double *box_max, const double *box_stp, double lambda,
                   int32_t as_written, double *rU);
/* samplingFromCovMatrix.m:47-64: Z (2*N*n_samples doubles) from C (2*N*N
 * doubles) and normals (2N per sample).  -1 if Sigma is not positive definite. */
int oracle_sample_cov(const double *C, int64_t N, int64_t n_samples, const double *normals, double *Z);

/* Philox-4x32-10 (Salmon et al., SC'11): one block. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The per-path streams (tag 0 uniform, tag 1 normal) of the walk. */
void oracle_philox_stream(uint64_t seed, uint64_t path, int32_t tag, int64_t n, double *out);

#ifdef __cplusplus
}
#endif
#endif
