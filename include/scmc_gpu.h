/*
 * scmc_gpu.h - C ABI of the B200 (sm_100a) Monte Carlo speckle path.
 *
 * This library replaces the Monte Carlo kernels of SCMC (cmu-ci-lab/mcspeckle):
 * the random walk through a box medium, next-event estimation (NEE) from the
 * first and last scatterer to every light and view, and the complex phase
 * accumulation into a speckle field u(v,l) or covariance C(v1,v2,l1,l2).
 *
 * Every entry point takes plain pointers and sizes.  Arrays follow MATLAB's
 * storage: real matrices column-major, complex values interleaved (re, im)
 * as in MATLAB R2018a+ interleaved complex.  All host-side outputs are
 * written only on success.  A non-zero return is an scmc_status; the message
 * is available from scmc_last_error() on the calling thread.
 */
#ifndef SCMC_GPU_H
#define SCMC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCMC_ABI_VERSION 2

typedef enum {
    SCMC_OK = 0,
    SCMC_ERR_INVALID = 1,   /* argument validation; message mirrors the reference's error() */
    SCMC_ERR_CUDA = 2,      /* CUDA runtime / driver error */
    SCMC_ERR_NOMEM = 3,     /* device or host allocation failed */
    SCMC_ERR_NODEVICE = 4,  /* no sm_100 device visible */
    SCMC_ERR_TIMEOUT = 5,   /* a bounded device wait gave up */
    SCMC_ERR_CANCELLED = 6, /* request cancelled through the serving API */
    SCMC_ERR_LIMIT = 7      /* a path exceeded max_events_per_path */
} scmc_status;

/* sct_type values, as in scmc.m:249-287 (1 isotropic, 2 tabulated, 3 HG). */
enum { SCMC_SCT_ISOTROPIC = 1, SCMC_SCT_TABULATED = 2, SCMC_SCT_HG = 3 };

/* Arithmetic of the NEE phase vectors and of the contraction.
 *  FP64  - reference arithmetic (every step in double); parity mode.
 *  MIXED - phase argument k*(w.x) reduced mod 2pi in FP64, sincos/exp in FP32,
 *          contraction on tcgen05 tensor cores with FP16 hi+lo split operands
 *          and FP32 accumulation, cross-batch sums in FP64.  The covariance
 *          compensates both operands (three products per term) in 4096-event
 *          chunks: about a tenth of FP16's error at a third of its speed; the
 *          field and FourierQuad forms compensate one operand.
 *  FP32  - plain FP32: FP32 phases without FP64 reduction, FP32 CUDA-core
 *          contraction, FP32 accumulation (the comparison baseline).
 *  FP16  - as MIXED but one FP16 product (no lo part), chunks of up to 65536
 *          events: the fastest mode, within 1e-3 of FP64.
 * The random walk itself is FP64 in every mode, so all modes see the same
 * paths for the same seed. */
enum { SCMC_PREC_FP64 = 0, SCMC_PREC_MIXED = 1, SCMC_PREC_FP32 = 2, SCMC_PREC_FP16 = 3 };

/* One scattering function: the (sct_type, ampfunc) pair of MCfield.m:1.
 * For SCMC_SCT_TABULATED the two tables are the fields evalAmp and
 * sampleIcdf built by tabulatedAmplitudeScatter.m:78-99. */
typedef struct {
    int32_t sct_type;
    double g;                  /* HG anisotropy (ampfunc for sct_type 3) */
    int32_t table_n;           /* length of the tabulated tables */
    const double *eval_amp;    /* 2*table_n doubles: interleaved complex evalAmp */
    const double *sample_icdf; /* table_n doubles: sampleIcdf (angles) */
    int32_t table_in_cos;      /* extension, 3-D only: 0 = the reference's tables on angle bins
                                  (evalAmp at theta_i = i pi/(n-1), sampleIcdf angles); 1 = on cos(theta)
                                  bins: evalAmp at cos_i = 1 - 2i/(n-1), sampleIcdf holds cosines */
} scmc_phase_function;

/* Positional arguments of MCfield / MCcov (MCfield.m:1, MCcov.m:1) plus the
 * execution controls that MATLAB's list has no slot for. */
typedef struct {
    int32_t dim;               /* 2 or 3: size(box_min,1) */
    double sigt;               /* extinction coefficient 1/MFP */
    double albedo;
    double box_min[3];
    double box_max[3];
    const double *l;           /* dim x nl, column-major (directions or positions) */
    int64_t nl;
    const double *v;           /* dim x nv, column-major */
    int64_t nv;
    int32_t is_ff_l;
    int32_t is_ff_v;
    int64_t max_itr;           /* number of paths (maxItr) */
    double lambda;
    int32_t do_cbs;
    int32_t smp_flg;           /* 1 uniform, 2 exponential first scatter */
    scmc_phase_function ampfunc;
    int32_t has_ampfunc0;      /* 15th argument present */
    scmc_phase_function ampfunc0;
    int32_t has_lmean0;        /* 16th argument of MCfield present */
    double lmean0[3];
    /* --- execution controls --- */
    uint64_t seed;             /* Philox-4x32-10 key */
    uint64_t path_offset;      /* global index of the first path (sharding / replicas) */
    int64_t norm_itr;          /* path count used in the normalisation; 0 = max_itr */
    int32_t precision;         /* SCMC_PREC_* */
    int32_t device;            /* CUDA ordinal */
    int64_t max_events_per_path; /* 0 = unlimited; exceeding it fails with SCMC_ERR_LIMIT */
} scmc_mc_args;

/* Positional arguments of MCfieldFourierQuad (MCfieldFourierQuad.m:1). */
typedef struct {
    double sigt;
    double albedo;
    double box_min[3];
    double box_max[3];
    const double *l;           /* 3 x nl light directions */
    int64_t nl;
    double v_max;
    double v_stp;
    int64_t max_itr;
    double lambda;
    int32_t do_cbs;
    int32_t smp_flg;
    int32_t has_lmean0;
    double lmean0[3];
    double vsign;              /* -1 or +1 */
    uint64_t seed;
    uint64_t path_offset;
    int32_t precision;
    int32_t device;
    /* --- extensions (zero = the reference's isotropic plane-wave form) --- */
    int32_t light_point;       /* 1: l holds point-source positions; each vertex's light factor is
                                  evalphaseatt.m:10-16's near-field term (phase k|x - s|, attenuation
                                  sigt/2 min(cubeDist, |x - s|), 1/(|x - s| + 0.01 lambda)) instead of the
                                  plane wave of MCfieldFourierQuad.m:272 */
    int32_t sct_type;          /* 0 or SCMC_SCT_ISOTROPIC: isotropic walk (MCfieldFourierQuad.m:208);
                                  SCMC_SCT_HG: scattering directions sampled from HG(g) as
                                  smpampfunc_general does (the call left commented out at line 208) */
    double g;
} scmc_fq_args;

/* ---------------------------------------------------------------------------
 * Field: u = MCfield(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v,
 *                     maxItr, lambda, doCBS, smpFlg, sct_type, ampfunc
 *                     [, ampfunc0 [, lmean0]])                  (MCfield.m:1)
 * u: nv x nl complex, interleaved, host memory (2*nv*nl doubles).
 * ------------------------------------------------------------------------- */
int scmc_field(const scmc_mc_args *args, double *u);

/* Same, with u in device memory (2*nv*nl doubles) and work on `stream`
 * (a cudaStream_t, NULL = legacy default stream).  Returns after the work is
 * enqueued and the batch bookkeeping synchronised. */
int scmc_field_device(const scmc_mc_args *args, double *d_u, void *stream);

/* Field without any device allocation.  For callers that cannot allocate
 * device memory while they call in: a process that reserved its GPU memory
 * budget up front, a real-time loop that must not take the allocator's locks
 * or let cudaFree synchronise the device, or a host thread on which
 * cudaMalloc / cudaFree are not allowed.  Same estimator as
 * scmc_field_device, with every piece of device scratch in one fixed 32 MiB
 * array inside the library, which each GPU that loads the library holds
 * until the process exits.  No counterpart in the reference (MATLAB manages
 * memory for its callers).
 * d_u: device memory, 2*nv*nl doubles.  Limits: nv*nl <= 65536, tabulated
 * tables <= 16384 entries, and no single path longer than the scratch holds
 * (about 400k events); beyond them it returns SCMC_ERR_INVALID.  The
 * accumulation is always the CUDA-core one: in MIXED / FP16 mode with
 * nv >= 64 and nl >= 32, where scmc_field_device uses tensor cores, the two
 * agree within the mixed tolerance rather than bit for bit.  The first call on
 * a device looks up the array's device address, so make that call before any
 * stream capture.  All calls share the array and it keeps the previous call's
 * contents (each call clears what must start at zero); two calls whose work
 * overlapped on the GPU would race on it, so the library serialises the calls
 * on one device and returns only after the call's work on `stream` has
 * finished (on an error return too). */
int scmc_field_noalloc(const scmc_mc_args *args, double *d_u, void *stream);

/* ---------------------------------------------------------------------------
 * Field on a wave: u = MCfieldOnWave(sigt, albedo, box_min, box_max, l, v,
 *     is_ff_l, is_ff_v, maxItr, lambda, doCBS, smpFlg, sct_type, ampfunc,
 *     ampfunc0, lmean0, Wl)                               (MCfieldOnWave.m:1)
 * The field of all lights at once, each weighted by the complex Wl_j: equal
 * to the MCfield result times Wl on the same paths, at O(nv + nl) instead of
 * O(nv nl) work per event.  Wl: nl complex (2*nl doubles, interleaved; the
 * reference needs it as a 1 x Nl row).  u: nv complex (2*nv doubles).  The
 * reference requires ampfunc0 and lmean0 (positional); here they may be
 * omitted (has_ampfunc0 / has_lmean0 = 0) with MCfield's defaults.  For
 * isotropic scattering the reference's single-scattering line
 * (MCfieldOnWave.m:221) is consistent only for one light; this computes
 * sum_j af e_l0_j Wl_j, which agrees with it there.
 * ------------------------------------------------------------------------- */
int scmc_field_onwave(const scmc_mc_args *args, const double *Wl, double *u);
/* Same with u in device memory (Wl stays in host memory) and work on `stream`. */
int scmc_field_onwave_device(const scmc_mc_args *args, const double *Wl, double *d_u, void *stream);

/* ---------------------------------------------------------------------------
 * Covariance: [Ms, Mm] = MCcov(sigt, albedo, box_min, box_max, l, v, is_ff_l,
 *                  is_ff_v, maxItr, lambda, doCBS, smpFlg, sct_type, ampfunc
 *                  [, ampfunc0])                                 (MCcov.m:1)
 * Ms, Mm: nv x nv x nl x nl complex (v1 fastest, then v2, l1, l2),
 * interleaved, host memory (2*nv*nv*nl*nl doubles each).  Either may be NULL
 * to skip copying it out.
 * ------------------------------------------------------------------------- */
int scmc_cov(const scmc_mc_args *args, double *Ms, double *Mm);

/* Same with Ms, Mm in device memory. */
int scmc_cov_device(const scmc_mc_args *args, double *d_Ms, double *d_Mm, void *stream);

/* ---------------------------------------------------------------------------
 * Heterogeneous (voxel) medium:
 *   [Ms, Mm, mean1] = MCCovHetro(sigt, albedo, box_min, box_max, box_bin, l, v,
 *        is_ff_l, is_ff_v, maxItr, lambda, doCBS, smpFlg, sct_type, ampfunc
 *        [, ampfunc0 [, lrad]])                              (MCCovHetro.m:1)
 *   u = MCsampleHetro(sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l,
 *        is_ff_v, maxItr, lambda, doCBS, smpFlg, sct_type, ampfunc
 *        [, ampfunc0 [, lmean0]])                          (MCsampleHetro.m:1)
 * `mc` carries the shared positional arguments (mc.sigt is unused: sigt is
 * the voxel grid).  Voxels follow findBin.m: nb = round((box_max-box_min)./
 * box_bin) per axis, x fastest.  Free flights are delta (Woodcock) tracking
 * against max(sigt) (smpWoodcock.m), NEE attenuation marches voxel to voxel
 * (evalphaseattHetro.m).  smpFlg 1 picks the first voxel with probability
 * proportional to sigt (invCDFvec.m / smpicdf.m); smpFlg 2 launches from a
 * plane (expSmpXHetro.m), whose lateral axes are null(meanl') - passed in
 * null_basis as MATLAB's SVD-based null() gives them (dim x (dim-1),
 * column-major).  Outputs as MCcov / MCfield; mean1: nv x nl complex.
 * ------------------------------------------------------------------------- */
typedef struct {
    scmc_mc_args mc;
    const double *sigt_grid;    /* prod(nb) extinction values */
    const double *albedo_grid;  /* prod(nb) albedos, or NULL for the scalar mc.albedo */
    double box_bin[3];
    int32_t has_lrad;           /* 17th argument of MCCovHetro (plane launch radius) */
    double lrad;
    double null_basis[6];
    int32_t trilinear;          /* extension: 0 = the reference's nearest voxel (findBin.m); 1 = sigt
                                   interpolated trilinearly between voxel centres (clamped at the faces)
                                   in the Woodcock acceptance, the attenuation integral (exact per
                                   piece between voxel-centre planes) and the first-scatter weight;
                                   per-voxel albedo stays nearest */
} scmc_hetero_args;

int scmc_cov_hetero(const scmc_hetero_args *args, double *Ms, double *Mm, double *mean1);
int scmc_field_hetero(const scmc_hetero_args *args, double *u);
/* Same with the outputs in device memory and the work on `stream`. */
int scmc_cov_hetero_device(const scmc_hetero_args *args, double *d_Ms, double *d_Mm, double *d_mean1, void *stream);
int scmc_field_hetero_device(const scmc_hetero_args *args, double *d_u, void *stream);

/* ---------------------------------------------------------------------------
 * Path records for oracle replay.  Walks paths [path_offset, path_offset +
 * max_itr) exactly as scmc_field (want_phase=1) or scmc_cov (want_phase=0)
 * do and copies out one record per scattering event, in path order:
 *   x[3*e..]   event position           ow[3*e..] incoming direction
 *   x1[3*e..]  first scatterer           w1[3*e..] first outgoing direction
 *   wpx[e]     weight/px                 xi[e]     random-phase uniform (field)
 *   plen[e]    1-based event index in its path (pL)
 *   path[e]    path index relative to path_offset
 * Each array has room for `capacity` events; *n_events receives the count
 * (also when it exceeds capacity, in which case nothing is written and
 * SCMC_ERR_LIMIT is returned).  Arrays for dim=2 still use stride 3.
 * ------------------------------------------------------------------------- */
int scmc_export_records(const scmc_mc_args *args, int32_t want_phase, int64_t capacity,
                        double *x, double *ow, double *x1, double *w1, double *wpx,
                        double *xi, int32_t *plen, int64_t *path, int64_t *n_events);

/* The field (MCfield.m:207-254 accumulation and normalisation) of n stored
 * records in the layout above, on the GPU: records exported on one machine
 * (and kept in the on-disk record format of mcspeckle_b200.formats) replay
 * on another.  args supplies the lights, views, medium and normalisation
 * (norm_itr, else max_itr); its walk-only fields are not used.  No
 * counterpart in the reference (it never stores its paths). */
int scmc_field_from_records(const scmc_mc_args *args, int64_t n, const double *x, const double *ow,
                            const double *x1, const double *w1, const double *wpx, const double *xi,
                            const int32_t *plen, const int64_t *path, double *u);

/* Philox-4x32-10 uniform / normal streams of one path, as used by the walk:
 * n values of stream `tag` (0 uniform, 1 normal) of path `path` under `seed`.
 * Host memory.  Exposed so the random streams can be checked bit for bit. */
int scmc_philox_stream(uint64_t seed, uint64_t path, int32_t tag, int64_t n, double *out);

/* ---------------------------------------------------------------------------
 * u = MCfieldFourierQuad(sigt, albedo, box_min, box_max, l, v_max, v_stp,
 *                        maxItr, lambda, doCBS, smpFlg, lmean0, vsign)
 *                                                 (MCfieldFourierQuad.m:1)
 * u: nv0 x nv0 x nl complex interleaved, nv0 = length(-v_max:v_stp:v_max)
 * (scmc_fq_grid_size).  Lights are 3 x nl directions.  The reference's FFT
 * needs integer padding (odd nv0); for even nv0 the same centred-DFT formula
 * is evaluated with half-integer offsets.
 * ------------------------------------------------------------------------- */
int scmc_fq_grid_size(double v_max, double v_stp, int64_t *nv0);
int scmc_field_fourier_quad(const scmc_fq_args *args, double *u);
int scmc_field_fourier_quad_device(const scmc_fq_args *args, double *d_u, void *stream);

/* u = MCfieldFourierQuadOnWave(sigt, albedo, box_min, box_max, l, v_max,
 *       v_stp, maxItr, lambda, doCBS, smpFlg, lmean0, Wl, vsign)
 *                                             (MCfieldFourierQuadOnWave.m:1)
 * The lights combined with complex weights Wl (2*nl doubles, interleaved,
 * host memory) into one nv0 x nv0 field (2*nv0*nv0 doubles), with that
 * file's conventions: the lateral pixel count takes the parity of the angular
 * grid (so even grids need no half-integer padding), vsign enters the light
 * and vertex phases and zexp0 has the opposite phase sign.  The light weight
 * of each vertex is evaluated at that vertex (the formula of line 279); the
 * reference's lines 282-292 evaluate the plane's j-th weight at the j-th
 * vertex of the whole depth-sorted list instead. */
int scmc_field_fourier_quad_onwave(const scmc_fq_args *args, const double *Wl, double *u);
int scmc_field_fourier_quad_onwave_device(const scmc_fq_args *args, const double *Wl, double *d_u, void *stream);

/* ---------------------------------------------------------------------------
 * Stage timing.  While enabled, every kernel launch of the walk, the row
 * generation, the contraction and the finalisation is bracketed by CUDA
 * events on the stream it runs on; scmc_profile_read resolves them.  The
 * reference has only tic/toc in its scripts; this is the per-stage form.
 * ------------------------------------------------------------------------- */
typedef struct {
    int64_t walk_launches;
    double walk_ms;
    int64_t rows_launches;      /* NEE vectors + rows / field accumulation */
    double rows_ms;
    int64_t contract_launches;  /* Hermitian rank-k updates (tensor / CUDA cores) */
    double contract_ms;
    int64_t finalize_launches;
    double finalize_ms;
    int64_t paths;              /* paths walked */
    int64_t events;             /* scattering events (single + multiple) */
    double contract_flops;      /* algorithmic: 4*N*(N+1) per event, N = nv*nl */
    double contract_busy_ms;    /* time with at least one contraction in flight (launches on
                                   several streams overlap; each instant counts once) */
    double rows_busy_ms;        /* the same for the row generation */
} scmc_stage_times;

int scmc_profile_enable(int32_t on);
int scmc_profile_read(scmc_stage_times *out, int32_t reset);

/* ---------------------------------------------------------------------------
 * Serving: a request server for streams of MCfield / MCcov solves of uneven
 * sizes.  No reference counterpart (the reference solves one call at a time
 * in the MATLAB interpreter, parfor workers aside: scmc.m:421-445); the
 * requests are exactly scmc_field / scmc_cov calls, with the same arguments
 * and results.
 *
 * The server owns n_slots worker slots, each with its own CUDA stream and
 * scratch memory (stream-ordered allocations).  A submitted request waits in
 * the queue until a slot is free and its estimated device memory fits the
 * HBM budget next to the requests already running (oldest first; a request
 * that does not fit is passed by younger ones a bounded number of times);
 * then it runs on that slot's stream, so requests on different slots overlap
 * on the device.  Small field requests on the CUDA-core accumulation (up to
 * 2^20 paths, same dimension and precision class) are packed: up to 64 run
 * as one walk, one accumulation and one finalisation launch per round of
 * 2^20 paths.  The
 * output arrays stay owned by the caller and must stay valid until
 * scmc_server_wait has reported the request finished.  A request's result does
 * not depend on what else runs: each path draws from its own Philox stream
 * and every accumulator is private to the slot.
 * ------------------------------------------------------------------------- */
typedef struct scmc_server scmc_server;

enum { SCMC_REQ_FIELD = 0, SCMC_REQ_COV = 1 };

typedef struct {
    int64_t ticket;
    int32_t kind;           /* SCMC_REQ_* */
    int32_t slot;           /* worker slot that ran it (-1 while queued) */
    int32_t status;         /* scmc_status of the solve once finished */
    int32_t finished;       /* 0 queued or running, 1 finished */
    double submit_ms;       /* host steady clock, ms since the server was created */
    double start_ms;        /* admitted to a slot */
    double done_ms;         /* result copied to the caller's arrays */
    double device_ms;       /* CUDA-event time on the slot stream, first to last launch */
    int64_t reserved_bytes; /* device memory reserved against the budget */
    int64_t peak_bytes;     /* device memory the slot actually held for it (for a pack: the pack) */
    int64_t paths;          /* max_itr of the request */
    int32_t packed;         /* requests that shared its launches (1: it ran alone) */
} scmc_request_info;

typedef struct {
    int32_t n_slots;
    int32_t busy_slots;
    int64_t queued;
    int64_t completed;
    int64_t failed;
    int64_t budget_bytes;
    int64_t reserved_bytes;      /* now */
    int64_t peak_reserved_bytes; /* high-water mark */
    int64_t paths_completed;
} scmc_server_stats;

/* hbm_budget_bytes <= 0: 80% of the device's free memory at creation. */
int scmc_server_create(int32_t device, int32_t n_slots, int64_t hbm_budget_bytes, scmc_server **out);
/* kind SCMC_REQ_FIELD: out0 = u (2*nv*nl doubles), out1 unused.
 * kind SCMC_REQ_COV: out0 = Ms, out1 = Mm (each 2*(nv*nl)^2 doubles; either may
 * be NULL).  Arguments are validated and copied at submission; a request
 * whose estimate alone exceeds the budget is refused with SCMC_ERR_NOMEM. */
int scmc_server_submit(scmc_server *s, int32_t kind, const scmc_mc_args *args, double *out0, double *out1,
                       int64_t *ticket);
/* Waits up to timeout_ms (< 0: no limit) for the request.  Returns the
 * request's status when it has finished (its message via scmc_last_error),
 * SCMC_ERR_TIMEOUT while it has not; info (may be NULL) is filled either way.
 * A finished request's record is dropped after the first successful wait. */
int scmc_server_wait(scmc_server *s, int64_t ticket, int64_t timeout_ms, scmc_request_info *info);
int scmc_server_stats_read(scmc_server *s, scmc_server_stats *out);
/* Runs the requests already admitted to completion, cancels the queued ones
 * (SCMC_ERR_CANCELLED) and frees the server. */
int scmc_server_destroy(scmc_server *s);

/* ---------------------------------------------------------------------------
 * Post-processing.
 *
 * rU = refocus(u, v, l, box_min, box_max, box_stp, lambda)    (refocus.m:1)
 * The field of nv far-field views u (2*nv doubles) back-propagated onto the
 * grid ndgrid(box_min(k):box_stp(k):box_max(k), ...) (dim 2 or 3, x fastest)
 * with light direction l:  rU(p) = (sum_v conj(u_v) exp(-2 pi i/lambda
 * v.p)) exp(2 pi i/lambda l.p).  v: dim x nv column-major.  rU: 2*N doubles,
 * N = prod(dims) from scmc_refocus_grid.  as_written = 1 leaves the first
 * grid point at 0 as the reference's chunk indices do (refocus.m:27).
 * precision: SCMC_PREC_FP64 or SCMC_PREC_MIXED (phase reduced in FP64,
 * sincos in FP32).
 * ------------------------------------------------------------------------- */
int scmc_refocus_grid(int32_t dim, const double *box_min, const double *box_max, const double *box_stp,
                      int64_t *dims, int64_t *n);
int scmc_refocus(const double *u, const double *v, int64_t nv, int32_t dim, const double *l, const double *box_min,
                 const double *box_max, const double *box_stp, double lambda, int32_t as_written, int32_t precision,
                 int32_t device, double *rU);

/* Field samples from a covariance, as examples/samplingFromCovMatrix/
 * samplingFromCovMatrix.m:47-64 does with mvnrnd: C is N x N complex
 * (2*N*N doubles, column-major, index v + nv*l as scmc's C(:,:,l1,l2) blocks
 * joined), Sigma = 0.5 [Re C, -Im C; Im C, Re C], sample t = g_t chol(Sigma)
 * with g_t the 2N standard normals of the Philox normal stream (seed, path t)
 * (scmc_philox_stream tag 1), z_t = s(1:N) + i s(N+1:2N).  Z: 2*N*n_samples
 * doubles.  Cholesky in FP64 on the GPU.  A singular Sigma (a covariance of
 * fewer events than 2N) returns SCMC_ERR_INVALID; mvnrnd's cholcov would
 * fall back to an eigendecomposition there. */
int scmc_sample_cov(const double *C, int64_t N, int64_t n_samples, uint64_t seed, int32_t device, double *Z);

/* The memory-effect view of a covariance (config: 64 x 64 covariance on
 * 8 x 8 angular grids).  C1 (+ C2 when not NULL, e.g. Ms + Mm) is
 * nv x nv x nl x nl complex as scmc_cov writes it, with the views on an
 * nvx x nvy grid and the lights on an nlx x nly grid (flat index x fastest).
 * R(dv, dl) = the mean of C(v1, v2, l1, l2) over all entries with view offset
 * v1 - v2 = dv and light offset l1 - l2 = dl: the diagonal means that
 * examples/memoryEffectMeasurements/memoryEffectMeasurements.m:72-86 takes
 * one pair of directions at a time.  R: complex FP32 (2 floats each),
 * (2nvx-1)(2nvy-1) view offsets fastest, then (2nlx-1)(2nly-1) light
 * offsets; offset (dx, dy) at index (dx + nx - 1) + (2nx - 1)(dy + ny - 1).
 * _device: C1, C2, R in device memory, work on `stream`. */
int scmc_cov_offsets(const double *C1, const double *C2, int32_t nvx, int32_t nvy, int32_t nlx, int32_t nly,
                     float *R, int32_t device);
int scmc_cov_offsets_device(const double *d_C1, const double *d_C2, int32_t nvx, int32_t nvy, int32_t nlx,
                            int32_t nly, float *d_R, int32_t device, void *stream);

/* ---------------------------------------------------------------------------
 * Tuning.  Launch parameters the project's autotuner (mcspeckle_b200.autotune)
 * chooses per (kind, precision, size) by timing candidates on the GPU; no
 * counterpart in the reference.  An entry applies to solves of its kind and
 * precision whose size n lies in [n_lo, n_hi] (n = nv*nl for field and cov,
 * nv0*nv0 for FourierQuad); the last matching entry wins, and a 0 field keeps
 * the built-in choice.  The library reads entries, at its first use, from the
 * file named by SCMC_TUNING_FILE, else from scmc_tuning.txt beside the
 * library; scmc_tuning_load reads another file.  File lines:
 *   kind precision n_lo n_hi path_batch chunk_events stages ksplit group_entries
 * with kind field | cov | fq and precision fp64 | mixed | fp32 | fp16; '#'
 * starts a comment.  The covariance's chunk is capped where its FP32 tensor
 * sums would exceed the tolerance (65536 events FP16, 32768 hi+lo; hi+lo
 * takes 4096 by default, its error growing with the chunk).
 * ------------------------------------------------------------------------- */
enum { SCMC_TUNE_FIELD = 0, SCMC_TUNE_COV = 1, SCMC_TUNE_FQ = 2 };

typedef struct {
    int32_t kind;            /* SCMC_TUNE_* */
    int32_t precision;       /* SCMC_PREC_* */
    int64_t n_lo, n_hi;
    int64_t path_batch;      /* paths walked per batch (built-in: 2^20) */
    int64_t chunk_events;    /* events per tensor-core chunk (built-in: from 1-2 GiB of operands) */
    int32_t stages;          /* CTA-pair pipeline stages, 2 or 3 (3: FP16 covariance only) */
    int32_t ksplit;          /* split-K slices of the tensor-core field (built-in: fill the SMs) */
    int64_t group_entries;   /* FourierQuad entries per plane group (built-in: 2^20) */
} scmc_tuning;

int scmc_tuning_set(const scmc_tuning *t);
int scmc_tuning_clear(void);
int scmc_tuning_load(const char *path);
/* The resolved parameters (built-in defaults filled in) for one solve shape. */
int scmc_tuning_get(int32_t kind, int32_t precision, int64_t n, scmc_tuning *out);

/* Library information and error reporting. */
int scmc_abi_version(void);
const char *scmc_last_error(void);
/* Kernel launches issued by this process since load (all entry points). */
int64_t scmc_launch_count(void);

/* Failure injection for the bounded device waits, for tests; no counterpart
 * in the reference.  While on (process-wide), every tensor-core kernel
 * (covariance, field, FourierQuad plane loop) issues no copy and its
 * consumers wait 1 ms instead of 2 s, so each such launch gives up, flags
 * its error, frees its tensor memory and returns, and the call reports
 * SCMC_ERR_TIMEOUT.  Nothing is in flight when the waits give up, and the
 * context stays usable: switch it off and the next call is correct. */
int scmc_test_wait_fault(int32_t on);

#ifdef __cplusplus
}
#endif

#endif /* SCMC_GPU_H */
