// scmc_capi.cu - host side of libscmc_gpu.so: argument validation, the
// process-lifetime device context, path batching and the C ABI entry points
// declared in include/scmc_gpu.h.
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/scmc_gpu.h"
#include "accum.cuh"
#include "herk_tc.cuh"
#include "field_tc.cuh"
#include "fq.cuh"
#include "onwave.cuh"
#include "postprocess.cuh"

using namespace scmc;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

namespace {

struct ScmcError {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg) { throw ScmcError{code, msg}; }

void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? SCMC_ERR_NOMEM : SCMC_ERR_CUDA;
        fail(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

#define CK(x) cuda_check((x), #x)
#define LAUNCHED() (g_launches.fetch_add(1, std::memory_order_relaxed))

// ---------------------------------------------------------------------------
// stage timing (scmc_profile_*)
// ---------------------------------------------------------------------------
enum Stage { ST_WALK = 0, ST_ROWS = 1, ST_CONTRACT = 2, ST_FINAL = 3 };

struct Profiler {
    std::mutex mu;
    std::atomic<bool> on{false};
    struct Pending {
        cudaEvent_t a, b;
        int stage;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    int64_t launches[4] = {0, 0, 0, 0};
    double ms[4] = {0, 0, 0, 0};
    // Launch intervals relative to `ref` (recorded when profiling is switched
    // on), so that launches overlapping on several streams are counted once
    // in the busy time of their stage.
    cudaEvent_t ref = nullptr;
    std::vector<std::pair<float, float>> iv[4];

    double busy_ms(int stage)
    {
        auto &v = iv[stage];
        std::sort(v.begin(), v.end());
        double t = 0.0, s = 0.0, e = -1.0;
        bool open = false;
        for (auto &x : v) {
            if (!open || x.first > e) {
                if (open) t += e - s;
                s = x.first;
                e = x.second;
                open = true;
            } else if (x.second > e) {
                e = x.second;
            }
        }
        if (open) t += e - s;
        return t;
    }
    int64_t paths = 0, events = 0;
    double flops = 0;

    cudaEvent_t take()
    {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        return e;
    }
    void resolve_locked()
    {
        for (auto &p : pending) {
            CK(cudaEventSynchronize(p.b));
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, p.a, p.b));
            ms[p.stage] += t;
            launches[p.stage] += 1;
            if (ref) {
                float t0 = 0.f, t1 = 0.f;
                CK(cudaEventElapsedTime(&t0, ref, p.a));
                CK(cudaEventElapsedTime(&t1, ref, p.b));
                iv[p.stage].emplace_back(t0, t1);
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
};
Profiler g_prof;

// Brackets the launches made in its scope with CUDA events when enabled.
struct StageScope {
    int stage;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    StageScope(int s, cudaStream_t stream) : stage(s), st(stream)
    {
        if (!g_prof.on.load(std::memory_order_relaxed)) return;
        std::lock_guard<std::mutex> lk(g_prof.mu);
        if (g_prof.pending.size() > 8192) g_prof.resolve_locked();
        a = g_prof.take();
        CK(cudaEventRecord(a, st));
    }
    ~StageScope() noexcept(false)
    {
        if (!a) return;
        std::lock_guard<std::mutex> lk(g_prof.mu);
        cudaEvent_t b = g_prof.take();
        CK(cudaEventRecord(b, st));
        g_prof.pending.push_back({a, b, stage});
    }
};

void prof_count(int64_t paths, int64_t events, double flops)
{
    if (!g_prof.on.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lk(g_prof.mu);
    g_prof.paths += paths;
    g_prof.events += events;
    g_prof.flops += flops;
}

template <typename F>
int guarded(F &&f)
{
    try {
        f();
        return SCMC_OK;
    } catch (const ScmcError &e) {
        g_last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return SCMC_ERR_NOMEM;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return SCMC_ERR_CUDA;
    } catch (...) {
        g_last_error = "unknown error";
        return SCMC_ERR_CUDA;
    }
}

// ---------------------------------------------------------------------------
// tuning table (scmc_tuning_*): launch parameters per (kind, precision, size)
// ---------------------------------------------------------------------------
std::mutex g_tune_mu;
std::vector<scmc_tuning> g_tune;
bool g_tune_loaded = false;

void tuning_parse_file(const char *path, bool must_exist)
{
    std::ifstream f(path);
    if (!f) {
        if (must_exist) fail(SCMC_ERR_INVALID, std::string("cannot read tuning file ") + path);
        return;
    }
    std::vector<scmc_tuning> add;
    std::string line;
    int lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        const size_t h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        std::istringstream is(line);
        std::string kind, prec;
        if (!(is >> kind)) continue;
        scmc_tuning t{};
        long long nlo = 0, nhi = 0, pb = 0, ce = 0, ge = 0;
        int st = 0, ks = 0;
        if (!(is >> prec >> nlo >> nhi >> pb >> ce >> st >> ks >> ge))
            fail(SCMC_ERR_INVALID, std::string("tuning file ") + path + ": bad line " + std::to_string(lineno));
        if (kind == "field") t.kind = SCMC_TUNE_FIELD;
        else if (kind == "cov") t.kind = SCMC_TUNE_COV;
        else if (kind == "fq") t.kind = SCMC_TUNE_FQ;
        else fail(SCMC_ERR_INVALID, std::string("tuning file ") + path + ": unknown kind " + kind);
        if (prec == "fp64") t.precision = SCMC_PREC_FP64;
        else if (prec == "mixed") t.precision = SCMC_PREC_MIXED;
        else if (prec == "fp32") t.precision = SCMC_PREC_FP32;
        else if (prec == "fp16") t.precision = SCMC_PREC_FP16;
        else fail(SCMC_ERR_INVALID, std::string("tuning file ") + path + ": unknown precision " + prec);
        t.n_lo = nlo;
        t.n_hi = nhi;
        t.path_batch = pb;
        t.chunk_events = ce;
        t.stages = st;
        t.ksplit = ks;
        t.group_entries = ge;
        add.push_back(t);
    }
    g_tune.insert(g_tune.end(), add.begin(), add.end());
}

// At the first use: SCMC_TUNING_FILE, else scmc_tuning.txt beside the library.
void tuning_autoload_locked()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    if (const char *env = std::getenv("SCMC_TUNING_FILE")) {
        tuning_parse_file(env, true);
        return;
    }
    Dl_info info;
    if (dladdr(reinterpret_cast<void *>(&tuning_parse_file), &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        const size_t slash = p.rfind('/');
        p = (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/scmc_tuning.txt";
        tuning_parse_file(p.c_str(), false);
    }
}

scmc_tuning tuning_for(int kind, int precision, int64_t n)
{
    scmc_tuning r{};
    r.kind = kind;
    r.precision = precision;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tuning_autoload_locked();
        for (const scmc_tuning &t : g_tune)
            if (t.kind == kind && t.precision == precision && n >= t.n_lo && n <= t.n_hi) {
                r.n_lo = t.n_lo;
                r.n_hi = t.n_hi;
                if (t.path_batch > 0) r.path_batch = t.path_batch;
                if (t.chunk_events > 0) r.chunk_events = t.chunk_events;
                if (t.stages > 0) r.stages = t.stages;
                if (t.ksplit > 0) r.ksplit = t.ksplit;
                if (t.group_entries > 0) r.group_entries = t.group_entries;
            }
    }
    if (r.path_batch <= 0) r.path_batch = (int64_t)1 << 20;
    if (r.stages != 3) r.stages = 2;
    if (r.group_entries <= 0) r.group_entries = (int64_t)1 << 20;
    r.group_entries = std::max<int64_t>(r.group_entries, 4096);
    return r;
}

// ---------------------------------------------------------------------------
// device buffers and the per-device context
// ---------------------------------------------------------------------------
// Scratch that grows on demand.  With a stream set (server slots) the memory
// comes from the stream-ordered pool, so growing or releasing it never
// synchronises the device with other slots' work.
struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    cudaStream_t ast = nullptr;
    bool ordered = false;
    void *ensure(size_t bytes)
    {
        if (bytes <= n) return p;
        release();
        size_t want = bytes + bytes / 8;
        if (ordered) CK(cudaMallocAsync(&p, want, ast));
        else CK(cudaMalloc(&p, want));
        n = want;
        return p;
    }
    void release()
    {
        if (p) {
            if (ordered) CK(cudaFreeAsync(p, ast));
            else CK(cudaFree(p));
        }
        p = nullptr;
        n = 0;
    }
    template <typename T> T *as() { return reinterpret_cast<T *>(p); }
};

// Pinned host staging that grows on demand (copies from it are truly
// asynchronous; a pageable source would make the copy wait for its stream).
struct PinnedBuf {
    void *p = nullptr;
    size_t n = 0;
    void *ensure(size_t bytes)
    {
        if (bytes <= n) return p;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        const size_t want = bytes + bytes / 4;
        CK(cudaMallocHost(&p, want));
        n = want;
        return p;
    }
    ~PinnedBuf()
    {
        if (p) cudaFreeHost(p);
    }
};

struct Ctx {
    int device = -1;
    std::mutex mu;
    PinnedBuf fq_hmeta[2];  // FourierQuad pair-form metadata, per batch parity
    DevBuf counts, mcnt, moff, scan_tmp, ctr, err;
    DevBuf s_x1, s_w1, s_wpx, s_xi, s_nev;
    DevBuf m_x, m_ow, m_wpx, m_xi, m_path, m_plen;
    DevBuf dirs_l, dirs_v, dirs_vs, tab0_amp, tab0_icdf, tab1_amp, tab1_icdf;
    DevBuf acc_s, acc_m, acc_f, rows, rows2, tiles, tc_a, out0, out1, out2, wl, offs, mcap_bounds, fq_err;
    DevBuf fq_gz, fq_zexp, fq_box, fq_tw, fq_twt, fq_rr, fq_counts, fq_offsets, fq_cursor, fq_planes;
    int64_t scap = 0, mcap = 0;
    double multi_per_path = 8.0;  // multiple-scattering events per path seen so far (one-pass capacity)
    size_t tc_chunk_bytes = (size_t)2 << 30;  // operand memory per tensor-core chunk
    // Extra streams and events of the covariance pipeline: the walk and row
    // generation run on `aux` (lowest priority), contractions alternate
    // between `aux3` and `aux2` (highest priority, so that when an SM frees
    // the block scheduler places the contraction before more rows).
    cudaStream_t aux = nullptr, aux2 = nullptr, aux3 = nullptr;
    cudaEvent_t ev[10] = {};

    void destroy_aux()
    {
        if (!aux) return;
        for (auto &e : ev) {
            cudaEventDestroy(e);
            e = nullptr;
        }
        cudaStreamDestroy(aux);
        cudaStreamDestroy(aux2);
        cudaStreamDestroy(aux3);
        aux = aux2 = aux3 = nullptr;
    }
    void make_aux()
    {
        if (aux) return;
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CK(cudaStreamCreateWithPriority(&aux, cudaStreamNonBlocking, least));
        CK(cudaStreamCreateWithPriority(&aux2, cudaStreamNonBlocking, greatest));
        CK(cudaStreamCreateWithPriority(&aux3, cudaStreamNonBlocking, greatest));
        for (auto &e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }

    template <typename F> void each(F &&f)
    {
        DevBuf *all[] = {&counts, &mcnt, &moff, &scan_tmp, &ctr, &err, &s_x1, &s_w1, &s_wpx, &s_xi, &s_nev,
                         &m_x, &m_ow, &m_wpx, &m_xi, &m_path, &m_plen, &dirs_l, &dirs_v, &dirs_vs, &tab0_amp,
                         &tab0_icdf, &tab1_amp, &tab1_icdf, &acc_s, &acc_m, &acc_f, &rows, &tiles, &tc_a, &out0, &wl, &offs,
                         &mcap_bounds, &rows2, &fq_err,
                         &out1, &out2, &fq_gz, &fq_zexp, &fq_box, &fq_tw, &fq_twt, &fq_rr, &fq_counts, &fq_offsets,
                         &fq_cursor, &fq_planes};
        for (DevBuf *b : all) f(*b);
    }
    void set_stream_ordered(cudaStream_t st)
    {
        each([&](DevBuf &b) {
            b.ast = st;
            b.ordered = true;
        });
    }
    size_t held()
    {
        size_t t = 0;
        each([&](DevBuf &b) { t += b.n; });
        return t;
    }
    void release_all()
    {
        each([](DevBuf &b) { b.release(); });
        scap = mcap = 0;
    }
};

std::mutex g_ctx_mu;
std::vector<Ctx *> g_ctx;

Ctx &context(int device)
{
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) fail(SCMC_ERR_NODEVICE, "no CUDA device visible");
    if (device < 0 || device >= n) fail(SCMC_ERR_INVALID, "invalid device ordinal");
    if ((int)g_ctx.size() < n) g_ctx.resize(n, nullptr);
    if (!g_ctx[device]) {
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10) fail(SCMC_ERR_NODEVICE, "an sm_100 (Blackwell) device is required");
        g_ctx[device] = new Ctx();
        g_ctx[device]->device = device;
    }
    return *g_ctx[device];
}

// ---------------------------------------------------------------------------
// validation (messages follow the reference's error() strings)
// ---------------------------------------------------------------------------
void validate_pf(const scmc_phase_function &pf, const char *name)
{
    if (pf.sct_type < 1 || pf.sct_type > 3) fail(SCMC_ERR_INVALID, std::string("invalid sct_type in ") + name);
    if (pf.sct_type == SCMC_SCT_TABULATED && (pf.table_n < 2 || !pf.eval_amp || !pf.sample_icdf))
        fail(SCMC_ERR_INVALID, std::string("tabulated ") + name + " needs evalAmp and sampleIcdf tables");
    if (pf.sct_type == SCMC_SCT_HG && !(std::fabs(pf.g) <= 1.0)) fail(SCMC_ERR_INVALID, "Invalid g input");
    if (pf.table_in_cos != 0 && pf.table_in_cos != 1) fail(SCMC_ERR_INVALID, "table_in_cos must be 0 or 1");
}

void validate(const scmc_mc_args *a)
{
    if (!a) fail(SCMC_ERR_INVALID, "null arguments");
    if (a->dim != 2 && a->dim != 3) fail(SCMC_ERR_INVALID, "Invalid box size");
    if (a->nl < 1 || !a->l) fail(SCMC_ERR_INVALID, "Invalid light source input");
    if (a->nv < 1 || !a->v) fail(SCMC_ERR_INVALID, "Invalid view source input");
    if (a->max_itr < 0) fail(SCMC_ERR_INVALID, "Invalid photons number");
    if (!(a->sigt > 0) || !std::isfinite(a->sigt)) fail(SCMC_ERR_INVALID, "sigt must be positive");
    if (!(a->lambda > 0)) fail(SCMC_ERR_INVALID, "lambda must be positive");
    if (a->smp_flg != 1 && a->smp_flg != 2) fail(SCMC_ERR_INVALID, "smpFlg must be 1 or 2");
    if (a->precision < 0 || a->precision > 3) fail(SCMC_ERR_INVALID, "invalid precision mode");
    for (int k = 0; k < a->dim; ++k)
        if (!(a->box_max[k] >= a->box_min[k])) fail(SCMC_ERR_INVALID, "Invalid box size");
    validate_pf(a->ampfunc, "ampfunc");
    if (a->has_ampfunc0) validate_pf(a->ampfunc0, "ampfunc0");
    if (a->dim != 3 && (a->ampfunc.table_in_cos || (a->has_ampfunc0 && a->ampfunc0.table_in_cos)))
        fail(SCMC_ERR_INVALID, "tables on cos(theta) bins are 3-D only");
}

// ---------------------------------------------------------------------------
// argument preparation
// ---------------------------------------------------------------------------
struct Prepared {
    WalkParams W;
    NeeParams Q;
    double volume;
};

PhaseFn upload_pf(const scmc_phase_function &pf, DevBuf &amp, DevBuf &icdf, cudaStream_t st)
{
    PhaseFn d{};
    d.sct_type = pf.sct_type;
    d.g = pf.g;
    d.table_n = pf.table_n;
    d.cos_bins = pf.table_in_cos;
    if (pf.sct_type == SCMC_SCT_TABULATED) {
        size_t n = (size_t)pf.table_n;
        amp.ensure(n * sizeof(double2));
        icdf.ensure(n * sizeof(double));
        CK(cudaMemcpyAsync(amp.p, pf.eval_amp, n * sizeof(double2), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(icdf.p, pf.sample_icdf, n * sizeof(double), cudaMemcpyHostToDevice, st));
        d.eval_amp = amp.as<double2>();
        d.sample_icdf = icdf.as<double>();
    }
    return d;
}

// The host-side parameters of a solve (MCfield.m:71-110, MCcov.m:78-110):
// everything except the device copies of the tables and directions, which
// the caller places (prepare: allocated scratch; scmc_field_noalloc: the fixed
// array) and then points W.pf / W.pf0 / Q.{l, v, vs, pf, pf0} at.
Prepared host_params(const scmc_mc_args *a, int want_phase)
{
    Prepared P{};
    const int dim = a->dim;
    WalkParams &W = P.W;
    W.dim = dim;
    W.smp_flg = a->smp_flg;
    W.has_pf0 = a->has_ampfunc0;
    W.want_phase = want_phase;
    W.sigt = a->sigt;
    W.albedo = a->albedo;
    P.volume = 1.0;
    for (int k = 0; k < 3; ++k) {
        W.box_min[k] = k < dim ? a->box_min[k] : 0.0;
        W.box_max[k] = k < dim ? a->box_max[k] : 0.0;
        W.box_w[k] = W.box_max[k] - W.box_min[k];
        if (k < dim) P.volume *= W.box_w[k];
    }
    // MCfield.m:77-82: unmeanl = mean(l,2) (or lmean0), meanl = unmeanl/norm
    double nrm = 0.0;
    for (int k = 0; k < 3; ++k) {
        double s = 0.0;
        if (k < dim)
            for (int64_t j = 0; j < a->nl; ++j) s += a->l[dim * j + k];
        W.unmeanl[k] = k < dim ? (a->has_lmean0 ? a->lmean0[k] : s / (double)a->nl) : 0.0;
        nrm += W.unmeanl[k] * W.unmeanl[k];
    }
    nrm = std::sqrt(nrm);
    for (int k = 0; k < 3; ++k) W.meanl[k] = W.unmeanl[k] / nrm;
    if (a->smp_flg == 2 && W.unmeanl[dim - 1] == 0.0)
        fail(SCMC_ERR_INVALID, "exponential first-scatter sampling needs a mean light direction with a non-zero last component");
    W.key0 = (uint32_t)a->seed;
    W.key1 = (uint32_t)(a->seed >> 32);
    W.max_events = a->max_events_per_path;
    // the reduced-precision modes walk once and take the records in any order;
    // FP64 (parity) keeps the two passes and path order
    W.any_order = a->precision != SCMC_PREC_FP64;
    W.pf.sct_type = a->ampfunc.sct_type;
    W.pf.g = a->ampfunc.g;
    W.pf.table_n = a->ampfunc.table_n;
    W.pf.cos_bins = a->ampfunc.table_in_cos;
    W.pf0 = W.pf;
    if (a->has_ampfunc0) {
        W.pf0.sct_type = a->ampfunc0.sct_type;
        W.pf0.g = a->ampfunc0.g;
        W.pf0.table_n = a->ampfunc0.table_n;
        W.pf0.cos_bins = a->ampfunc0.table_in_cos;
    }

    NeeParams &Q = P.Q;
    Q.nv = (int)a->nv;
    Q.nl = (int)a->nl;
    Q.is_ff_l = a->is_ff_l;
    Q.is_ff_v = a->is_ff_v;
    Q.cbs = a->do_cbs;
    Q.sigt_half = a->sigt / 2.0;
    Q.kw = SCMC_PI * 2.0 / a->lambda;
    Q.lambda = a->lambda;
    for (int k = 0; k < 3; ++k) {
        Q.box_min[k] = W.box_min[k];
        Q.box_max[k] = W.box_max[k];
        Q.meanl[k] = W.meanl[k];
    }
    nee_set_fbox(Q);
    Q.has_pf0 = a->has_ampfunc0;
    return P;
}

// Points the phase functions of P at their device tables (amp0/icdf0 for
// ampfunc, amp1/icdf1 for ampfunc0; null where a function is not tabulated).
void set_tables(Prepared &P, const scmc_mc_args *a, const double2 *amp0, const double *icdf0, const double2 *amp1,
                const double *icdf1)
{
    if (a->ampfunc.sct_type == SCMC_SCT_TABULATED) {
        P.W.pf.eval_amp = amp0;
        P.W.pf.sample_icdf = icdf0;
    }
    if (a->has_ampfunc0) {
        if (a->ampfunc0.sct_type == SCMC_SCT_TABULATED) {
            P.W.pf0.eval_amp = amp1;
            P.W.pf0.sample_icdf = icdf1;
        }
    } else {
        P.W.pf0 = P.W.pf;
    }
    P.Q.pf = P.W.pf;
    P.Q.pf0 = P.W.pf0;
}

Prepared prepare(Ctx &c, const scmc_mc_args *a, int want_phase, cudaStream_t st)
{
    Prepared P = host_params(a, want_phase);
    const int dim = a->dim;
    const PhaseFn d0 = upload_pf(a->ampfunc, c.tab0_amp, c.tab0_icdf, st);
    const PhaseFn d1 = a->has_ampfunc0 ? upload_pf(a->ampfunc0, c.tab1_amp, c.tab1_icdf, st) : PhaseFn{};
    set_tables(P, a, d0.eval_amp, d0.sample_icdf, d1.eval_amp, d1.sample_icdf);

    // directions as [n][3]
    std::vector<double> hl(3 * a->nl, 0.0), hv(3 * a->nv, 0.0), hvs(3 * a->nv, 0.0);
    double ff_sign = a->is_ff_v ? -1.0 : 1.0;  // MCfield.m:106
    for (int64_t j = 0; j < a->nl; ++j)
        for (int k = 0; k < dim; ++k) hl[3 * j + k] = a->l[dim * j + k];
    for (int64_t i = 0; i < a->nv; ++i)
        for (int k = 0; k < dim; ++k) {
            hv[3 * i + k] = a->v[dim * i + k];
            hvs[3 * i + k] = ff_sign * a->v[dim * i + k];
        }
    c.dirs_l.ensure(hl.size() * 8);
    c.dirs_v.ensure(hv.size() * 8);
    c.dirs_vs.ensure(hvs.size() * 8);
    CK(cudaMemcpyAsync(c.dirs_l.p, hl.data(), hl.size() * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c.dirs_v.p, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c.dirs_vs.p, hvs.data(), hvs.size() * 8, cudaMemcpyHostToDevice, st));
    P.Q.l = c.dirs_l.as<double>();
    P.Q.v = c.dirs_v.as<double>();
    P.Q.vs = c.dirs_vs.as<double>();
    // the host copies above must complete before the vectors go out of scope
    CK(cudaStreamSynchronize(st));
    return P;
}

// ---------------------------------------------------------------------------
// the walk of one batch of paths -> records
// ---------------------------------------------------------------------------
__global__ void count_to_multi_kernel(const int32_t *__restrict__ counts, int64_t n, int64_t *__restrict__ m)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        m[p] = (int64_t)counts[p] - 1;
}

int sm_count(int device)
{
    static int cached[64] = {0};
    if (device < 64 && cached[device]) return cached[device];
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    if (device < 64) cached[device] = n;
    return n;
}

struct Batch {
    SingleRec S;
    MultiRec M;
    int64_t n_paths = 0, n_multi = 0;
};

void ensure_single_records(Ctx &c, int64_t n_paths)
{
    if (c.scap >= n_paths) return;
    const int64_t cap = n_paths;
    c.s_x1.ensure(3 * cap * 8);
    c.s_w1.ensure(3 * cap * 8);
    c.s_wpx.ensure(cap * 8);
    c.s_xi.ensure(cap * 8);
    c.s_nev.ensure(cap * 4);
    c.scap = cap;
}

void ensure_multi_records(Ctx &c, int64_t n_multi)
{
    if (c.mcap >= std::max<int64_t>(n_multi, 1)) return;
    const int64_t cap = std::max<int64_t>(n_multi + n_multi / 4, 1024);
    c.m_x.ensure(3 * cap * 8);
    c.m_ow.ensure(3 * cap * 8);
    c.m_wpx.ensure(cap * 8);
    c.m_xi.ensure(cap * 8);
    c.m_path.ensure(cap * 4);
    c.m_plen.ensure(cap * 4);
    c.mcap = cap;
}

void batch_views(Ctx &c, int64_t n_paths, int64_t n_multi, Batch &B)
{
    B.S = SingleRec{c.s_x1.as<double>(), c.s_w1.as<double>(), c.s_wpx.as<double>(), c.s_xi.as<double>(),
                    c.s_nev.as<int32_t>()};
    B.M = MultiRec{c.m_x.as<double>(), c.m_ow.as<double>(), c.m_wpx.as<double>(), c.m_xi.as<double>(),
                   c.m_path.as<int32_t>(), c.m_plen.as<int32_t>()};
    B.n_paths = n_paths;
    B.n_multi = n_multi;
}

// One walk pass writing records in any order (reduced-precision modes): the
// multiple-scattering capacity comes from the events per path of earlier
// batches; a batch with more events than that is walked again with room for
// all of them.
template <int DIM>
void walk_batch_onepass(Ctx &c, WalkParams W, int64_t n_paths, cudaStream_t st, Batch &B)
{
    const int sms = sm_count(c.device);
    const int threads = 128;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_paths + threads - 1) / threads, (int64_t)sms * 8));
    W.n_paths = n_paths;
    ensure_single_records(c, n_paths);
    ensure_multi_records(c, (int64_t)((double)n_paths * c.multi_per_path * 1.15) + 1024);
    c.ctr.ensure(2 * sizeof(unsigned long long));
    c.err.ensure(sizeof(int));
    unsigned long long *ctr = c.ctr.as<unsigned long long>();
    for (int attempt = 0;; ++attempt) {
        batch_views(c, n_paths, 0, B);
        CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), st));
        CK(cudaMemsetAsync(c.err.p, 0, sizeof(int), st));
        {
            StageScope sc(ST_WALK, st);
            walk_onepass_kernel<DIM><<<grid, threads, 0, st>>>(W, B.S, c.scap, B.M, c.mcap, ctr, c.err.as<int>());
            CK(cudaGetLastError());
            LAUNCHED();
        }
        unsigned long long n_multi = 0;
        int herr = 0;
        CK(cudaMemcpyAsync(&n_multi, ctr + 1, sizeof(n_multi), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&herr, c.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr) fail(SCMC_ERR_LIMIT, "a path exceeded max_events_per_path");
        const double ratio = (double)n_multi / (double)std::max<int64_t>(n_paths, 1);
        c.multi_per_path = std::max(ratio, 0.5 * c.multi_per_path);
        if ((int64_t)n_multi <= c.mcap) {
            batch_views(c, n_paths, (int64_t)n_multi, B);
            prof_count(n_paths, n_paths + (int64_t)n_multi, 0.0);
            return;
        }
        if (attempt > 0) fail(SCMC_ERR_CUDA, "one-pass walk: record count changed between two walks of a batch");
        ensure_multi_records(c, (int64_t)n_multi);
    }
}

template <int DIM>
void walk_batch_dim(Ctx &c, WalkParams W, int64_t n_paths, cudaStream_t st, Batch &B)
{
    if (W.any_order) {
        walk_batch_onepass<DIM>(c, W, n_paths, st, B);
        return;
    }
    const int sms = sm_count(c.device);
    const int threads = 128;
    int grid = (int)std::min<int64_t>((n_paths + threads - 1) / threads, (int64_t)sms * 8);
    if (grid < 1) grid = 1;
    W.n_paths = n_paths;
    c.counts.ensure(n_paths * sizeof(int32_t));
    c.mcnt.ensure(n_paths * sizeof(int64_t));
    c.moff.ensure((n_paths + 1) * sizeof(int64_t));
    c.ctr.ensure(2 * sizeof(unsigned long long));
    c.err.ensure(sizeof(int));
    unsigned long long *ctr = c.ctr.as<unsigned long long>();
    CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), st));
    CK(cudaMemsetAsync(c.err.p, 0, sizeof(int), st));
    {
        StageScope sc(ST_WALK, st);
        walk_count_kernel<DIM><<<grid, threads, 0, st>>>(W, c.counts.as<int32_t>(), ctr, c.err.as<int>());
        CK(cudaGetLastError());
        LAUNCHED();
    }
    count_to_multi_kernel<<<std::max(1, std::min(sms * 4, (int)((n_paths + 255) / 256))), 256, 0, st>>>(
        c.counts.as<int32_t>(), n_paths, c.mcnt.as<int64_t>());
    CK(cudaGetLastError());
    LAUNCHED();
    size_t tmp = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, c.mcnt.as<int64_t>(), c.moff.as<int64_t>(), n_paths, st));
    c.scan_tmp.ensure(tmp);
    CK(cub::DeviceScan::ExclusiveSum(c.scan_tmp.p, tmp, c.mcnt.as<int64_t>(), c.moff.as<int64_t>(), n_paths, st));
    LAUNCHED();
    int64_t last[2];
    int herr = 0;
    CK(cudaMemcpyAsync(&last[0], c.moff.as<int64_t>() + n_paths - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last[1], c.mcnt.as<int64_t>() + n_paths - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&herr, c.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr) fail(SCMC_ERR_LIMIT, "a path exceeded max_events_per_path");
    const int64_t n_multi = last[0] + last[1];

    // record storage
    ensure_single_records(c, n_paths);
    ensure_multi_records(c, n_multi);
    batch_views(c, n_paths, n_multi, B);
    CK(cudaMemsetAsync(ctr + 1, 0, sizeof(unsigned long long), st));
    {
        StageScope sc(ST_WALK, st);
        walk_record_kernel<DIM><<<grid, threads, 0, st>>>(W, c.moff.as<int64_t>(), B.S, c.scap, B.M, c.mcap, ctr + 1);
        CK(cudaGetLastError());
        LAUNCHED();
    }
    prof_count(n_paths, n_paths + n_multi, 0.0);
}

void walk_batch(Ctx &c, const WalkParams &W, int64_t n_paths, cudaStream_t st, Batch &B)
{
    if (W.dim == 3) walk_batch_dim<3>(c, W, n_paths, st, B);
    else walk_batch_dim<2>(c, W, n_paths, st, B);
}

int64_t path_batch_size(int64_t remaining, int64_t limit = (int64_t)1 << 20)
{
    return std::min<int64_t>(remaining, std::max<int64_t>(limit, 1));
}

// ---------------------------------------------------------------------------
// field
// ---------------------------------------------------------------------------
template <int DIM, int POL, bool SINGLE, typename AccT>
void launch_field_accum(Ctx &c, const Prepared &P, const Batch &B, AccT *U, int64_t n_ev, cudaStream_t st,
                        int mean_mode = 0)
{
    if (n_ev <= 0) return;
    const int nv = P.Q.nv, nl = P.Q.nl;
    int tv = std::min(nv, 32), tl = std::min(nl, 32);
    while (tv * tl > kFieldMaxTile) tl /= 2;
    const int n_vtiles = (nv + tv - 1) / tv, n_ltiles = (nl + tl - 1) / tl;
    const int tiles = n_vtiles * n_ltiles;
    const int sms = sm_count(c.device);
    int64_t target = (int64_t)sms * 6;
    int64_t ranges = std::max<int64_t>(1, target / tiles);
    int64_t per = (n_ev + ranges - 1) / ranges;
    per = std::max<int64_t>(per, kFieldEB * 4);
    ranges = (n_ev + per - 1) / per;
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    size_t smem = sizeof(C) * (2 * kFieldEB * (tv + tl) + kFieldEB) + sizeof(EventView) * kFieldEB + 16;
    auto kern = field_accum_kernel<DIM, POL, SINGLE, AccT>;
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid(tiles, (unsigned)ranges);
    StageScope sc(ST_ROWS, st);
    kern<<<grid, kFieldThreads, smem, st>>>(P.Q, B.S, c.scap, B.M, c.mcap, n_ev, tv, tl, n_vtiles, per, U,
                                            mean_mode ? 0 : P.W.want_phase, mean_mode);
    CK(cudaGetLastError());
    LAUNCHED();
}

// The tensor-core field path pays off once the output fills a good part of a
// 128 x 256 tile; smaller fields stay on the CUDA-core accumulation.
bool use_field_tc(const scmc_mc_args *a)
{
    return (a->precision == SCMC_PREC_MIXED || a->precision == SCMC_PREC_FP16) && a->nv >= 64 && a->nl >= 32;
}

template <int DIM>
void field_run_tc(Ctx &c, const scmc_mc_args *a, const Prepared &P, double2 *d_u, cudaStream_t st)
{
    const int nv = (int)a->nv, nl = (int)a->nl;
    const bool split = a->precision == SCMC_PREC_MIXED;
    const int terms_m = a->do_cbs ? 2 : 1;
    const scmc_tuning T = tuning_for(SCMC_TUNE_FIELD, a->precision, (int64_t)nv * nl);
    const FieldTcPlan plan = field_tc_plan(nv, nl, terms_m, split, sm_count(c.device), c.tc_chunk_bytes, T.ksplit);
    const bool ffff = a->is_ff_l && a->is_ff_v;
    const size_t slice = (size_t)2 * nv * nl;
    const size_t d_bytes = (size_t)plan.ksplit * slice * sizeof(double);
    double *Ds = reinterpret_cast<double *>(c.acc_s.ensure(ffff ? d_bytes : slice * sizeof(double)));
    double *Dm = reinterpret_cast<double *>(c.acc_m.ensure(d_bytes));
    CK(cudaMemsetAsync(Ds, 0, ffff ? d_bytes : slice * sizeof(double), st));
    CK(cudaMemsetAsync(Dm, 0, d_bytes, st));
    FieldTcOps ops = field_tc_ops(plan, c.tc_a.ensure(field_tc_bytes(plan)), st);
    const size_t smem = field_tc_rows_smem();
    const int64_t chunk = plan.events_per_chunk;
    const int phase = P.W.want_phase;
    WalkParams W = P.W;
    for (int64_t done = 0; done < a->max_itr;) {
        int64_t nb = path_batch_size(a->max_itr - done, T.path_batch);
        W.path_base = a->path_offset + (uint64_t)done;
        Batch B;
        walk_batch(c, W, nb, st, B);
        if (!ffff) launch_field_accum<DIM, PMIX, true, double>(c, P, B, Ds, B.n_paths, st);
        for (int pass = ffff ? 0 : 1; pass < 2; ++pass) {
            const bool single = pass == 0;
            const int terms = single ? 1 : terms_m;
            const int64_t n_ev = single ? B.n_paths : B.n_multi;
            double *D = single ? Ds : Dm;
            for (int64_t e0 = 0; e0 < n_ev; e0 += chunk) {
                const int64_t n = std::min(chunk, n_ev - e0);
                const unsigned grid = (unsigned)((n + 31) / 32);
                {
                    StageScope sc(ST_ROWS, st);
#define SCMC_FT_ROWS(S_, P_)                                                                                      \
    do {                                                                                                          \
        auto k_ = field_tc_rows_kernel<DIM, S_, P_>;                                                              \
        if (smem > 48 * 1024) CK(cudaFuncSetAttribute(k_, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        k_<<<grid, 256, smem, st>>>(P.Q, B.S, c.scap, B.M, c.mcap, e0, n, terms, plan.K, ops.ahi, ops.alo, ops.b,  \
                                    phase);                                                                       \
    } while (0)
                    if (single && split) SCMC_FT_ROWS(true, true);
                    else if (single) SCMC_FT_ROWS(true, false);
                    else if (split) SCMC_FT_ROWS(false, true);
                    else SCMC_FT_ROWS(false, false);
#undef SCMC_FT_ROWS
                    CK(cudaGetLastError());
                    LAUNCHED();
                }
                {
                    StageScope sc(ST_CONTRACT, st);
                    const int num_kb = (int)((2 * terms * n + TC_BK - 1) / TC_BK);
                    if (split)
                        tc_gemm_launch<true>(ops.m_ahi, ops.m_alo, ops.m_b, ops.tiles, ops.n_tiles, num_kb,
                                             plan.ksplit, 2 * nv, nl, D, ops.err, st);
                    else
                        tc_gemm_launch<false>(ops.m_ahi, ops.m_alo, ops.m_b, ops.tiles, ops.n_tiles, num_kb,
                                              plan.ksplit, 2 * nv, nl, D, ops.err, st);
                    CK(cudaGetLastError());
                    LAUNCHED();
                }
                prof_count(0, 0, 8.0 * nv * nl * terms * (double)n);
            }
        }
        done += nb;
    }
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, ops.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr) fail(SCMC_ERR_TIMEOUT, "tensor-core contraction: a bounded wait gave up");
    const double m = (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
    const double norm = m > 0 ? std::sqrt(1.0 / m * P.volume * a->sigt) : 0.0;  // MCfield.m:253-254
    const int64_t n = (int64_t)nv * nl;
    StageScope sc(ST_FINAL, st);
    field_tc_finalize_kernel<DIM><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 2048)), 256, 0,
                                    st>>>(P.Q, Ds, ffff ? plan.ksplit : 0, Dm, plan.ksplit, norm, d_u);
    CK(cudaGetLastError());
    LAUNCHED();
}

template <int DIM, int POL, typename AccT>
void field_run(Ctx &c, const scmc_mc_args *a, const Prepared &P, double2 *d_u, cudaStream_t st)
{
    if (POL == PMIX && use_field_tc(a)) {
        field_run_tc<DIM>(c, a, P, d_u, st);
        return;
    }
    const int64_t n = a->nv * a->nl;
    const scmc_tuning T = tuning_for(SCMC_TUNE_FIELD, a->precision, n);
    AccT *Us = reinterpret_cast<AccT *>(c.acc_s.ensure(2 * n * sizeof(AccT)));
    AccT *Um = reinterpret_cast<AccT *>(c.acc_m.ensure(2 * n * sizeof(AccT)));
    CK(cudaMemsetAsync(Us, 0, 2 * n * sizeof(AccT), st));
    CK(cudaMemsetAsync(Um, 0, 2 * n * sizeof(AccT), st));
    WalkParams W = P.W;
    for (int64_t done = 0; done < a->max_itr;) {
        int64_t nb = path_batch_size(a->max_itr - done, T.path_batch);
        W.path_base = a->path_offset + (uint64_t)done;
        Batch B;
        walk_batch(c, W, nb, st, B);
        launch_field_accum<DIM, POL, true, AccT>(c, P, B, Us, B.n_paths, st);
        launch_field_accum<DIM, POL, false, AccT>(c, P, B, Um, B.n_multi, st);
        done += nb;
    }
    double m = (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
    double norm = m > 0 ? std::sqrt(1.0 / m * P.volume * a->sigt) : 0.0;  // MCfield.m:253-254
    int grid = (int)std::min<int64_t>((n + 255) / 256, 1024);
    StageScope sc(ST_FINAL, st);
    field_finalize_kernel<DIM, AccT><<<std::max(grid, 1), 256, 0, st>>>(P.Q, Us, Um, norm, d_u);
    CK(cudaGetLastError());
    LAUNCHED();
}

void field_device_locked(Ctx &c, const scmc_mc_args *a, double *d_u, cudaStream_t st)
{
    CK(cudaSetDevice(a->device));
    Prepared P = prepare(c, a, 1, st);
    double2 *u = reinterpret_cast<double2 *>(d_u);
    if (a->dim == 3) {
        if (a->precision == SCMC_PREC_FP64) field_run<3, P64, double>(c, a, P, u, st);
        else if (a->precision == SCMC_PREC_MIXED || a->precision == SCMC_PREC_FP16) field_run<3, PMIX, double>(c, a, P, u, st);
        else field_run<3, P32, float>(c, a, P, u, st);
    } else {
        if (a->precision == SCMC_PREC_FP64) field_run<2, P64, double>(c, a, P, u, st);
        else if (a->precision == SCMC_PREC_MIXED || a->precision == SCMC_PREC_FP16) field_run<2, PMIX, double>(c, a, P, u, st);
        else field_run<2, P32, float>(c, a, P, u, st);
    }
}

// ---------------------------------------------------------------------------
// field on a wave (MCfieldOnWave.m): lights combined with weights Wl
// ---------------------------------------------------------------------------
template <int DIM, int POL>
void onwave_run(Ctx &c, const scmc_mc_args *a, const Prepared &P, const double2 *d_wl, double2 *d_u,
                cudaStream_t st)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    const int nv = (int)a->nv, nl = (int)a->nl;
    double2 *U = reinterpret_cast<double2 *>(c.acc_f.ensure(nv * sizeof(double2)));
    CK(cudaMemsetAsync(U, 0, nv * sizeof(double2), st));
    const int nvc = std::min(nv, kOwMaxViews);
    const int nchunks = (nv + nvc - 1) / nvc;
    const size_t smem = onwave_smem(nvc, nl, sizeof(C));
    if (smem > 227 * 1024) fail(SCMC_ERR_INVALID, "too many lights for the field on a wave");
    auto ks = onwave_accum_kernel<DIM, POL, true>;
    auto km = onwave_accum_kernel<DIM, POL, false>;
    if (smem > 48 * 1024) {
        CK(cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CK(cudaFuncSetAttribute(km, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    const int sms = sm_count(c.device);
    const scmc_tuning T = tuning_for(SCMC_TUNE_FIELD, a->precision, (int64_t)nv * nl);
    WalkParams W = P.W;
    for (int64_t done = 0; done < a->max_itr;) {
        int64_t nb = path_batch_size(a->max_itr - done, T.path_batch);
        W.path_base = a->path_offset + (uint64_t)done;
        Batch B;
        walk_batch(c, W, nb, st, B);
        for (int pass = 0; pass < 2; ++pass) {
            const int64_t n_ev = pass == 0 ? B.n_paths : B.n_multi;
            if (n_ev <= 0) continue;
            const int64_t target = std::max<int64_t>(1, (int64_t)sms * 4 / nchunks);
            const int64_t per = std::max<int64_t>(kOwWarps * 4, (n_ev + target - 1) / target);
            dim3 grid((unsigned)((n_ev + per - 1) / per), (unsigned)nchunks);
            StageScope sc(ST_ROWS, st);
            if (pass == 0) ks<<<grid, kOwWarps * 32, smem, st>>>(P.Q, B.S, c.scap, B.M, c.mcap, n_ev, per, nvc, d_wl, U);
            else km<<<grid, kOwWarps * 32, smem, st>>>(P.Q, B.S, c.scap, B.M, c.mcap, n_ev, per, nvc, d_wl, U);
            CK(cudaGetLastError());
            LAUNCHED();
        }
        done += nb;
    }
    const double m = (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
    const double norm = m > 0 ? std::sqrt(1.0 / m * P.volume * a->sigt) : 0.0;  // MCfieldOnWave.m:265-266
    StageScope fin(ST_FINAL, st);
    onwave_finalize_kernel<<<std::max(1, std::min(1024, (nv + 255) / 256)), 256, 0, st>>>(U, nv, norm, d_u);
    CK(cudaGetLastError());
    LAUNCHED();
}

void onwave_device_locked(Ctx &c, const scmc_mc_args *a, const double *Wl, double *d_u, cudaStream_t st)
{
    CK(cudaSetDevice(a->device));
    if (!Wl) fail(SCMC_ERR_INVALID, "null light weights");
    Prepared P = prepare(c, a, 1, st);
    double2 *dw = reinterpret_cast<double2 *>(c.wl.ensure(a->nl * sizeof(double2)));
    CK(cudaMemcpyAsync(dw, Wl, a->nl * sizeof(double2), cudaMemcpyHostToDevice, st));
    double2 *u = reinterpret_cast<double2 *>(d_u);
    if (a->dim == 3) {
        if (a->precision == SCMC_PREC_FP64) onwave_run<3, P64>(c, a, P, dw, u, st);
        else if (a->precision == SCMC_PREC_FP32) onwave_run<3, P32>(c, a, P, dw, u, st);
        else onwave_run<3, PMIX>(c, a, P, dw, u, st);
    } else {
        if (a->precision == SCMC_PREC_FP64) onwave_run<2, P64>(c, a, P, dw, u, st);
        else if (a->precision == SCMC_PREC_FP32) onwave_run<2, P32>(c, a, P, dw, u, st);
        else onwave_run<2, PMIX>(c, a, P, dw, u, st);
    }
}

// ---------------------------------------------------------------------------
// covariance
// ---------------------------------------------------------------------------
std::vector<int2> upper_tiles(int N, int tile)
{
    int nt = (N + tile - 1) / tile;
    std::vector<int2> t;
    for (int i = 0; i < nt; ++i)
        for (int j = i; j < nt; ++j) t.push_back(make_int2(i, j));
    return t;
}

template <int DIM, int POL, bool SINGLE>
void cov_rows(Ctx &c, const Prepared &P, const Batch &B, int64_t e0, int64_t n, void *T, cudaStream_t st)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    const int nv = P.Q.nv, nl = P.Q.nl;
    int eb = 4;
    size_t per_ev = sizeof(C) * 2 * (nv + nl) + sizeof(double) + sizeof(EventView);
    while (eb > 1 && per_ev * eb > 96 * 1024) eb /= 2;
    size_t smem = per_ev * eb + 64;
    auto kern = cov_rows_kernel<DIM, POL, SINGLE>;
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int grid = (int)((n + eb - 1) / eb);
    StageScope sc(ST_ROWS, st);
    kern<<<grid, 256, smem, st>>>(P.Q, B.S, c.scap, B.M, c.mcap, e0, n, eb, reinterpret_cast<C *>(T));
    CK(cudaGetLastError());
    LAUNCHED();
}

template <typename R, typename A>
void herk_cc(Ctx &c, const void *T, int64_t n, int N, void *Cacc, cudaStream_t st)
{
    constexpr int RPT = std::is_same<R, double>::value ? 4 : 8;
    constexpr int BK = std::is_same<R, double>::value ? 8 : 16;
    std::vector<int2> tl = upper_tiles(N, 16 * RPT);
    c.tiles.ensure(tl.size() * sizeof(int2));
    CK(cudaMemcpyAsync(c.tiles.p, tl.data(), tl.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    {
        StageScope sc(ST_CONTRACT, st);
        herk_cc_kernel<R, A, RPT, BK><<<(unsigned)tl.size(), 256, 0, st>>>(
            reinterpret_cast<const typename cplx_t<R>::type *>(T), n, N, c.tiles.as<int2>(),
            reinterpret_cast<typename cplx_t<A>::type *>(Cacc));
        CK(cudaGetLastError());
        LAUNCHED();
    }
    prof_count(0, 0, 4.0 * (double)N * (double)(N + 1) * (double)n);
    CK(cudaStreamSynchronize(st));  // tile list is a stack vector
}

template <int DIM, int POL>
void cov_run_cc(Ctx &c, const scmc_mc_args *a, const Prepared &P, double2 *d_Ms, double2 *d_Mm, cudaStream_t st,
                double *mean1_acc = nullptr)
{
    using R = typename std::conditional<POL == P64, double, float>::type;
    using A = R;  // plain FP32 keeps FP32 accumulators; FP64 mode keeps FP64
    using C = typename cplx_t<R>::type;
    const int N = (int)(a->nv * a->nl);
    const size_t acc_bytes = (size_t)N * N * 2 * sizeof(A);
    void *Cs = c.acc_s.ensure(acc_bytes);
    void *Cm = c.acc_m.ensure(acc_bytes);
    CK(cudaMemsetAsync(Cs, 0, acc_bytes, st));
    CK(cudaMemsetAsync(Cm, 0, acc_bytes, st));
    int64_t chunk = std::max<int64_t>(64, std::min<int64_t>(8192, ((int64_t)256 << 20) / ((int64_t)N * sizeof(C))));
    void *T = c.rows.ensure((size_t)chunk * N * sizeof(C));
    const scmc_tuning tune = tuning_for(SCMC_TUNE_COV, a->precision, N);
    WalkParams W = P.W;
    for (int64_t done = 0; done < a->max_itr;) {
        int64_t nb = path_batch_size(a->max_itr - done, tune.path_batch);
        W.path_base = a->path_offset + (uint64_t)done;
        Batch B;
        walk_batch(c, W, nb, st, B);
        if (mean1_acc) launch_field_accum<DIM, POL, true, double>(c, P, B, mean1_acc, B.n_paths, st, 1);
        for (int64_t e0 = 0; e0 < B.n_paths; e0 += chunk) {
            int64_t n = std::min(chunk, B.n_paths - e0);
            cov_rows<DIM, POL, true>(c, P, B, e0, n, T, st);
            herk_cc<R, A>(c, T, n, N, Cs, st);
        }
        for (int64_t e0 = 0; e0 < B.n_multi; e0 += chunk) {
            int64_t n = std::min(chunk, B.n_multi - e0);
            cov_rows<DIM, POL, false>(c, P, B, e0, n, T, st);
            herk_cc<R, A>(c, T, n, N, Cm, st);
        }
        done += nb;
    }
    double m = (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
    double sc = m > 0 ? 1.0 / m * P.volume * a->sigt : 0.0;  // MCcov.m:293-299
    double scm = a->do_cbs ? sc / 2.0 : sc;
    int64_t total = (int64_t)N * N;
    int grid = (int)std::min<int64_t>((total + 255) / 256, 4096);
    StageScope fin(ST_FINAL, st);
    if (d_Ms) {
        cov_finalize_kernel<A><<<grid, 256, 0, st>>>(reinterpret_cast<const A *>(Cs), nullptr, 0, (int)a->nv, (int)a->nl, sc, d_Ms);
        CK(cudaGetLastError());
        LAUNCHED();
    }
    if (d_Mm) {
        cov_finalize_kernel<A><<<grid, 256, 0, st>>>(reinterpret_cast<const A *>(Cm), nullptr, 0, (int)a->nv, (int)a->nl, scm, d_Mm);
        CK(cudaGetLastError());
        LAUNCHED();
    }
}

template <int DIM>
void cov_run_tc(Ctx &c, const scmc_mc_args *a, const Prepared &P, double2 *d_Ms, double2 *d_Mm, cudaStream_t st,
                double *mean1_acc = nullptr)
{
    // Three streams: the walk and the row generation on `rs`, contractions of
    // even chunks on `st` and of odd chunks on `cs1`, each into its own FP64
    // accumulator.  Rows of later chunks overlap the contraction in flight,
    // and the tail wave of one contraction overlaps the head of the next.
    // Three operand buffers: rows of chunk i reuse the buffer of chunk i-3.
    const int N = (int)(a->nv * a->nl);
    const scmc_tuning T = tuning_for(SCMC_TUNE_COV, a->precision, N);
    TcPlan plan = tc_plan(N, a->precision == SCMC_PREC_MIXED, c.tc_chunk_bytes, T.chunk_events, T.stages);
    const size_t acc_bytes = (size_t)2 * N * N * sizeof(double);
    double *Ds0 = reinterpret_cast<double *>(c.acc_s.ensure(2 * acc_bytes));
    double *Dm0 = reinterpret_cast<double *>(c.acc_m.ensure(2 * acc_bytes));
    double *Ds[2] = {Ds0, Ds0 + acc_bytes / sizeof(double)};
    double *Dm[2] = {Dm0, Dm0 + acc_bytes / sizeof(double)};
    CK(cudaMemsetAsync(Ds0, 0, 2 * acc_bytes, st));
    CK(cudaMemsetAsync(Dm0, 0, 2 * acc_bytes, st));
    const int64_t chunk = plan.events_per_chunk;
    constexpr int NB = 3;
    const size_t ob = tc_operand_bytes(plan);
    char *omem = reinterpret_cast<char *>(c.tc_a.ensure(NB * ob));
    TcOperands ops[NB];
    for (int k = 0; k < NB; ++k) ops[k] = tc_make_operands(plan, omem + k * ob, st);
    for (int k = 1; k < NB; ++k) ops[k].af = ops[0].af;
    const bool ffff = a->is_ff_l && a->is_ff_v;
    if (ffff) {
        af_table_kernel<DIM><<<std::max(1, std::min(1024, (N + 255) / 256)), 256, 0, st>>>(P.Q, ops[0].af);
        CK(cudaGetLastError());
        LAUNCHED();
    }
    c.make_aux();
    cudaStream_t rs = c.aux, cs0 = c.aux3, cs1 = c.aux2;
    cudaEvent_t *ev_rows = &c.ev[0], *ev_free = &c.ev[3];
    cudaEvent_t ev_setup = c.ev[6], ev_end_rs = c.ev[7], ev_end_c1 = c.ev[8], ev_end_c0 = c.ev[9];
    CK(cudaEventRecord(ev_setup, st));
    CK(cudaStreamWaitEvent(rs, ev_setup, 0));   // accumulators, operands, af table, mean1
    CK(cudaStreamWaitEvent(cs0, ev_setup, 0));
    CK(cudaStreamWaitEvent(cs1, ev_setup, 0));
    int64_t chunk_id = 0;
    WalkParams W = P.W;
    for (int64_t done = 0; done < a->max_itr;) {
        int64_t nb = path_batch_size(a->max_itr - done, T.path_batch);
        W.path_base = a->path_offset + (uint64_t)done;
        Batch B;
        walk_batch(c, W, nb, rs, B);  // after the previous batch's rows (same stream)
        if (mean1_acc) launch_field_accum<DIM, PMIX, true, double>(c, P, B, mean1_acc, B.n_paths, rs, 1);
        for (int pass = 0; pass < 2; ++pass) {
            const bool single = pass == 0;
            const int64_t n_ev = single ? B.n_paths : B.n_multi;
            for (int64_t e0 = 0; e0 < n_ev; e0 += chunk, ++chunk_id) {
                const int64_t n = std::min(chunk, n_ev - e0);
                const int b = (int)(chunk_id % NB), d = (int)(chunk_id & 1);
                cudaStream_t cs = d ? cs1 : cs0;
                if (chunk_id >= NB) CK(cudaStreamWaitEvent(rs, ev_free[b], 0));  // chunk_id - NB has read buffer b
                {
                    StageScope sc(ST_ROWS, rs);
                    if (plan.split) {
                        if (single) tc_rows<DIM, true, true>(plan, ops[b], P.Q, B.S, c.scap, B.M, c.mcap, e0, n, ffff, rs);
                        else tc_rows<DIM, false, true>(plan, ops[b], P.Q, B.S, c.scap, B.M, c.mcap, e0, n, false, rs);
                    } else {
                        if (single) tc_rows<DIM, true, false>(plan, ops[b], P.Q, B.S, c.scap, B.M, c.mcap, e0, n, ffff, rs);
                        else tc_rows<DIM, false, false>(plan, ops[b], P.Q, B.S, c.scap, B.M, c.mcap, e0, n, false, rs);
                    }
                    CK(cudaGetLastError());
                    LAUNCHED();
                }
                CK(cudaEventRecord(ev_rows[b], rs));
                CK(cudaStreamWaitEvent(cs, ev_rows[b], 0));
                {
                    StageScope sc(ST_CONTRACT, cs);
                    tc_herk(plan, ops[b], n, single ? Ds[d] : Dm[d], cs);
                    CK(cudaGetLastError());
                    LAUNCHED();
                }
                CK(cudaEventRecord(ev_free[b], cs));
                prof_count(0, 0, 4.0 * (double)N * (double)(N + 1) * (double)n);
            }
        }
        done += nb;
    }
    CK(cudaEventRecord(ev_end_rs, rs));
    CK(cudaEventRecord(ev_end_c0, cs0));
    CK(cudaEventRecord(ev_end_c1, cs1));
    CK(cudaStreamWaitEvent(st, ev_end_rs, 0));
    CK(cudaStreamWaitEvent(st, ev_end_c0, 0));
    CK(cudaStreamWaitEvent(st, ev_end_c1, 0));
    int herr[NB] = {0, 0, 0};
    for (int k = 0; k < NB; ++k) CK(cudaMemcpyAsync(&herr[k], ops[k].err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr[0] || herr[1] || herr[2]) fail(SCMC_ERR_TIMEOUT, "tensor-core contraction: a bounded wait gave up");
    double m = (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
    double sc = m > 0 ? 1.0 / m * P.volume * a->sigt : 0.0;
    double scm = a->do_cbs ? sc / 2.0 : sc;
    int64_t total = (int64_t)N * N;
    int grid = (int)std::min<int64_t>((total + 255) / 256, 4096);
    StageScope fin(ST_FINAL, st);
    if (d_Ms) {
        cov_finalize_kernel<double><<<grid, 256, 0, st>>>(Ds[0], Ds[1], 1, (int)a->nv, (int)a->nl, sc, d_Ms);
        CK(cudaGetLastError());
        LAUNCHED();
    }
    if (d_Mm) {
        cov_finalize_kernel<double><<<grid, 256, 0, st>>>(Dm[0], Dm[1], 1, (int)a->nv, (int)a->nl, scm, d_Mm);
        CK(cudaGetLastError());
        LAUNCHED();
    }
}

void cov_device_locked(Ctx &c, const scmc_mc_args *a, double *d_Ms, double *d_Mm, cudaStream_t st)
{
    CK(cudaSetDevice(a->device));
    Prepared P = prepare(c, a, 0, st);
    double2 *Ms = reinterpret_cast<double2 *>(d_Ms), *Mm = reinterpret_cast<double2 *>(d_Mm);
    if (a->dim == 3) {
        if (a->precision == SCMC_PREC_FP64) cov_run_cc<3, P64>(c, a, P, Ms, Mm, st);
        else if (a->precision == SCMC_PREC_FP32) cov_run_cc<3, P32>(c, a, P, Ms, Mm, st);
        else cov_run_tc<3>(c, a, P, Ms, Mm, st);
    } else {
        if (a->precision == SCMC_PREC_FP64) cov_run_cc<2, P64>(c, a, P, Ms, Mm, st);
        else if (a->precision == SCMC_PREC_FP32) cov_run_cc<2, P32>(c, a, P, Ms, Mm, st);
        else cov_run_tc<2>(c, a, P, Ms, Mm, st);
    }
}

// ---------------------------------------------------------------------------
// records export
// ---------------------------------------------------------------------------
__global__ void expand_records_kernel(SingleRec S, int64_t scap, MultiRec M, int64_t mcap, const int64_t *moff,
                                      int64_t n_paths, int64_t base_ev, int64_t base_path, double *x, double *ow,
                                      double *x1, double *w1, double *wpx, double *xi, int32_t *plen, int64_t *path)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n_paths; p += (int64_t)gridDim.x * blockDim.x) {
        int64_t mo = moff[p];
        int64_t e = base_ev + mo + p;  // events of earlier paths: singles p + multis mo
        int nev = S.nev[p];
        for (int k = 0; k < nev; ++k) {
            int64_t o = e + k;
            for (int d = 0; d < 3; ++d) {
                double xv = k == 0 ? S.x1[d * scap + p] : M.x[d * mcap + mo + k - 1];
                double ov = k == 0 ? 0.0 : M.ow[d * mcap + mo + k - 1];
                x[3 * o + d] = xv;
                ow[3 * o + d] = ov;
                x1[3 * o + d] = S.x1[d * scap + p];
                w1[3 * o + d] = S.w1[d * scap + p];
            }
            wpx[o] = k == 0 ? S.wpx[p] : M.wpx[mo + k - 1];
            xi[o] = k == 0 ? S.xi[p] : M.xi[mo + k - 1];
            plen[o] = k + 1;
            path[o] = base_path + p;
        }
    }
}

void export_records(const scmc_mc_args *a, int want_phase, int64_t capacity, double *x, double *ow, double *x1,
                    double *w1, double *wpx, double *xi, int32_t *plen, int64_t *path, int64_t *n_events)
{
    validate(a);
    Ctx &c = context(a->device);
    std::lock_guard<std::mutex> lk(c.mu);
    CK(cudaSetDevice(a->device));
    cudaStream_t st = 0;
    Prepared P = prepare(c, a, want_phase, st);
    WalkParams W = P.W;
    W.any_order = 0;  // the export is in path order
    int64_t total = 0;
    std::vector<Batch> dummy;
    // first pass: count all events
    for (int64_t done = 0; done < a->max_itr;) {
        int64_t nb = path_batch_size(a->max_itr - done);
        W.path_base = a->path_offset + (uint64_t)done;
        Batch B;
        walk_batch(c, W, nb, st, B);
        total += B.n_paths + B.n_multi;
        done += nb;
    }
    *n_events = total;
    if (total > capacity) fail(SCMC_ERR_LIMIT, "record capacity too small");
    DevBuf out;
    size_t bytes = (size_t)std::max<int64_t>(total, 1) * (12 * 8 + 8 + 8 + 4 + 8);
    char *base = reinterpret_cast<char *>(out.ensure(bytes));
    int64_t T = std::max<int64_t>(total, 1);
    double *dx = reinterpret_cast<double *>(base);
    double *dow = dx + 3 * T, *dx1 = dow + 3 * T, *dw1 = dx1 + 3 * T, *dwpx = dw1 + 3 * T, *dxi = dwpx + T;
    int64_t *dpath = reinterpret_cast<int64_t *>(dxi + T);
    int32_t *dplen = reinterpret_cast<int32_t *>(dpath + T);
    int64_t ev = 0;
    for (int64_t done = 0; done < a->max_itr;) {
        int64_t nb = path_batch_size(a->max_itr - done);
        W.path_base = a->path_offset + (uint64_t)done;
        Batch B;
        walk_batch(c, W, nb, st, B);
        expand_records_kernel<<<256, 128, 0, st>>>(B.S, c.scap, B.M, c.mcap, c.moff.as<int64_t>(), nb, ev, done,
                                                   dx, dow, dx1, dw1, dwpx, dxi, dplen, dpath);
        CK(cudaGetLastError());
        LAUNCHED();
        ev += B.n_paths + B.n_multi;
        done += nb;
    }
    if (total > 0) {
        CK(cudaMemcpyAsync(x, dx, 3 * total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(ow, dow, 3 * total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(x1, dx1, 3 * total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(w1, dw1, 3 * total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(wpx, dwpx, total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(xi, dxi, total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(plen, dplen, total * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(path, dpath, total * 8, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    CK(cudaFree(out.p));
}

// The per-path streams exactly as the walk draws them (device arithmetic).
__global__ void philox_stream_kernel(uint64_t seed, uint64_t path, int tag, int64_t n, double *out)
{
    PathRng r;
    r.init((uint32_t)seed, (uint32_t)(seed >> 32), path);
    for (int64_t i = 0; i < n; ++i) out[i] = tag ? r.randn() : r.rand();
}

// ---------------------------------------------------------------------------
// heterogeneous medium (MCCovHetro / MCsampleHetro)
// ---------------------------------------------------------------------------
struct HeteroBufs {
    DevBuf sigt, sigt_f, alb, cdf, mean1, zeros;
};
HeteroBufs g_hbufs[64];

// The positional arguments as the homogeneous kernels see them (sigt = 1 and
// unit volume, so their normalisations reduce to 1/maxItr, MCCovHetro.m:268-269)
// plus the voxel grid.
Prepared prepare_hetero(Ctx &c, const scmc_hetero_args *h, int want_phase, bool cov, cudaStream_t st,
                        scmc_mc_args &mc)
{
    mc = h->mc;
    mc.sigt = 1.0;
    if (cov) mc.has_lmean0 = 0;  // MCCovHetro.m:38 uses mean(l,2)
    validate(&mc);
    if (!h->sigt_grid) fail(SCMC_ERR_INVALID, "null sigt grid");
    if (mc.smp_flg == 1 && h->has_lrad)
        fail(SCMC_ERR_INVALID, "lrad with uniform voxel sampling (smpFlg 1) is not supported");
    const int dim = mc.dim;
    HGrid g{};
    g.dim = dim;
    int64_t nv = 1;
    double vb = 1.0, diag = 0.0;
    for (int k = 0; k < dim; ++k) {
        if (!(h->box_bin[k] > 0)) fail(SCMC_ERR_INVALID, "box_bin must be positive");
        g.bmin[k] = mc.box_min[k];
        g.bmax[k] = mc.box_max[k];
        g.bbin[k] = h->box_bin[k];
        g.ibbin[k] = 1.0 / g.bbin[k];
        g.nb[k] = (int)std::llround((g.bmax[k] - g.bmin[k]) / g.bbin[k]);  // findBin.m:4
        if (g.nb[k] < 1) fail(SCMC_ERR_INVALID, "the box holds no voxel");
        nv *= g.nb[k];
        vb *= g.bbin[k];
        diag += (g.bmax[k] - g.bmin[k]) * (g.bmax[k] - g.bmin[k]);
    }
    g.n_vox = nv;
    g.n_icdf = nv * 100;  // MCCovHetro.m:63
    double ssum = 0.0, smax = 0.0;
    std::vector<double> cdf(nv);
    for (int64_t i = 0; i < nv; ++i) {
        if (!(h->sigt_grid[i] >= 0)) fail(SCMC_ERR_INVALID, "sigt must be non-negative");
        ssum += h->sigt_grid[i];
        smax = std::fmax(smax, h->sigt_grid[i]);
    }
    if (!(smax > 0)) fail(SCMC_ERR_INVALID, "sigt grid is all zero");
    double acc = 0.0, lo = INFINITY, hi = -INFINITY;
    for (int64_t i = 0; i < nv; ++i) {
        acc += h->sigt_grid[i] / ssum;
        cdf[i] = acc;
        lo = std::fmin(lo, acc);
        hi = std::fmax(hi, acc);
    }
    g.sigt_max = smax;
    g.cdf_lo = lo;
    g.cdf_step = (hi - lo) / (double)g.n_icdf;
    g.inv_V = 1.0 / (ssum * vb);  // px = 1/V, V = sum(sigt) prod(box_bin)
    g.lrad = h->has_lrad ? h->lrad : std::sqrt(diag);
    if (h->trilinear != 0 && h->trilinear != 1) fail(SCMC_ERR_INVALID, "trilinear must be 0 or 1");
    g.trilinear = h->trilinear;
    for (int k = 0; k < 6; ++k) g.basis[k] = h->null_basis[k];
    HeteroBufs &hb = g_hbufs[c.device];
    double *dsig = reinterpret_cast<double *>(hb.sigt.ensure(nv * sizeof(double)));
    double *dcdf = reinterpret_cast<double *>(hb.cdf.ensure(nv * sizeof(double)));
    CK(cudaMemcpyAsync(dsig, h->sigt_grid, nv * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dcdf, cdf.data(), nv * sizeof(double), cudaMemcpyHostToDevice, st));
    g.sigt = dsig;
    g.cdf = dcdf;
    g.sigt_f = nullptr;
    std::vector<float> sig_f;
    if (g.trilinear && mc.precision != SCMC_PREC_FP64) {  // the FP32 NEE march reads an FP32 copy
        sig_f.assign(h->sigt_grid, h->sigt_grid + nv);
        float *dsf = reinterpret_cast<float *>(hb.sigt_f.ensure(nv * sizeof(float)));
        CK(cudaMemcpyAsync(dsf, sig_f.data(), nv * sizeof(float), cudaMemcpyHostToDevice, st));
        g.sigt_f = dsf;
    }
    g.alb_scalar = mc.albedo;
    g.alb = nullptr;
    if (h->albedo_grid) {
        double *dalb = reinterpret_cast<double *>(hb.alb.ensure(nv * sizeof(double)));
        CK(cudaMemcpyAsync(dalb, h->albedo_grid, nv * sizeof(double), cudaMemcpyHostToDevice, st));
        g.alb = dalb;
    }
    Prepared P = prepare(c, &mc, want_phase, st);  // synchronises the stream (host vectors above)
    P.volume = 1.0;
    P.W.hetero = 1;
    P.W.hg = g;
    P.Q.hetero = 1;
    P.Q.hg = g;
    return P;
}

void cov_hetero_locked(Ctx &c, const scmc_hetero_args *h, double *d_Ms, double *d_Mm, double *d_mean1,
                       cudaStream_t st)
{
    CK(cudaSetDevice(h->mc.device));
    scmc_mc_args mc;
    Prepared P = prepare_hetero(c, h, 0, true, st, mc);
    HeteroBufs &hb = g_hbufs[c.device];
    const int64_t n1 = mc.nv * mc.nl;
    double *m1 = reinterpret_cast<double *>(hb.mean1.ensure(2 * n1 * sizeof(double)));
    double *z = reinterpret_cast<double *>(hb.zeros.ensure(2 * n1 * sizeof(double)));
    CK(cudaMemsetAsync(m1, 0, 2 * n1 * sizeof(double), st));
    CK(cudaMemsetAsync(z, 0, 2 * n1 * sizeof(double), st));
    double2 *Ms = reinterpret_cast<double2 *>(d_Ms), *Mm = reinterpret_cast<double2 *>(d_Mm);
    const scmc_mc_args *a = &mc;
    if (mc.dim == 3) {
        if (mc.precision == SCMC_PREC_FP64) cov_run_cc<3, P64>(c, a, P, Ms, Mm, st, m1);
        else if (mc.precision == SCMC_PREC_FP32) cov_run_cc<3, P32>(c, a, P, Ms, Mm, st, m1);
        else cov_run_tc<3>(c, a, P, Ms, Mm, st, m1);
    } else {
        if (mc.precision == SCMC_PREC_FP64) cov_run_cc<2, P64>(c, a, P, Ms, Mm, st, m1);
        else if (mc.precision == SCMC_PREC_FP32) cov_run_cc<2, P32>(c, a, P, Ms, Mm, st, m1);
        else cov_run_tc<2>(c, a, P, Ms, Mm, st, m1);
    }
    if (d_mean1) {
        // MCCovHetro.m:276: mean1 / maxItr / sqrt(cs), cs = 1 (see the header)
        const double m = (double)(mc.norm_itr > 0 ? mc.norm_itr : mc.max_itr);
        const double norm = m > 0 ? 1.0 / m : 0.0;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n1 + 255) / 256, 1024));
        if (mc.dim == 3)
            field_finalize_kernel<3, double><<<grid, 256, 0, st>>>(P.Q, m1, z, norm, reinterpret_cast<double2 *>(d_mean1));
        else
            field_finalize_kernel<2, double><<<grid, 256, 0, st>>>(P.Q, m1, z, norm, reinterpret_cast<double2 *>(d_mean1));
        CK(cudaGetLastError());
        LAUNCHED();
    }
}

void field_hetero_locked(Ctx &c, const scmc_hetero_args *h, double *d_u, cudaStream_t st)
{
    CK(cudaSetDevice(h->mc.device));
    scmc_mc_args mc;
    Prepared P = prepare_hetero(c, h, 1, false, st, mc);
    double2 *u = reinterpret_cast<double2 *>(d_u);
    const scmc_mc_args *a = &mc;
    if (mc.dim == 3) {
        if (mc.precision == SCMC_PREC_FP64) field_run<3, P64, double>(c, a, P, u, st);
        else if (mc.precision == SCMC_PREC_FP32) field_run<3, P32, float>(c, a, P, u, st);
        else field_run<3, PMIX, double>(c, a, P, u, st);
    } else {
        if (mc.precision == SCMC_PREC_FP64) field_run<2, P64, double>(c, a, P, u, st);
        else if (mc.precision == SCMC_PREC_FP32) field_run<2, P32, float>(c, a, P, u, st);
        else field_run<2, PMIX, double>(c, a, P, u, st);
    }
}

// ---------------------------------------------------------------------------
// MCfieldFourierQuad
// ---------------------------------------------------------------------------
int64_t colon_count(double a, double st, double b)
{
    if (st == 0 || (st > 0 && a > b) || (st < 0 && a < b)) return 0;
    double q = (b - a) / st;
    return (int64_t)std::floor(q + 1e-10 * std::fmax(1.0, std::fabs(q))) + 1;
}

void validate_fq(const scmc_fq_args *a)
{
    if (!a) fail(SCMC_ERR_INVALID, "null arguments");
    for (int k = 0; k < 3; ++k)
        if (!(a->box_max[k] >= a->box_min[k])) fail(SCMC_ERR_INVALID, "Invalid box size");
    if (a->nl < 1 || !a->l) fail(SCMC_ERR_INVALID, "Invalid light source input");
    if (!(a->sigt > 0) || !(a->lambda > 0)) fail(SCMC_ERR_INVALID, "sigt and lambda must be positive");
    if (!(a->v_stp > 0) || !(a->v_max >= 0)) fail(SCMC_ERR_INVALID, "v_max must be >= 0 and v_stp > 0");
    if (a->max_itr < 0) fail(SCMC_ERR_INVALID, "Invalid photons number");
    if (a->smp_flg != 1 && a->smp_flg != 2) fail(SCMC_ERR_INVALID, "smpFlg must be 1 or 2");
    if (a->precision < 0 || a->precision > 3) fail(SCMC_ERR_INVALID, "invalid precision mode");
    if (colon_count(-a->v_max, a->v_stp, a->v_max) > 4096) fail(SCMC_ERR_INVALID, "angular grid longer than 4096");
    if (a->light_point != 0 && a->light_point != 1) fail(SCMC_ERR_INVALID, "light_point must be 0 or 1");
    if (a->sct_type != 0 && a->sct_type != SCMC_SCT_ISOTROPIC && a->sct_type != SCMC_SCT_HG)
        fail(SCMC_ERR_INVALID, "FourierQuad sct_type must be isotropic or HG");
    if (a->sct_type == SCMC_SCT_HG && !(std::fabs(a->g) <= 1.0)) fail(SCMC_ERR_INVALID, "Invalid g input");
}

// The per-plane DFT sums of one batch on tcgen05 (fq.cuh, tensor-core form),
// added into U stored [light][r1][r2] in FP64 (each plane's sum is FP32 in
// TMEM; the sum across planes and batches is FP64).  Tt: the twiddles stored [p][r]; dz: zexp0 stored [r2][r1].
// Nonempty planes are taken in groups of at most group_entries padded entries
// (operand memory; tuned, 2^20 built in) and kFqTcPlanes planes.
constexpr int kFqTcPlanes = 16384;

void fq_tc_batch(Ctx &c, const FqParams &F, int nl_out, const FqEntry *Es, const std::vector<int> &hcounts,
                 const std::vector<int> &hoff, const std::vector<int> &hplanes, const float2 *Tt, const double2 *dz,
                 const float2 *rr, int n_uniform, double *U, bool split, int64_t group_entries, cudaStream_t st)
{
    const int nv0 = F.nv0;
    const int Mr = 2 * nv0;
    std::vector<int2> tiles;
    for (int tn = 0; tn < (nv0 + TC_BN - 1) / TC_BN; ++tn)
        for (int tm = 0; tm < (Mr + TC_BM - 1) / TC_BM; ++tm) tiles.push_back(make_int2(tm, tn));
    // Every group's metadata is built first and uploaded in one copy, so the
    // groups then run back to back with one synchronisation at the end.
    struct Group {
        int64_t nblk, blk0, kr0, pl0, pr0;
        int n_pl, n_pr;
        int64_t entries;
    };
    std::vector<Group> groups;
    std::vector<int2> blk, kr, prs;
    std::vector<int> gpl;
    int64_t max_nblk = 0;
    constexpr int64_t kFqPlaneCost = 1;  // a plane's epilogue step, in K blocks, for balancing the plane ranges
    const int want_max = std::max(1, sm_count(c.device) / std::max(1, (int)tiles.size()));
    for (size_t g0 = 0; g0 < hplanes.size();) {
        // group [g0, g1): blocks of 32 entries per plane
        Group G{0, (int64_t)blk.size(), (int64_t)kr.size(), (int64_t)gpl.size(), (int64_t)prs.size(), 0, 0, 0};
        size_t g1 = g0;
        while (g1 < hplanes.size() && G.n_pl < kFqTcPlanes) {
            const int p = hplanes[g1];
            const int cnt = hcounts[p];
            const int nb = (cnt + 31) / 32;
            if (G.n_pl > 0 && (G.nblk + nb) * 32 > group_entries) break;
            kr.push_back(make_int2((int)G.nblk, nb));
            for (int b = 0; b < nb; ++b) blk.push_back(make_int2(hoff[p] + 32 * b, std::min(32, cnt - 32 * b)));
            gpl.push_back(p);
            G.nblk += nb;
            G.entries += cnt;
            ++G.n_pl;
            ++g1;
        }
        // plane ranges of about equal work (K blocks plus a fixed cost per
        // plane), about one CTA per SM over the tiles
        const int want = std::min(G.n_pl, want_max);
        const int64_t per = (G.nblk + kFqPlaneCost * G.n_pl + want - 1) / want;
        int first = 0;
        int64_t acc = 0;
        for (int i = 0; i < G.n_pl; ++i) {
            acc += kr[G.kr0 + i].y + kFqPlaneCost;
            if (acc >= per || i + 1 == G.n_pl) {
                prs.push_back(make_int2(first, i - first + 1));
                first = i + 1;
                acc = 0;
            }
        }
        G.n_pr = (int)(prs.size() - G.pr0);
        max_nblk = std::max(max_nblk, G.nblk);
        groups.push_back(G);
        g0 = g1;
    }
    if (groups.empty()) return;
    const int64_t Kmax = 64 * max_nblk;
    const size_t ab = tc_align((size_t)Mr * Kmax * sizeof(__half)), bb = tc_align((size_t)nv0 * Kmax * sizeof(__half));
    // metadata: tiles, blocks, K ranges, planes, plane ranges, error flag
    const size_t o_tiles = 0, o_blk = o_tiles + tc_align(tiles.size() * sizeof(int2));
    const size_t o_kr = o_blk + tc_align(blk.size() * sizeof(int2));
    const size_t o_pl = o_kr + tc_align(kr.size() * sizeof(int2));
    const size_t o_pr = o_pl + tc_align(gpl.size() * sizeof(int));
    const size_t o_err = o_pr + tc_align(prs.size() * sizeof(int2));
    const size_t o_max = o_err + 256;  // the group's max |s_e| bits (reset per group and light)
    const size_t meta = o_err + 1024;
    char *mem = reinterpret_cast<char *>(c.tc_a.ensure((split ? 2 : 1) * ab + bb + meta));
    __half *ahi = reinterpret_cast<__half *>(mem);
    __half *alo = split ? reinterpret_cast<__half *>(mem + ab) : ahi;
    __half *bm = reinterpret_cast<__half *>(mem + (split ? 2 : 1) * ab);
    char *dmeta = mem + (split ? 2 : 1) * ab + bb;
    std::vector<char> hmeta(o_err, 0);
    std::memcpy(hmeta.data() + o_tiles, tiles.data(), tiles.size() * sizeof(int2));
    std::memcpy(hmeta.data() + o_blk, blk.data(), blk.size() * sizeof(int2));
    std::memcpy(hmeta.data() + o_kr, kr.data(), kr.size() * sizeof(int2));
    std::memcpy(hmeta.data() + o_pl, gpl.data(), gpl.size() * sizeof(int));
    std::memcpy(hmeta.data() + o_pr, prs.data(), prs.size() * sizeof(int2));
    CK(cudaMemcpyAsync(dmeta, hmeta.data(), o_err, cudaMemcpyHostToDevice, st));
    int2 *d_tiles = reinterpret_cast<int2 *>(dmeta + o_tiles), *d_blk = reinterpret_cast<int2 *>(dmeta + o_blk);
    int2 *d_kr = reinterpret_cast<int2 *>(dmeta + o_kr), *d_pr = reinterpret_cast<int2 *>(dmeta + o_pr);
    int *d_pl = reinterpret_cast<int *>(dmeta + o_pl), *d_err = reinterpret_cast<int *>(dmeta + o_err);
    unsigned *d_max = reinterpret_cast<unsigned *>(dmeta + o_max);
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    for (const Group &G : groups) {
        const int64_t K = 64 * G.nblk;
        const CUtensorMap m_ahi = tc_map(ahi, (uint64_t)K, (uint64_t)Mr, (uint64_t)K * 2, TC_BM);
        const CUtensorMap m_alo = tc_map(alo, (uint64_t)K, (uint64_t)Mr, (uint64_t)K * 2, TC_BM);
        const CUtensorMap m_b = tc_map(bm, (uint64_t)K, (uint64_t)nv0, (uint64_t)K * 2, TC_BN);
        for (int j = 0; j < nl_out; ++j) {
            {
                StageScope sc(ST_ROWS, st);
                CK(cudaMemsetAsync(d_max, 0, sizeof(unsigned), st));
                fq_scale_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((G.nblk * 32 + 255) / 256,
                                                                                   (int64_t)sm_count(c.device) * 8)),
                                  256, 0, st>>>(F, Es, d_blk + G.blk0, G.nblk, 32, j, d_max);
                CK(cudaGetLastError());
                LAUNCHED();
                if (split)
                    fq_tc_rows_kernel<true><<<(unsigned)G.nblk, 256, 0, st>>>(F, Es, d_blk + G.blk0, j, Tt, K, ahi,
                                                                                alo, bm, d_max);
                else
                    fq_tc_rows_kernel<false><<<(unsigned)G.nblk, 256, 0, st>>>(F, Es, d_blk + G.blk0, j, Tt, K, ahi,
                                                                                 alo, bm, d_max);
                CK(cudaGetLastError());
                LAUNCHED();
            }
            {
                StageScope sc(ST_CONTRACT, st);
                const PlaneEpi pe{dz, rr, F.gz, d_pl + G.pl0, U + 2 * (int64_t)nv0 * nv0 * j, nv0, n_uniform, d_max};
                if (split)
                    tc_gemm_plane_loop_launch<true>(m_ahi, m_alo, m_b, d_tiles, (int)tiles.size(), d_kr + G.kr0,
                                                    d_pr + G.pr0, G.n_pr, Mr, nv0, pe, d_err, st);
                else
                    tc_gemm_plane_loop_launch<false>(m_ahi, m_alo, m_b, d_tiles, (int)tiles.size(), d_kr + G.kr0,
                                                     d_pr + G.pr0, G.n_pr, Mr, nv0, pe, d_err, st);
                CK(cudaGetLastError());
                LAUNCHED();
            }
            prof_count(0, 0, 8.0 * (double)nv0 * nv0 * (double)G.entries);
        }
    }
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));  // the operand memory and metadata are reused by the next batch
    if (herr) fail(SCMC_ERR_TIMEOUT, "tensor-core contraction: a bounded wait gave up");
}

// The same on CTA pairs from planar operands (grids of at least 128 angles):
// 64-entry blocks, one K column per entry, a pair per 256 x 256 output tile,
// one Horner chain per pair (fq_pair_planes_kernel).  r1step: exp(zexp0 z_bin).
void fq_tc_batch_pair(Ctx &c, const FqParams &F, int nl_out, const void *Es, bool compact, const std::vector<int> &hcounts,
                      const std::vector<int> &hoff, const std::vector<int> &hplanes, const float2 *Tt,
                      const double2 *dz, const float2 *r1step, int n_uniform, double *U, bool split,
                      int64_t group_entries, int *d_err, PinnedBuf &hpin, cudaStream_t st)
{
    const int nv0 = F.nv0;
    std::vector<int2> tiles;
    const int nt = (nv0 + 255) / 256;
    for (int tn = 0; tn < nt; ++tn)
        for (int tm = 0; tm < nt; ++tm) tiles.push_back(make_int2(tm, tn));
    struct Group {
        int64_t nblk, blk0, kr0, pl0, pr0;
        int n_pl, n_pr;
        int64_t entries;
    };
    std::vector<Group> groups;
    std::vector<int2> blk, kr, prs;
    std::vector<int> gpl;
    int64_t max_nblk = 0;
    constexpr int64_t kPlaneCost = 1;
    const int want_max = std::max(1, (sm_count(c.device) / 2) / std::max(1, (int)tiles.size()));
    for (size_t g0 = 0; g0 < hplanes.size();) {
        Group G{0, (int64_t)blk.size(), (int64_t)kr.size(), (int64_t)gpl.size(), (int64_t)prs.size(), 0, 0, 0};
        size_t g1 = g0;
        while (g1 < hplanes.size() && G.n_pl < kFqTcPlanes) {
            const int p = hplanes[g1];
            const int cnt = hcounts[p];
            const int nb = (cnt + 63) / 64;
            if (G.n_pl > 0 && (G.nblk + nb) * 64 > group_entries) break;
            kr.push_back(make_int2((int)G.nblk, nb));
            for (int b = 0; b < nb; ++b) blk.push_back(make_int2(hoff[p] + 64 * b, std::min(64, cnt - 64 * b)));
            gpl.push_back(p);
            G.nblk += nb;
            G.entries += cnt;
            ++G.n_pl;
            ++g1;
        }
        const int want = std::min(G.n_pl, want_max);
        const int64_t per = (G.nblk + kPlaneCost * G.n_pl + want - 1) / want;
        int first = 0;
        int64_t acc = 0;
        for (int i = 0; i < G.n_pl; ++i) {
            acc += kr[G.kr0 + i].y + kPlaneCost;
            if (acc >= per || i + 1 == G.n_pl) {
                prs.push_back(make_int2(first, i - first + 1));
                first = i + 1;
                acc = 0;
            }
        }
        G.n_pr = (int)(prs.size() - G.pr0);
        max_nblk = std::max(max_nblk, G.nblk);
        groups.push_back(G);
        g0 = g1;
    }
    if (groups.empty()) return;
    const size_t pb = tc_align((size_t)nv0 * 64 * max_nblk * sizeof(__half));  // one plane: [block][row][64]
    const int n_planes = split ? 6 : 4;                                // Re A, Im A, [Re lo, Im lo], Re B, Im B
    const size_t o_tiles = 0, o_blk = o_tiles + tc_align(tiles.size() * sizeof(int2));
    const size_t o_kr = o_blk + tc_align(blk.size() * sizeof(int2));
    const size_t o_pl = o_kr + tc_align(kr.size() * sizeof(int2));
    const size_t o_pr = o_pl + tc_align(gpl.size() * sizeof(int));
    const size_t o_err = o_pr + tc_align(prs.size() * sizeof(int2));
    const size_t o_max = o_err + 256;
    const size_t o_sv = o_err + 1024;                                   // sv per K column
    const size_t o_pp = o_sv + tc_align((size_t)64 * max_nblk * sizeof(float2));  // (p1, p2) per K column
    const size_t meta = o_pp + tc_align((size_t)64 * max_nblk * sizeof(int2));
    char *mem = reinterpret_cast<char *>(c.tc_a.ensure(n_planes * pb + meta));
    __half *are = reinterpret_cast<__half *>(mem), *aim = reinterpret_cast<__half *>(mem + pb);
    __half *alr = split ? reinterpret_cast<__half *>(mem + 2 * pb) : are;
    __half *ali = split ? reinterpret_cast<__half *>(mem + 3 * pb) : aim;
    __half *bre = reinterpret_cast<__half *>(mem + (split ? 4 : 2) * pb);
    __half *bim = reinterpret_cast<__half *>(mem + (split ? 5 : 3) * pb);
    char *dmeta = mem + n_planes * pb;
    // the caller guarantees that the previous copy out of hpin has completed
    char *hmeta = reinterpret_cast<char *>(hpin.ensure(o_err));
    std::memset(hmeta, 0, o_err);
    std::memcpy(hmeta + o_tiles, tiles.data(), tiles.size() * sizeof(int2));
    std::memcpy(hmeta + o_blk, blk.data(), blk.size() * sizeof(int2));
    std::memcpy(hmeta + o_kr, kr.data(), kr.size() * sizeof(int2));
    std::memcpy(hmeta + o_pl, gpl.data(), gpl.size() * sizeof(int));
    std::memcpy(hmeta + o_pr, prs.data(), prs.size() * sizeof(int2));
    CK(cudaMemcpyAsync(dmeta, hmeta, o_err, cudaMemcpyHostToDevice, st));
    int2 *d_tiles = reinterpret_cast<int2 *>(dmeta + o_tiles), *d_blk = reinterpret_cast<int2 *>(dmeta + o_blk);
    int2 *d_kr = reinterpret_cast<int2 *>(dmeta + o_kr), *d_pr = reinterpret_cast<int2 *>(dmeta + o_pr);
    int *d_pl = reinterpret_cast<int *>(dmeta + o_pl);
    unsigned *d_max = reinterpret_cast<unsigned *>(dmeta + o_max);
    float2 *d_sv = reinterpret_cast<float2 *>(dmeta + o_sv);
    int2 *d_pp = reinterpret_cast<int2 *>(dmeta + o_pp);
    for (const Group &G : groups) {
        CUtensorMap maps[6];
        __half *planes[6] = {are, aim, alr, ali, bre, bim};
        for (int k = 0; k < 6; ++k) maps[k] = tc_map_kblocks(planes[k], (uint64_t)nv0, (uint64_t)G.nblk);
        for (int j = 0; j < nl_out; ++j) {
            {
                StageScope sc(ST_ROWS, st);
                CK(cudaMemsetAsync(d_max, 0, sizeof(unsigned), st));
                const unsigned pg = (unsigned)std::max<int64_t>(
                    1, std::min<int64_t>((G.nblk * 64 + 255) / 256, (int64_t)sm_count(c.device) * 8));
                if (compact)
                    fq_pair_prep_compact_kernel<<<pg, 256, 0, st>>>(reinterpret_cast<const FqEntryC *>(Es), d_blk + G.blk0,
                                                                    G.nblk, d_sv, d_pp, d_max);
                else
                    fq_pair_prep_kernel<<<pg, 256, 0, st>>>(F, reinterpret_cast<const FqEntry *>(Es), d_blk + G.blk0,
                                                            G.nblk, j, d_sv, d_pp, d_max);
                CK(cudaGetLastError());
                LAUNCHED();
                if (split)
                    fq_tc_rows_planar_kernel<true><<<(unsigned)G.nblk, 256, 0, st>>>(nv0, d_sv, d_pp, Tt, are, aim, alr,
                                                                                       ali, bre, bim, d_max);
                else
                    fq_tc_rows_planar_kernel<false><<<(unsigned)G.nblk, 256, 0, st>>>(nv0, d_sv, d_pp, Tt, are, aim, alr,
                                                                                        ali, bre, bim, d_max);
                CK(cudaGetLastError());
                LAUNCHED();
            }
            {
                StageScope sc(ST_CONTRACT, st);
                const PlaneEpi2 pe{dz, r1step, F.gz, d_pl + G.pl0, U + 2 * (int64_t)nv0 * nv0 * j, nv0, n_uniform, d_max};
                if (split)
                    fq_pair_planes_launch<true>(maps, d_tiles, (int)tiles.size(), d_kr + G.kr0, d_pr + G.pr0, G.n_pr, pe,
                                                d_err, st);
                else
                    fq_pair_planes_launch<false>(maps, d_tiles, (int)tiles.size(), d_kr + G.kr0, d_pr + G.pr0, G.n_pr,
                                                 pe, d_err, st);
                CK(cudaGetLastError());
                LAUNCHED();
            }
            prof_count(0, 0, 8.0 * (double)nv0 * nv0 * (double)G.entries);
        }
    }
    // no synchronisation: the next batch's metadata and operands are written on
    // the same stream after these kernels; d_err (set only on a failed wait)
    // is read once at the end of the solve
}

// Wl == null: MCfieldFourierQuad.m.  Wl (nl complex, host): MCfieldFourierQuadOnWave.m,
// which makes the pixel count's parity match the angular grid's (lines 97-99),
// flips the sign of zexp0's phase (line 140), uses vsign in the light and
// vertex phases and sums the weighted lights into one output (lines 278-302).
template <int POL, typename AccT>
void fq_run(Ctx &c, const scmc_fq_args *a, const double *Wl, double2 *d_u, cudaStream_t st)
{
    const int64_t nl_out = Wl ? 1 : a->nl;
    using R = typename std::conditional<POL == P64, double, float>::type;
    using Cx = typename cplx_t<R>::type;
    // geometry, as MCfieldFourierQuad.m:59-138
    const double lambda = a->lambda, sigt = a->sigt;
    double bmin[3], bmax[3], bw[3];
    for (int k = 0; k < 3; ++k) {
        bmin[k] = a->box_min[k];
        bmax[k] = a->box_max[k];
        bw[k] = bmax[k] - bmin[k];
    }
    double unmeanl[3] = {0, 0, 1};
    if (a->has_lmean0)
        for (int k = 0; k < 3; ++k) unmeanl[k] = a->lmean0[k];
    const int64_t Nv = colon_count(-a->v_max, a->v_stp, a->v_max);
    const double box_stp = lambda / (a->v_max * 2 + a->v_stp);
    int64_t Nx = (int64_t)std::ceil(bw[0] / box_stp / 2) * 2 + 1;
    if (Wl && (((Nv - Nx) % 2) + 2) % 2 == 1) Nx += 1;  // MCfieldFourierQuadOnWave.m:97-99
    if (Nx > (int64_t)1 << 20) fail(SCMC_ERR_INVALID, "lateral pixel grid too large");
    const double box_w_n = Nx * box_stp, grow = (box_w_n - bw[0]) / 2;
    for (int k = 0; k < 2; ++k) {
        bmin[k] -= grow;
        bmax[k] += grow;
        bw[k] = box_w_n;
    }
    const double nx_pad = std::fmax((double)(Nv - Nx) / 2, 0.0), nv_pad = std::fmax((double)(Nx - Nv) / 2, 0.0);
    const double M = (double)Nx + 2 * nx_pad;
    std::vector<double> theta(Nv);
    for (int64_t k = 0; k < Nv; ++k) theta[k] = -a->v_max + (double)k * a->v_stp;
    std::vector<double2> zexp0(Nv * Nv), boxexp0(Nv * Nv);
    double maxdiff = -INFINITY;
    std::vector<double> vzr(Nv * Nv), vzi(Nv * Nv);
    for (int64_t j = 0; j < Nv; ++j)
        for (int64_t i = 0; i < Nv; ++i) {
            const double vx = -theta[i], vy = -theta[j], r = 1 - vx * vx - vy * vy;
            double zr = r >= 0 ? std::sqrt(r) : 0.0, zi = r >= 0 ? 0.0 : std::sqrt(-r);
            zr *= a->vsign;
            zi *= a->vsign;
            vzr[i + Nv * j] = zr;
            vzi[i + Nv * j] = zi;
            maxdiff = std::fmax(maxdiff, 1 - std::hypot(zr, zi));
        }
    double z_bin = lambda / maxdiff / 5;
    z_bin = z_bin / 2;
    const int64_t ng = colon_count(bmin[2], z_bin, bmax[2]);
    const int64_t Nz = ng + 1;
    if (Nz > 1000000) fail(SCMC_ERR_INVALID, "too many z planes");
    std::vector<double> gz(Nz);
    for (int64_t k = 0; k < ng; ++k) gz[k] = bmin[2] + (double)k * z_bin;
    gz[ng] = bmax[2];
    const double twopi = 2 * SCMC_PI;
    for (int64_t q = 0; q < Nv * Nv; ++q) {
        const double zr = vzr[q], zi = vzi[q], av = std::hypot(zr, zi);
        const double dir = zr < 0 ? 1.0 / av : 0.0, idir = zr > 0 ? 1.0 / av : 0.0;
        // zexp0 = -2 pi i/lambda vz vsign - sigt/2 (diratt - idiratt); OnWave: +2 pi i/lambda
        const double zs = Wl ? -1.0 : 1.0;
        zexp0[q] = make_double2(zs * twopi / lambda * zi * a->vsign - sigt / 2 * (dir - idir),
                                -zs * twopi / lambda * zr * a->vsign);
        const double amp = std::exp(-sigt / 2 * (-bmin[2] * dir + bmax[2] * idir));
        const double sel = (zr < 0 ? -bmin[2] : 0.0) + (zr > 0 ? bmax[2] : 0.0);
        // exp(2 pi i/lambda * sel * vz)
        const double er = -twopi / lambda * sel * zi, ei = twopi / lambda * sel * zr;
        const double m = amp * std::exp(er);
        boxexp0[q] = make_double2(m * std::cos(ei), m * std::sin(ei));
    }
    // the Horner ratio of the tensor-core form: exp(zexp0 * 2 z_bin), planes P and P - 2
    std::vector<float2> rrh(Nv * Nv);
    for (int64_t q = 0; q < Nv * Nv; ++q) {
        const double m = std::exp(zexp0[q].x * 2 * z_bin), ph = zexp0[q].y * 2 * z_bin;
        rrh[q] = make_float2((float)(m * std::cos(ph)), (float)(m * std::sin(ph)));
    }
    std::vector<float2> r1h(Nv * Nv);  // the pair form's ratio between planes P and P - 1
    for (int64_t q = 0; q < Nv * Nv; ++q) {
        const double m = std::exp(zexp0[q].x * z_bin), ph = zexp0[q].y * z_bin;
        r1h[q] = make_float2((float)(m * std::cos(ph)), (float)(m * std::sin(ph)));
    }
    const int n_uniform = (int)(ng - 1);
    const double l_end = a->l[3 * (a->nl - 1) + 2];

    FqParams F{};
    F.nv0 = (int)Nv;
    F.nx = (int)Nx;
    F.nz = (int)Nz;
    F.nl = (int)a->nl;
    if (Wl && a->light_point) fail(SCMC_ERR_INVALID, "point sources are not supported with light weights");
    F.light_point = a->light_point;
    if (a->light_point) {
        NeeParams &Q = F.nf;
        Q.sigt_half = sigt / 2;
        Q.kw = twopi / lambda;
        Q.lambda = lambda;
        for (int k = 0; k < 3; ++k) {
            Q.box_min[k] = bmin[k];  // the padded box the walk runs in
            Q.box_max[k] = bmax[k];
        }
        nee_set_fbox(Q);
    }
    if (Wl) {
        F.lsign = a->vsign;
        F.vsign_vertex = a->vsign;
        double2 *dw = reinterpret_cast<double2 *>(c.wl.ensure(a->nl * sizeof(double2)));
        CK(cudaMemcpyAsync(dw, Wl, a->nl * sizeof(double2), cudaMemcpyHostToDevice, st));
        F.wl = dw;
    }
    F.cbs = a->do_cbs;
    F.box_stp = box_stp;
    F.gx1 = bmin[0] + box_stp / 2;
    F.gy1 = bmin[1] + box_stp / 2;
    F.kw = twopi / lambda;
    F.sigt_half = sigt / 2;
    F.bmin_z = bmin[2];
    F.bmax_z = bmax[2];
    F.l_diratt = l_end > 0 ? 1.0 / std::fabs(l_end) : 0.0;
    F.l_idiratt = l_end < 0 ? 1.0 / std::fabs(l_end) : 0.0;
    double *dgz = reinterpret_cast<double *>(c.fq_gz.ensure(Nz * sizeof(double)));
    double2 *dz = reinterpret_cast<double2 *>(c.fq_zexp.ensure(Nv * Nv * sizeof(double2)));
    double2 *db = reinterpret_cast<double2 *>(c.fq_box.ensure(Nv * Nv * sizeof(double2)));
    double *dl = reinterpret_cast<double *>(c.dirs_l.ensure(3 * a->nl * sizeof(double)));
    Cx *T = reinterpret_cast<Cx *>(c.fq_tw.ensure(Nv * Nx * sizeof(Cx)));
    CK(cudaMemcpyAsync(dgz, gz.data(), Nz * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dz, zexp0.data(), Nv * Nv * sizeof(double2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(db, boxexp0.data(), Nv * Nv * sizeof(double2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dl, a->l, 3 * a->nl * sizeof(double), cudaMemcpyHostToDevice, st));
    F.gz = dgz;
    F.l = dl;
    // MIXED / FP16 with at least 64 angles per axis: the per-plane sums on tcgen05
    const bool use_tc = POL == PMIX && (a->precision == SCMC_PREC_MIXED || a->precision == SCMC_PREC_FP16) &&
                        Nv >= 64;
    // the tensor-core rows read the twiddles transposed, [p][r]
    float2 *Tt = use_tc ? reinterpret_cast<float2 *>(c.fq_twt.ensure(Nv * Nx * sizeof(float2))) : nullptr;
    // at least 128 angles per axis: the CTA-pair form on planar operands
    const bool use_pair = use_tc && Nv >= 128;
    float2 *drr = use_tc ? reinterpret_cast<float2 *>(c.fq_rr.ensure(Nv * Nv * sizeof(float2))) : nullptr;
    if (use_tc)
        CK(cudaMemcpyAsync(drr, use_pair ? r1h.data() : rrh.data(), Nv * Nv * sizeof(float2), cudaMemcpyHostToDevice, st));
    {
        StageScope sc(ST_ROWS, st);
        const int tg = (int)std::max<int64_t>(1, std::min<int64_t>((Nv * Nx + 255) / 256, 4096));
        fq_twiddle_kernel<Cx><<<tg, 256, 0, st>>>((int)Nv, (int)Nx, M, nx_pad, nv_pad, T, 0);
        CK(cudaGetLastError());
        LAUNCHED();
        if (use_tc) {
            fq_twiddle_kernel<float2><<<tg, 256, 0, st>>>((int)Nv, (int)Nx, M, nx_pad, nv_pad, Tt, 1);
            CK(cudaGetLastError());
            LAUNCHED();
        }
    }
    // the walk: isotropic, phase per event, padded box (lines 146-213)
    WalkParams W{};
    W.dim = 3;
    W.smp_flg = a->smp_flg;
    W.has_pf0 = 0;
    W.want_phase = 1;
    W.sigt = sigt;
    W.albedo = a->albedo;
    double nrm = 0;
    for (int k = 0; k < 3; ++k) {
        W.box_min[k] = bmin[k];
        W.box_max[k] = bmax[k];
        W.box_w[k] = bw[k];
        W.unmeanl[k] = unmeanl[k];
        nrm += unmeanl[k] * unmeanl[k];
    }
    nrm = std::sqrt(nrm);
    for (int k = 0; k < 3; ++k) W.meanl[k] = unmeanl[k] / nrm;
    W.pf.sct_type = SCMC_SCT_ISOTROPIC;
    W.pf0 = W.pf;  // the first direction stays isotropic (line 171)
    if (a->sct_type == SCMC_SCT_HG) {  // extension: HG scattering directions (line 208's commented call)
        W.pf.sct_type = SCMC_SCT_HG;
        W.pf.g = a->g;
    }
    W.key0 = (uint32_t)a->seed;
    W.key1 = (uint32_t)(a->seed >> 32);
    W.any_order = a->precision != SCMC_PREC_FP64;
    const int64_t nout = Nv * Nv * nl_out;
    AccT *U = reinterpret_cast<AccT *>(c.acc_s.ensure(2 * nout * sizeof(AccT)));
    CK(cudaMemsetAsync(U, 0, 2 * nout * sizeof(AccT), st));
    int *counts = reinterpret_cast<int *>(c.fq_counts.ensure((Nz + 1) * sizeof(int)));
    int *offsets = reinterpret_cast<int *>(c.fq_offsets.ensure((Nz + 1) * sizeof(int)));
    int *cursor = reinterpret_cast<int *>(c.fq_cursor.ensure((Nz + 1) * sizeof(int)));
    int *planes = reinterpret_cast<int *>(c.fq_planes.ensure((Nz + 1) * sizeof(int)));
    std::vector<int> hcounts(Nz + 1);
    std::vector<int> hplanes;
    const int sms = sm_count(c.device);
    const scmc_tuning tune = tuning_for(SCMC_TUNE_FQ, a->precision, Nv * Nv);
    int64_t total_vert = 0;
    const int passes = a->do_cbs ? 2 : 1;
    // The pair form pipelines batches: the walk, the entries and the plane
    // sort of a batch run on `ps` (with entry buffers of their own parity)
    // while the previous batch's operands and products run on `st`; the host
    // plans a batch's plane groups meanwhile.  Other forms stay on `st`.
    const bool pipe = use_pair;
    cudaStream_t ps = st;
    int *d_err = reinterpret_cast<int *>(c.fq_err.ensure(sizeof(int)));
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    if (pipe) {
        c.make_aux();
        ps = c.aux;
        CK(cudaEventRecord(c.ev[4], st));  // accumulator, twiddles, tables
        CK(cudaStreamWaitEvent(ps, c.ev[4], 0));
    }
    cudaEvent_t *ev_prod = &c.ev[0], *ev_cons = &c.ev[2];  // per parity
    int64_t bi = 0;
    try {
        for (int64_t done = 0; done < a->max_itr; ++bi) {
            const int par = (int)(bi & 1);
            const int64_t nb = path_batch_size(a->max_itr - done, tune.path_batch);
            W.path_base = a->path_offset + (uint64_t)done;
            Batch B;
            if (pipe && bi >= 2) CK(cudaStreamWaitEvent(ps, ev_cons[par], 0));  // batch bi - 2 has read this parity's entries
            walk_batch(c, W, nb, ps, B);
            const int64_t nvert = B.n_paths + B.n_multi;
            total_vert += nvert;
            const int64_t nent = nvert * passes;
            if (nent > INT32_MAX) fail(SCMC_ERR_INVALID, "batch too large");
            // one output light on the pair form: 16-byte entries with the light factor applied
            const bool compact = use_pair && nl_out == 1 && Nx <= 65535;
            const size_t rec = compact ? sizeof(FqEntryC) : sizeof(FqEntry);
            DevBuf &ebuf = (pipe && par) ? c.rows2 : c.rows;
            char *Ein_b = reinterpret_cast<char *>(ebuf.ensure(2 * nent * rec));
            char *Es_b = Ein_b + nent * rec;
            FqEntry *Es = reinterpret_cast<FqEntry *>(Es_b);  // the full-entry forms
            CK(cudaMemsetAsync(counts, 0, (Nz + 1) * sizeof(int), ps));
            {
                StageScope sc(ST_ROWS, ps);
                const int eg = (int)std::min<int64_t>((nent + 255) / 256, (int64_t)sms * 16);
                if (compact)
                    fq_entries_kernel<true><<<eg, 256, 0, ps>>>(F, B.S, c.scap, B.M, c.mcap, B.n_paths, B.n_multi, Ein_b,
                                                                 counts);
                else
                    fq_entries_kernel<false><<<eg, 256, 0, ps>>>(F, B.S, c.scap, B.M, c.mcap, B.n_paths, B.n_multi, Ein_b,
                                                                  counts);
                CK(cudaGetLastError());
                LAUNCHED();
            }
            CK(cudaMemcpyAsync(hcounts.data(), counts, Nz * sizeof(int), cudaMemcpyDeviceToHost, ps));
            CK(cudaStreamSynchronize(ps));
            std::vector<int> hoff(Nz + 1, 0);
            hplanes.clear();
            for (int64_t k = 0; k < Nz; ++k) {
                hoff[k + 1] = hoff[k] + hcounts[k];
                if (hcounts[k] > 0 && k < Nz - 1) hplanes.push_back((int)k);
            }
            if (hplanes.empty()) {
                done += nb;
                continue;
            }
            CK(cudaMemcpyAsync(offsets, hoff.data(), (Nz + 1) * sizeof(int), cudaMemcpyHostToDevice, ps));
            CK(cudaMemcpyAsync(planes, hplanes.data(), hplanes.size() * sizeof(int), cudaMemcpyHostToDevice, ps));
            CK(cudaMemsetAsync(cursor, 0, (Nz + 1) * sizeof(int), ps));
            {
                StageScope sc(ST_ROWS, ps);
                const int sg = (int)std::min<int64_t>((nent + 255) / 256, (int64_t)sms * 16);
                if (compact)
                    fq_scatter_kernel<FqEntryC><<<sg, 256, 0, ps>>>(reinterpret_cast<const FqEntryC *>(Ein_b), nent, offsets,
                                                                    cursor, reinterpret_cast<FqEntryC *>(Es_b));
                else
                    fq_scatter_kernel<FqEntry><<<sg, 256, 0, ps>>>(reinterpret_cast<const FqEntry *>(Ein_b), nent, offsets,
                                                                   cursor, Es);
                CK(cudaGetLastError());
                LAUNCHED();
            }
            if (pipe) {
                CK(cudaEventRecord(ev_prod[par], ps));
                CK(cudaStreamWaitEvent(st, ev_prod[par], 0));
                CK(cudaEventSynchronize(ev_cons[par]));  // batch bi - 2's metadata copy out of fq_hmeta[par] is done
            }
            if (use_tc) {
                if (use_pair)
                    fq_tc_batch_pair(c, F, (int)nl_out, Es_b, compact, hcounts, hoff, hplanes, Tt, dz, drr, n_uniform,
                                     reinterpret_cast<double *>(U), a->precision == SCMC_PREC_MIXED, tune.group_entries,
                                     d_err, c.fq_hmeta[par], st);
                else
                    fq_tc_batch(c, F, (int)nl_out, Es, hcounts, hoff, hplanes, Tt, dz, drr, n_uniform,
                                reinterpret_cast<double *>(U), a->precision == SCMC_PREC_MIXED, tune.group_entries, st);
            } else {
                const int nvt = (int)((Nv + kFqTile - 1) / kFqTile);
                for (size_t p0 = 0; p0 < hplanes.size(); p0 += 65535) {
                    const unsigned gy = (unsigned)std::min<size_t>(65535, hplanes.size() - p0);
                    dim3 grid((unsigned)(nvt * nvt * nl_out), gy);
                    StageScope sc(ST_CONTRACT, st);
                    fq_accum_kernel<POL, AccT><<<grid, 256, 0, st>>>(F, Es, offsets, planes + p0, T, dz, U);
                    CK(cudaGetLastError());
                    LAUNCHED();
                }
            }
            if (pipe) CK(cudaEventRecord(ev_cons[par], st));
            else CK(cudaStreamSynchronize(st));  // host vectors above are reused next batch
            done += nb;
        }
    } catch (...) {
        // nothing of the failed solve stays in flight on either stream
        if (pipe) cudaStreamSynchronize(ps);
        cudaStreamSynchronize(st);
        throw;
    }
    {
        int herr = 0;  // a bounded wait of the pair form gave up somewhere in the solve
        CK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr) fail(SCMC_ERR_TIMEOUT, "tensor-core contraction: a bounded wait gave up");
    }
    const double V = bw[0] * bw[1] * bw[2];
    const double norm = total_vert > 0 ? std::sqrt(1.0 / (double)total_vert * V * sigt) : 0.0;  // lines 214, 302-303
    StageScope fin(ST_FINAL, st);
    const int fgrid = (int)std::max<int64_t>(1, std::min<int64_t>((nout + 255) / 256, 4096));
    if (use_tc)  // FP64 accumulator stored [light][r1][r2] ([light][r2][r1] by the pair form)
        fq_finalize_kernel<double><<<fgrid, 256, 0, st>>>(reinterpret_cast<const double *>(U), db, (int)Nv, (int)nl_out,
                                                          norm, d_u, use_pair ? 0 : 1);
    else
        fq_finalize_kernel<AccT><<<fgrid, 256, 0, st>>>(U, db, (int)Nv, (int)nl_out, norm, d_u, 0);
    CK(cudaGetLastError());
    LAUNCHED();
}

void fq_device_locked(Ctx &c, const scmc_fq_args *a, double *d_u, cudaStream_t st, const double *Wl = nullptr)
{
    CK(cudaSetDevice(a->device));
    double2 *u = reinterpret_cast<double2 *>(d_u);
    if (a->precision == SCMC_PREC_FP64) fq_run<P64, double>(c, a, Wl, u, st);
    else if (a->precision == SCMC_PREC_FP32) fq_run<P32, float>(c, a, Wl, u, st);
    else fq_run<PMIX, double>(c, a, Wl, u, st);
}

// ---------------------------------------------------------------------------
// packs of field requests (the request server): many small MCfield solves of
// one dimension and precision class, all on the CUDA-core accumulation, run
// as one walk, one accumulation and one finalisation launch per round of up
// to 2^20 paths instead of a launch sequence each.
// ---------------------------------------------------------------------------
struct PackItem {
    const scmc_mc_args *a;
    double *d_u;  // device output, 2*nv*nl doubles
};

__global__ void pack_bounds_kernel(const int64_t *__restrict__ moff, const int64_t *__restrict__ mcnt,
                                   const int64_t *__restrict__ prefix, int n_req, int64_t n_paths,
                                   int64_t *__restrict__ out)
{
    const int64_t total = n_paths > 0 ? moff[n_paths - 1] + mcnt[n_paths - 1] : 0;
    for (int r = threadIdx.x; r <= n_req; r += blockDim.x) out[r] = prefix[r] < n_paths ? moff[prefix[r]] : total;
}

// Host staging of the pack's read-only inputs (directions, tables), uploaded in one copy.
struct PackStage {
    std::vector<char> bytes;
    size_t put(const void *src, size_t n)
    {
        const size_t off = (bytes.size() + 255) & ~(size_t)255;
        bytes.resize(off + n);
        if (n) std::memcpy(bytes.data() + off, src, n);
        return off;
    }
};

template <int DIM, int POL, typename AccT>
void field_pack_run(Ctx &c, const std::vector<PackItem> &items, cudaStream_t st)
{
    const int K = (int)items.size();
    const int sms = sm_count(c.device);
    std::vector<Prepared> P(K);
    std::vector<PackTiling> tiling(K);
    PackStage sg;
    struct Offs {
        size_t l, v, vs, a0, i0, a1, i1;
    };
    std::vector<Offs> off(K);
    int64_t arena = 0;
    size_t smem = 0;
    using R = typename std::conditional<POL == P64, double, float>::type;
    using Cx = typename cplx_t<R>::type;
    for (int k = 0; k < K; ++k) {
        const scmc_mc_args *a = items[k].a;
        P[k] = host_params(a, 1);
        std::vector<double> hl(3 * a->nl, 0.0), hv(3 * a->nv, 0.0), hvs(3 * a->nv, 0.0);
        const double ff_sign = a->is_ff_v ? -1.0 : 1.0;  // MCfield.m:106
        for (int64_t j = 0; j < a->nl; ++j)
            for (int d = 0; d < DIM; ++d) hl[3 * j + d] = a->l[DIM * j + d];
        for (int64_t i = 0; i < a->nv; ++i)
            for (int d = 0; d < DIM; ++d) {
                hv[3 * i + d] = a->v[DIM * i + d];
                hvs[3 * i + d] = ff_sign * a->v[DIM * i + d];
            }
        Offs &o = off[k];
        o.l = sg.put(hl.data(), hl.size() * 8);
        o.v = sg.put(hv.data(), hv.size() * 8);
        o.vs = sg.put(hvs.data(), hvs.size() * 8);
        o.a0 = o.i0 = o.a1 = o.i1 = (size_t)-1;
        if (a->ampfunc.sct_type == SCMC_SCT_TABULATED) {
            o.a0 = sg.put(a->ampfunc.eval_amp, (size_t)a->ampfunc.table_n * sizeof(double2));
            o.i0 = sg.put(a->ampfunc.sample_icdf, (size_t)a->ampfunc.table_n * sizeof(double));
        }
        if (a->has_ampfunc0 && a->ampfunc0.sct_type == SCMC_SCT_TABULATED) {
            o.a1 = sg.put(a->ampfunc0.eval_amp, (size_t)a->ampfunc0.table_n * sizeof(double2));
            o.i1 = sg.put(a->ampfunc0.sample_icdf, (size_t)a->ampfunc0.table_n * sizeof(double));
        }
        PackTiling &t = tiling[k];
        const int nv = (int)a->nv, nl = (int)a->nl;
        t.tv = std::min(nv, 32);
        t.tl = std::min(nl, 32);
        while (t.tv * t.tl > kFieldMaxTile) t.tl /= 2;
        t.n_vtiles = (nv + t.tv - 1) / t.tv;
        t.acc_s = arena;
        t.acc_m = arena + 2 * (int64_t)nv * nl;
        arena += 4 * (int64_t)nv * nl;
        smem = std::max(smem, sizeof(Cx) * (2 * kFieldEB * (t.tv + t.tl) + kFieldEB) + sizeof(EventView) * kFieldEB + 16);
    }
    char *din = reinterpret_cast<char *>(c.wl.ensure(sg.bytes.size() + 256));
    CK(cudaMemcpyAsync(din, sg.bytes.data(), sg.bytes.size(), cudaMemcpyHostToDevice, st));
    auto dptr = [&](size_t o) { return o == (size_t)-1 ? nullptr : din + o; };
    for (int k = 0; k < K; ++k) {
        const Offs &o = off[k];
        set_tables(P[k], items[k].a, reinterpret_cast<const double2 *>(dptr(o.a0)),
                   reinterpret_cast<const double *>(dptr(o.i0)), reinterpret_cast<const double2 *>(dptr(o.a1)),
                   reinterpret_cast<const double *>(dptr(o.i1)));
        P[k].Q.l = reinterpret_cast<const double *>(din + o.l);
        P[k].Q.v = reinterpret_cast<const double *>(din + o.v);
        P[k].Q.vs = reinterpret_cast<const double *>(din + o.vs);
        P[k].W.any_order = 0;
    }
    AccT *acc = reinterpret_cast<AccT *>(c.acc_s.ensure((size_t)arena * sizeof(AccT)));
    CK(cudaMemsetAsync(acc, 0, (size_t)arena * sizeof(AccT), st));
    // per-pack device tables: NEE parameters, tiling, outputs, norms (fixed), then per round the walk
    // parameters, path prefix and jobs
    std::vector<NeeParams> hQ(K);
    std::vector<double> norms(K);
    std::vector<double2 *> outs(K);
    for (int k = 0; k < K; ++k) {
        const scmc_mc_args *a = items[k].a;
        hQ[k] = P[k].Q;
        const double m = (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
        norms[k] = m > 0 ? std::sqrt(1.0 / m * P[k].volume * a->sigt) : 0.0;  // MCfield.m:253-254
        outs[k] = reinterpret_cast<double2 *>(items[k].d_u);
    }
    PackStage fixed;
    const size_t oQ = fixed.put(hQ.data(), hQ.size() * sizeof(NeeParams));
    const size_t oT = fixed.put(tiling.data(), tiling.size() * sizeof(PackTiling));
    const size_t oN = fixed.put(norms.data(), norms.size() * sizeof(double));
    const size_t oO = fixed.put(outs.data(), outs.size() * sizeof(double2 *));
    char *dfix = reinterpret_cast<char *>(c.tiles.ensure(fixed.bytes.size() + 256));
    CK(cudaMemcpyAsync(dfix, fixed.bytes.data(), fixed.bytes.size(), cudaMemcpyHostToDevice, st));
    const NeeParams *dQ = reinterpret_cast<const NeeParams *>(dfix + oQ);
    const PackTiling *dT = reinterpret_cast<const PackTiling *>(dfix + oT);
    auto kacc = field_accum_packed_kernel<DIM, POL, AccT>;
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kacc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

    std::vector<int64_t> done(K, 0);
    const int64_t round_paths = (int64_t)1 << 20;
    for (;;) {
        // this round: every unfinished request gets an equal share of the round's paths
        int open = 0;
        for (int k = 0; k < K; ++k) open += done[k] < items[k].a->max_itr;
        if (!open) break;
        std::vector<WalkParams> hW(K);
        std::vector<int64_t> prefix(K + 1, 0);
        const int64_t share = std::max<int64_t>(1, round_paths / open);
        for (int k = 0; k < K; ++k) {
            const int64_t take = std::min<int64_t>(items[k].a->max_itr - done[k], share);
            hW[k] = P[k].W;
            hW[k].path_base = items[k].a->path_offset + (uint64_t)done[k];
            hW[k].n_paths = take;
            prefix[k + 1] = prefix[k] + take;
        }
        const int64_t n = prefix[K];
        PackStage rs;
        const size_t oW = rs.put(hW.data(), hW.size() * sizeof(WalkParams));
        const size_t oP = rs.put(prefix.data(), prefix.size() * sizeof(int64_t));
        char *drs = reinterpret_cast<char *>(c.out2.ensure(rs.bytes.size() + 256));
        CK(cudaMemcpyAsync(drs, rs.bytes.data(), rs.bytes.size(), cudaMemcpyHostToDevice, st));
        const WalkParams *dW = reinterpret_cast<const WalkParams *>(drs + oW);
        const int64_t *dP = reinterpret_cast<const int64_t *>(drs + oP);
        // pass 1: events per path, offsets of the multiple-scattering records
        c.counts.ensure(n * sizeof(int32_t));
        c.mcnt.ensure(n * sizeof(int64_t));
        c.moff.ensure((n + 1) * sizeof(int64_t));
        c.ctr.ensure(2 * sizeof(unsigned long long));
        c.err.ensure(sizeof(int));
        int64_t *dbounds = reinterpret_cast<int64_t *>(c.mcap_bounds.ensure((K + 1) * sizeof(int64_t)));
        unsigned long long *ctr = c.ctr.as<unsigned long long>();
        CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), st));
        CK(cudaMemsetAsync(c.err.p, 0, sizeof(int), st));
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 127) / 128, (int64_t)sms * 8));
        {
            StageScope sc(ST_WALK, st);
            walk_count_packed_kernel<DIM><<<grid, 128, 0, st>>>(dW, dP, K, n, c.counts.as<int32_t>(), ctr, c.err.as<int>());
            CK(cudaGetLastError());
            LAUNCHED();
        }
        count_to_multi_kernel<<<std::max(1, std::min(sms * 4, (int)((n + 255) / 256))), 256, 0, st>>>(
            c.counts.as<int32_t>(), n, c.mcnt.as<int64_t>());
        CK(cudaGetLastError());
        LAUNCHED();
        size_t tmp = 0;
        CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, c.mcnt.as<int64_t>(), c.moff.as<int64_t>(), n, st));
        c.scan_tmp.ensure(tmp);
        CK(cub::DeviceScan::ExclusiveSum(c.scan_tmp.p, tmp, c.mcnt.as<int64_t>(), c.moff.as<int64_t>(), n, st));
        LAUNCHED();
        pack_bounds_kernel<<<1, 256, 0, st>>>(c.moff.as<int64_t>(), c.mcnt.as<int64_t>(), dP, K, n, dbounds);
        CK(cudaGetLastError());
        LAUNCHED();
        std::vector<int64_t> mb(K + 1);
        int herr = 0;
        CK(cudaMemcpyAsync(mb.data(), dbounds, (K + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&herr, c.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr) fail(SCMC_ERR_LIMIT, "a path exceeded max_events_per_path");
        const int64_t n_multi = mb[K];
        // pass 2: records
        ensure_single_records(c, n);
        ensure_multi_records(c, n_multi);
        Batch B;
        batch_views(c, n, n_multi, B);
        CK(cudaMemsetAsync(ctr + 1, 0, sizeof(unsigned long long), st));
        {
            StageScope sc(ST_WALK, st);
            walk_record_packed_kernel<DIM><<<grid, 128, 0, st>>>(dW, dP, K, n, c.moff.as<int64_t>(), B.S, c.scap, B.M,
                                                                 c.mcap, ctr + 1);
            CK(cudaGetLastError());
            LAUNCHED();
        }
        prof_count(n, n + n_multi, 0.0);
        // one accumulation launch: jobs of (request, tile, event range, singles / multis)
        std::vector<PackJob> jobs;
        for (int k = 0; k < K; ++k) {
            const PackTiling &t = tiling[k];
            const int tiles = t.n_vtiles * (int)((items[k].a->nl + t.tl - 1) / t.tl);
            for (int single = 1; single >= 0; --single) {
                const int64_t e0 = single ? prefix[k] : mb[k], e1 = single ? prefix[k + 1] : mb[k + 1];
                const int64_t ne = e1 - e0;
                if (ne <= 0) continue;
                const int64_t ranges = std::max<int64_t>(1, (int64_t)sms * 6 / std::max(1, tiles * K));
                const int64_t per = std::max<int64_t>((int64_t)kFieldEB * 4, (ne + ranges - 1) / ranges);
                for (int tile = 0; tile < tiles; ++tile)
                    for (int64_t e = e0; e < e1; e += per)
                        jobs.push_back(PackJob{k, tile, single, 0, e, std::min(e1, e + per)});
            }
        }
        if (!jobs.empty()) {
            PackJob *dj = reinterpret_cast<PackJob *>(c.fq_planes.ensure(jobs.size() * sizeof(PackJob)));
            CK(cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(PackJob), cudaMemcpyHostToDevice, st));
            StageScope sc(ST_ROWS, st);
            kacc<<<(unsigned)jobs.size(), kFieldThreads, smem, st>>>(dQ, dT, dj, B.S, c.scap, B.M, c.mcap, acc);
            CK(cudaGetLastError());
            LAUNCHED();
        }
        CK(cudaStreamSynchronize(st));  // the host vectors of this round go out of scope
        for (int k = 0; k < K; ++k) done[k] += prefix[k + 1] - prefix[k];
    }
    int64_t nmax = 0;
    for (int k = 0; k < K; ++k) nmax = std::max<int64_t>(nmax, items[k].a->nv * items[k].a->nl);
    StageScope fin(ST_FINAL, st);
    field_finalize_packed_kernel<DIM, AccT><<<dim3((unsigned)std::max<int64_t>(1, std::min<int64_t>((nmax + 255) / 256, 64)),
                                                   (unsigned)K),
                                              256, 0, st>>>(dQ, dT, acc, reinterpret_cast<const double *>(dfix + oN),
                                                            reinterpret_cast<double2 *const *>(dfix + oO));
    CK(cudaGetLastError());
    LAUNCHED();
    CK(cudaStreamSynchronize(st));
}

// A pack's items must share dim and precision class and take the CUDA-core
// accumulation (use_field_tc false).
void field_pack_device(Ctx &c, const std::vector<PackItem> &items, cudaStream_t st)
{
    if (items.empty()) return;
    const scmc_mc_args *a = items[0].a;
    CK(cudaSetDevice(a->device));
    const bool mix = a->precision == SCMC_PREC_MIXED || a->precision == SCMC_PREC_FP16;
    if (a->dim == 3) {
        if (a->precision == SCMC_PREC_FP64) field_pack_run<3, P64, double>(c, items, st);
        else if (mix) field_pack_run<3, PMIX, double>(c, items, st);
        else field_pack_run<3, P32, float>(c, items, st);
    } else {
        if (a->precision == SCMC_PREC_FP64) field_pack_run<2, P64, double>(c, items, st);
        else if (mix) field_pack_run<2, PMIX, double>(c, items, st);
        else field_pack_run<2, P32, float>(c, items, st);
    }
}

// The precision class a request packs with (-1: never packed).
int pack_class(int kind, const scmc_mc_args &a, int64_t max_paths)
{
    if (kind != SCMC_REQ_FIELD || a.max_itr > max_paths || a.max_itr < 1 || use_field_tc(&a)) return -1;
    const int pol = a.precision == SCMC_PREC_FP64 ? 0 : (a.precision == SCMC_PREC_FP32 ? 2 : 1);
    return a.dim * 4 + pol;
}

#include "server.cuh"

}  // namespace

struct scmc_server {
    Server impl;
};

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int scmc_abi_version(void) { return SCMC_ABI_VERSION; }

const char *scmc_last_error(void) { return g_last_error.c_str(); }

int64_t scmc_launch_count(void) { return g_launches.load(); }

int scmc_tuning_set(const scmc_tuning *t)
{
    return guarded([&] {
        if (!t) fail(SCMC_ERR_INVALID, "null tuning entry");
        if (t->kind < SCMC_TUNE_FIELD || t->kind > SCMC_TUNE_FQ) fail(SCMC_ERR_INVALID, "invalid tuning kind");
        if (t->precision < 0 || t->precision > 3) fail(SCMC_ERR_INVALID, "invalid precision mode");
        if (t->stages != 0 && t->stages != 2 && t->stages != 3) fail(SCMC_ERR_INVALID, "stages must be 2 or 3");
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tuning_autoload_locked();
        g_tune.push_back(*t);
    });
}

int scmc_tuning_clear(void)
{
    return guarded([&] {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune.clear();
        g_tune_loaded = true;  // cleared on purpose: do not load the default file later
    });
}

int scmc_tuning_load(const char *path)
{
    return guarded([&] {
        if (!path) fail(SCMC_ERR_INVALID, "null path");
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_loaded = true;
        tuning_parse_file(path, true);
    });
}

int scmc_tuning_get(int32_t kind, int32_t precision, int64_t n, scmc_tuning *out)
{
    return guarded([&] {
        if (!out) fail(SCMC_ERR_INVALID, "null output");
        *out = tuning_for(kind, precision, n);
    });
}

int scmc_test_wait_fault(int32_t on)
{
    tc_test_fault().store(on ? 1 : 0);
    return SCMC_OK;
}

int scmc_field_device(const scmc_mc_args *args, double *d_u, void *stream)
{
    return guarded([&] {
        if (!d_u) fail(SCMC_ERR_INVALID, "null output");
        validate(args);
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        field_device_locked(c, args, d_u, st);
        CK(cudaStreamSynchronize(st));
    });
}

int scmc_field(const scmc_mc_args *args, double *u)
{
    return guarded([&] {
        validate(args);
        if (!u) fail(SCMC_ERR_INVALID, "null output");
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        const size_t bytes = (size_t)args->nv * args->nl * 2 * sizeof(double);
        double *d = reinterpret_cast<double *>(c.out0.ensure(bytes));
        field_device_locked(c, args, d, 0);
        CK(cudaMemcpy(u, d, bytes, cudaMemcpyDeviceToHost));
    });
}

int scmc_field_onwave_device(const scmc_mc_args *args, const double *Wl, double *d_u, void *stream)
{
    return guarded([&] {
        if (!d_u) fail(SCMC_ERR_INVALID, "null output");
        validate(args);
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        onwave_device_locked(c, args, Wl, d_u, st);
        CK(cudaStreamSynchronize(st));
    });
}

int scmc_field_onwave(const scmc_mc_args *args, const double *Wl, double *u)
{
    return guarded([&] {
        validate(args);
        if (!u) fail(SCMC_ERR_INVALID, "null output");
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        const size_t bytes = (size_t)args->nv * 2 * sizeof(double);
        double *d = reinterpret_cast<double *>(c.out0.ensure(bytes));
        onwave_device_locked(c, args, Wl, d, 0);
        CK(cudaMemcpy(u, d, bytes, cudaMemcpyDeviceToHost));
    });
}

int scmc_cov_device(const scmc_mc_args *args, double *d_Ms, double *d_Mm, void *stream)
{
    return guarded([&] {
        validate(args);
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        cov_device_locked(c, args, d_Ms, d_Mm, st);
        CK(cudaStreamSynchronize(st));
    });
}

int scmc_cov(const scmc_mc_args *args, double *Ms, double *Mm)
{
    return guarded([&] {
        validate(args);
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        const size_t bytes = (size_t)args->nv * args->nv * args->nl * args->nl * 2 * sizeof(double);
        double *d0 = Ms ? reinterpret_cast<double *>(c.out0.ensure(bytes)) : nullptr;
        double *d1 = Mm ? reinterpret_cast<double *>(c.out1.ensure(bytes)) : nullptr;
        cov_device_locked(c, args, d0, d1, 0);
        if (Ms) CK(cudaMemcpy(Ms, d0, bytes, cudaMemcpyDeviceToHost));
        if (Mm) CK(cudaMemcpy(Mm, d1, bytes, cudaMemcpyDeviceToHost));
    });
}

int scmc_fq_grid_size(double v_max, double v_stp, int64_t *nv0)
{
    return guarded([&] {
        if (!nv0) fail(SCMC_ERR_INVALID, "null output");
        if (!(v_stp > 0) || !(v_max >= 0)) fail(SCMC_ERR_INVALID, "v_max must be >= 0 and v_stp > 0");
        *nv0 = colon_count(-v_max, v_stp, v_max);
    });
}

int scmc_field_fourier_quad_device(const scmc_fq_args *args, double *d_u, void *stream)
{
    return guarded([&] {
        validate_fq(args);
        if (!d_u) fail(SCMC_ERR_INVALID, "null output");
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        fq_device_locked(c, args, d_u, st);
        CK(cudaStreamSynchronize(st));
    });
}

int scmc_field_fourier_quad(const scmc_fq_args *args, double *u)
{
    return guarded([&] {
        validate_fq(args);
        if (!u) fail(SCMC_ERR_INVALID, "null output");
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        const int64_t nv0 = colon_count(-args->v_max, args->v_stp, args->v_max);
        const size_t bytes = (size_t)nv0 * nv0 * args->nl * 2 * sizeof(double);
        double *d = reinterpret_cast<double *>(c.out0.ensure(bytes));
        fq_device_locked(c, args, d, 0);
        CK(cudaMemcpy(u, d, bytes, cudaMemcpyDeviceToHost));
    });
}

int scmc_field_fourier_quad_onwave_device(const scmc_fq_args *args, const double *Wl, double *d_u, void *stream)
{
    return guarded([&] {
        validate_fq(args);
        if (!d_u || !Wl) fail(SCMC_ERR_INVALID, "null output or weights");
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        fq_device_locked(c, args, d_u, st, Wl);
        CK(cudaStreamSynchronize(st));
    });
}

int scmc_field_fourier_quad_onwave(const scmc_fq_args *args, const double *Wl, double *u)
{
    return guarded([&] {
        validate_fq(args);
        if (!u || !Wl) fail(SCMC_ERR_INVALID, "null output or weights");
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        const int64_t nv0 = colon_count(-args->v_max, args->v_stp, args->v_max);
        const size_t bytes = (size_t)nv0 * nv0 * 2 * sizeof(double);
        double *d = reinterpret_cast<double *>(c.out0.ensure(bytes));
        fq_device_locked(c, args, d, 0, Wl);
        CK(cudaMemcpy(u, d, bytes, cudaMemcpyDeviceToHost));
    });
}

int scmc_cov_hetero(const scmc_hetero_args *args, double *Ms, double *Mm, double *mean1)
{
    return guarded([&] {
        if (!args) fail(SCMC_ERR_INVALID, "null arguments");
        validate(&args->mc);
        Ctx &c = context(args->mc.device);
        std::lock_guard<std::mutex> lk(c.mu);
        const size_t bytes = (size_t)args->mc.nv * args->mc.nv * args->mc.nl * args->mc.nl * 2 * sizeof(double);
        const size_t b1 = (size_t)args->mc.nv * args->mc.nl * 2 * sizeof(double);
        double *d0 = Ms ? reinterpret_cast<double *>(c.out0.ensure(bytes)) : nullptr;
        double *d1 = Mm ? reinterpret_cast<double *>(c.out1.ensure(bytes)) : nullptr;
        double *d2 = mean1 ? reinterpret_cast<double *>(c.out2.ensure(b1)) : nullptr;
        cov_hetero_locked(c, args, d0, d1, d2, 0);
        if (Ms) CK(cudaMemcpy(Ms, d0, bytes, cudaMemcpyDeviceToHost));
        if (Mm) CK(cudaMemcpy(Mm, d1, bytes, cudaMemcpyDeviceToHost));
        if (mean1) CK(cudaMemcpy(mean1, d2, b1, cudaMemcpyDeviceToHost));
    });
}

int scmc_field_hetero(const scmc_hetero_args *args, double *u)
{
    return guarded([&] {
        if (!args || !u) fail(SCMC_ERR_INVALID, "null arguments");
        validate(&args->mc);
        Ctx &c = context(args->mc.device);
        std::lock_guard<std::mutex> lk(c.mu);
        const size_t bytes = (size_t)args->mc.nv * args->mc.nl * 2 * sizeof(double);
        double *d = reinterpret_cast<double *>(c.out0.ensure(bytes));
        field_hetero_locked(c, args, d, 0);
        CK(cudaMemcpy(u, d, bytes, cudaMemcpyDeviceToHost));
    });
}

int scmc_cov_hetero_device(const scmc_hetero_args *args, double *d_Ms, double *d_Mm, double *d_mean1, void *stream)
{
    return guarded([&] {
        if (!args) fail(SCMC_ERR_INVALID, "null arguments");
        validate(&args->mc);
        Ctx &c = context(args->mc.device);
        std::lock_guard<std::mutex> lk(c.mu);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        cov_hetero_locked(c, args, d_Ms, d_Mm, d_mean1, st);
        CK(cudaStreamSynchronize(st));
    });
}

int scmc_field_hetero_device(const scmc_hetero_args *args, double *d_u, void *stream)
{
    return guarded([&] {
        if (!args || !d_u) fail(SCMC_ERR_INVALID, "null arguments");
        validate(&args->mc);
        Ctx &c = context(args->mc.device);
        std::lock_guard<std::mutex> lk(c.mu);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        field_hetero_locked(c, args, d_u, st);
        CK(cudaStreamSynchronize(st));
    });
}

int scmc_profile_enable(int32_t on)
{
    return guarded([&] {
        std::lock_guard<std::mutex> lk(g_prof.mu);
        if (on && !g_prof.on.load()) {
            // time origin of the launch intervals: recorded now on the legacy stream
            if (g_prof.ref) CK(cudaEventDestroy(g_prof.ref));
            g_prof.ref = nullptr;
            g_prof.resolve_locked();
            CK(cudaEventCreate(&g_prof.ref));
            CK(cudaEventRecord(g_prof.ref, 0));
        }
        g_prof.on.store(on != 0);
    });
}

int scmc_profile_read(scmc_stage_times *out, int32_t reset)
{
    return guarded([&] {
        if (!out) fail(SCMC_ERR_INVALID, "null output");
        std::lock_guard<std::mutex> lk(g_prof.mu);
        g_prof.resolve_locked();
        out->walk_launches = g_prof.launches[ST_WALK];
        out->walk_ms = g_prof.ms[ST_WALK];
        out->rows_launches = g_prof.launches[ST_ROWS];
        out->rows_ms = g_prof.ms[ST_ROWS];
        out->contract_launches = g_prof.launches[ST_CONTRACT];
        out->contract_ms = g_prof.ms[ST_CONTRACT];
        out->finalize_launches = g_prof.launches[ST_FINAL];
        out->finalize_ms = g_prof.ms[ST_FINAL];
        out->paths = g_prof.paths;
        out->events = g_prof.events;
        out->contract_flops = g_prof.flops;
        out->contract_busy_ms = g_prof.busy_ms(ST_CONTRACT);
        out->rows_busy_ms = g_prof.busy_ms(ST_ROWS);
        if (reset) {
            for (int k = 0; k < 4; ++k) {
                g_prof.launches[k] = 0;
                g_prof.ms[k] = 0;
                g_prof.iv[k].clear();
            }
            g_prof.paths = g_prof.events = 0;
            g_prof.flops = 0;
        }
    });
}

int scmc_export_records(const scmc_mc_args *args, int32_t want_phase, int64_t capacity, double *x, double *ow,
                        double *x1, double *w1, double *wpx, double *xi, int32_t *plen, int64_t *path,
                        int64_t *n_events)
{
    return guarded([&] {
        if (!n_events) fail(SCMC_ERR_INVALID, "null n_events");
        export_records(args, want_phase, capacity, x, ow, x1, w1, wpx, xi, plen, path, n_events);
    });
}

int scmc_philox_stream(uint64_t seed, uint64_t path, int32_t tag, int64_t n, double *out)
{
    return guarded([&] {
        if (n < 0 || (n > 0 && !out)) fail(SCMC_ERR_INVALID, "invalid output");
        if (n == 0) return;
        context(0);
        CK(cudaSetDevice(0));
        double *d = nullptr;
        CK(cudaMalloc(&d, n * sizeof(double)));
        philox_stream_kernel<<<1, 1>>>(seed, path, tag, n, d);
        cudaError_t e = cudaGetLastError();
        LAUNCHED();
        if (e == cudaSuccess) e = cudaMemcpy(out, d, n * sizeof(double), cudaMemcpyDeviceToHost);
        cudaFree(d);
        CK(e);
    });
}

// ---------------------------------------------------------------------------
// field from stored path records (replay on any machine)
// ---------------------------------------------------------------------------
int scmc_field_from_records(const scmc_mc_args *args, int64_t n, const double *x, const double *ow, const double *x1,
                            const double *w1, const double *wpx, const double *xi, const int32_t *plen,
                            const int64_t *path, double *u)
{
    return guarded([&] {
        validate(args);
        if (n < 0 || (n > 0 && (!x || !ow || !x1 || !w1 || !wpx || !xi || !plen || !path)) || !u)
            fail(SCMC_ERR_INVALID, "invalid records");
        // singles (pL == 1) index the paths; multis point at their path's single
        std::unordered_map<int64_t, int32_t> first;
        int64_t ns = 0, nm = 0;
        for (int64_t e = 0; e < n; ++e) {
            if (plen[e] == 1) {
                if (!first.emplace(path[e], (int32_t)ns).second) fail(SCMC_ERR_INVALID, "a path has two first events");
                ++ns;
            } else if (plen[e] > 1) {
                ++nm;
            } else {
                fail(SCMC_ERR_INVALID, "event with pL < 1");
            }
        }
        if (ns > INT32_MAX) fail(SCMC_ERR_INVALID, "too many paths in one record set");
        std::vector<double> sx1(3 * ns), sw1(3 * ns), swpx(ns), sxi(ns);
        std::vector<int32_t> snev(ns, 1);
        std::vector<double> mx(3 * std::max<int64_t>(nm, 1)), mow(3 * std::max<int64_t>(nm, 1)), mwpx(nm), mxi(nm);
        std::vector<int32_t> mpath(nm), mplen(nm);
        int64_t is = 0, im = 0;
        for (int64_t e = 0; e < n; ++e) {
            if (plen[e] == 1) {
                for (int d = 0; d < 3; ++d) {
                    sx1[d * ns + is] = x1[3 * e + d];
                    sw1[d * ns + is] = w1[3 * e + d];
                }
                swpx[is] = wpx[e];
                sxi[is] = xi[e];
                ++is;
            } else {
                auto it = first.find(path[e]);
                if (it == first.end()) fail(SCMC_ERR_INVALID, "a record's path has no first event");
                for (int d = 0; d < 3; ++d) {
                    mx[d * nm + im] = x[3 * e + d];
                    mow[d * nm + im] = ow[3 * e + d];
                }
                mwpx[im] = wpx[e];
                mxi[im] = xi[e];
                mpath[im] = it->second;
                mplen[im] = plen[e];
                ++snev[it->second];
                ++im;
            }
        }
        Ctx &c = context(args->device);
        std::lock_guard<std::mutex> lk(c.mu);
        CK(cudaSetDevice(args->device));
        cudaStream_t st = 0;
        Prepared P = prepare(c, args, 1, st);
        const int64_t scap = std::max<int64_t>(ns, 1), mcap = std::max<int64_t>(nm, 1);
        auto up = [&](DevBuf &b, const void *h, size_t bytes, size_t cap_bytes) {
            b.ensure(cap_bytes);
            if (bytes) CK(cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice));
        };
        up(c.s_x1, sx1.data(), 3 * ns * 8, 3 * scap * 8);
        up(c.s_w1, sw1.data(), 3 * ns * 8, 3 * scap * 8);
        up(c.s_wpx, swpx.data(), ns * 8, scap * 8);
        up(c.s_xi, sxi.data(), ns * 8, scap * 8);
        up(c.s_nev, snev.data(), ns * 4, scap * 4);
        up(c.m_x, mx.data(), 3 * nm * 8, 3 * mcap * 8);
        up(c.m_ow, mow.data(), 3 * nm * 8, 3 * mcap * 8);
        up(c.m_wpx, mwpx.data(), nm * 8, mcap * 8);
        up(c.m_xi, mxi.data(), nm * 8, mcap * 8);
        up(c.m_path, mpath.data(), nm * 4, mcap * 4);
        up(c.m_plen, mplen.data(), nm * 4, mcap * 4);
        // strides of the uploaded layout; the walk re-sizes these if it needs more
        c.scap = ns;
        c.mcap = nm;
        Batch B;
        B.S = SingleRec{c.s_x1.as<double>(), c.s_w1.as<double>(), c.s_wpx.as<double>(), c.s_xi.as<double>(),
                        c.s_nev.as<int32_t>()};
        B.M = MultiRec{c.m_x.as<double>(), c.m_ow.as<double>(), c.m_wpx.as<double>(), c.m_xi.as<double>(),
                       c.m_path.as<int32_t>(), c.m_plen.as<int32_t>()};
        B.n_paths = ns;
        B.n_multi = nm;
        const int64_t nq = args->nv * args->nl;
        double2 *d = reinterpret_cast<double2 *>(c.out0.ensure(nq * sizeof(double2)));
        auto run = [&](auto dimc, auto polc, auto acc) {
            constexpr int DIM = decltype(dimc)::value;
            constexpr int POL = decltype(polc)::value;
            using AccT = decltype(acc);
            AccT *Us = reinterpret_cast<AccT *>(c.acc_s.ensure(2 * nq * sizeof(AccT)));
            AccT *Um = reinterpret_cast<AccT *>(c.acc_m.ensure(2 * nq * sizeof(AccT)));
            CK(cudaMemsetAsync(Us, 0, 2 * nq * sizeof(AccT), st));
            CK(cudaMemsetAsync(Um, 0, 2 * nq * sizeof(AccT), st));
            launch_field_accum<DIM, POL, true, AccT>(c, P, B, Us, ns, st);
            launch_field_accum<DIM, POL, false, AccT>(c, P, B, Um, nm, st);
            const double m = (double)(args->norm_itr > 0 ? args->norm_itr : args->max_itr);
            const double norm = m > 0 ? std::sqrt(1.0 / m * P.volume * args->sigt) : 0.0;  // MCfield.m:253-254
            field_finalize_kernel<DIM, AccT><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((nq + 255) / 256, 1024)),
                                               256, 0, st>>>(P.Q, Us, Um, norm, d);
            CK(cudaGetLastError());
            LAUNCHED();
        };
        using I3 = std::integral_constant<int, 3>;
        using I2 = std::integral_constant<int, 2>;
        using F64 = std::integral_constant<int, P64>;
        using FMX = std::integral_constant<int, PMIX>;
        using F32 = std::integral_constant<int, P32>;
        if (args->dim == 3) {
            if (args->precision == SCMC_PREC_FP64) run(I3{}, F64{}, double{});
            else if (args->precision == SCMC_PREC_FP32) run(I3{}, F32{}, float{});
            else run(I3{}, FMX{}, double{});
        } else {
            if (args->precision == SCMC_PREC_FP64) run(I2{}, F64{}, double{});
            else if (args->precision == SCMC_PREC_FP32) run(I2{}, F32{}, float{});
            else run(I2{}, FMX{}, double{});
        }
        CK(cudaMemcpy(u, d, nq * sizeof(double2), cudaMemcpyDeviceToHost));
    });
}

// ---------------------------------------------------------------------------
// post-processing: refocus, samples from a covariance
// ---------------------------------------------------------------------------
static int64_t pp_colon(double a, double st, double b)
{
    if (st == 0 || (st > 0 && a > b) || (st < 0 && a < b)) return 0;
    const double q = (b - a) / st;
    return (int64_t)std::floor(q + 1e-10 * std::fmax(1.0, std::fabs(q))) + 1;
}

int scmc_refocus_grid(int32_t dim, const double *box_min, const double *box_max, const double *box_stp,
                      int64_t *dims, int64_t *n)
{
    return guarded([&] {
        if ((dim != 2 && dim != 3) || !box_min || !box_max || !box_stp || !dims || !n)
            fail(SCMC_ERR_INVALID, "invalid refocus grid");
        int64_t t = 1;
        for (int k = 0; k < dim; ++k) {
            dims[k] = pp_colon(box_min[k], box_stp[k], box_max[k]);
            t *= dims[k];
        }
        *n = t;
    });
}

int scmc_refocus(const double *u, const double *v, int64_t nv, int32_t dim, const double *l, const double *box_min,
                 const double *box_max, const double *box_stp, double lambda, int32_t as_written, int32_t precision,
                 int32_t device, double *rU)
{
    return guarded([&] {
        if ((dim != 2 && dim != 3) || nv < 1 || !u || !v || !l || !box_min || !box_max || !box_stp || !rU)
            fail(SCMC_ERR_INVALID, "invalid refocus arguments");
        if (!(lambda > 0)) fail(SCMC_ERR_INVALID, "lambda must be positive");
        if (precision != SCMC_PREC_FP64 && precision != SCMC_PREC_MIXED)
            fail(SCMC_ERR_INVALID, "refocus runs in FP64 or MIXED precision");
        RefocusGrid G{};
        G.dim = dim;
        int64_t N = 1;
        for (int k = 0; k < 3; ++k) {
            G.n[k] = k < dim ? pp_colon(box_min[k], box_stp[k], box_max[k]) : 1;
            G.bmin[k] = k < dim ? box_min[k] : 0.0;
            G.stp[k] = k < dim ? box_stp[k] : 0.0;
            N *= G.n[k];
        }
        if (N < 1) fail(SCMC_ERR_INVALID, "empty refocus grid");
        Ctx &c = context(device);
        std::lock_guard<std::mutex> lk(c.mu);
        CK(cudaSetDevice(device));
        double2 *du = reinterpret_cast<double2 *>(c.out1.ensure(nv * sizeof(double2)));
        double *dv = reinterpret_cast<double *>(c.dirs_v.ensure(dim * nv * sizeof(double)));
        double2 *dr = reinterpret_cast<double2 *>(c.out0.ensure(N * sizeof(double2)));
        CK(cudaMemcpy(du, u, nv * sizeof(double2), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dv, v, dim * nv * sizeof(double), cudaMemcpyHostToDevice));
        const double kw = 2 * SCMC_PI / lambda;
        const double l2 = dim == 3 ? l[2] : 0.0;
        const unsigned grid = (unsigned)((N + 255) / 256);
        {
            StageScope sc(ST_CONTRACT, 0);
            if (precision == SCMC_PREC_MIXED)
                refocus_kernel<true><<<grid, 256>>>(G, du, dv, nv, l[0], l[1], l2, kw, as_written, dr);
            else
                refocus_kernel<false><<<grid, 256>>>(G, du, dv, nv, l[0], l[1], l2, kw, as_written, dr);
            CK(cudaGetLastError());
            LAUNCHED();
        }
        CK(cudaMemcpy(rU, dr, N * sizeof(double2), cudaMemcpyDeviceToHost));
    });
}

int scmc_sample_cov(const double *C, int64_t N, int64_t n_samples, uint64_t seed, int32_t device, double *Z)
{
    return guarded([&] {
        if (!C || !Z || N < 1 || n_samples < 0) fail(SCMC_ERR_INVALID, "invalid sampling arguments");
        if (N > 32768) fail(SCMC_ERR_INVALID, "covariance too large to factorise (N <= 32768)");
        if (n_samples == 0) return;
        Ctx &c = context(device);
        std::lock_guard<std::mutex> lk(c.mu);
        CK(cudaSetDevice(device));
        const int64_t n = 2 * N;
        double2 *dC = reinterpret_cast<double2 *>(c.acc_m.ensure(N * N * sizeof(double2)));
        double *S = reinterpret_cast<double *>(c.acc_s.ensure(n * n * sizeof(double)));
        double *g = reinterpret_cast<double *>(c.rows.ensure(n * n_samples * sizeof(double)));
        double2 *dZ = reinterpret_cast<double2 *>(c.out0.ensure(N * n_samples * sizeof(double2)));
        int *err = reinterpret_cast<int *>(c.err.ensure(sizeof(int)));
        CK(cudaMemcpy(dC, C, N * N * sizeof(double2), cudaMemcpyHostToDevice));
        CK(cudaMemset(err, 0, sizeof(int)));
        const int sms = sm_count(device);
        sigma_build_kernel<<<sms * 8, 256>>>(dC, N, S);
        CK(cudaGetLastError());
        LAUNCHED();
        {
            StageScope sc(ST_CONTRACT, 0);
            for (int64_t k0 = 0; k0 < n; k0 += kCholNB) {
                const int nb = (int)std::min<int64_t>(kCholNB, n - k0);
                chol_diag_kernel<<<1, 256>>>(S, n, k0, nb, err);
                LAUNCHED();
                const int64_t rest = n - k0 - nb;
                if (rest <= 0) break;
                chol_panel_kernel<<<(unsigned)((rest + 127) / 128), 128>>>(S, n, k0, nb);
                LAUNCHED();
                const int64_t nt = (rest + kCholNB - 1) / kCholNB;
                chol_update_kernel<<<(unsigned)(nt * (nt + 1) / 2), 256>>>(S, n, k0, nb);
                LAUNCHED();
            }
            CK(cudaGetLastError());
        }
        int herr = 0;
        CK(cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) fail(SCMC_ERR_INVALID, "Sigma is not positive definite (a covariance of too few paths is singular)");
        normals_kernel<<<sms * 8, 256>>>((uint32_t)seed, (uint32_t)(seed >> 32), n_samples, n, g);
        CK(cudaGetLastError());
        LAUNCHED();
        sample_product_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((N * n_samples + 255) / 256, sms * 32)),
                                256>>>(S, N, n_samples, g, dZ);
        CK(cudaGetLastError());
        LAUNCHED();
        CK(cudaMemcpy(Z, dZ, N * n_samples * sizeof(double2), cudaMemcpyDeviceToHost));
    });
}

// ---------------------------------------------------------------------------
// memory-effect view: means of a covariance over equal view / light offsets
// ---------------------------------------------------------------------------
static void offsets_run(Ctx &c, const double *d_C1, const double *d_C2, const OffsetGrid &g, float *d_R,
                        cudaStream_t st)
{
    const int nv = g.nvx * g.nvy, nl = g.nlx * g.nly;
    const int64_t nvo = (int64_t)(2 * g.nvx - 1) * (2 * g.nvy - 1);
    const int64_t nlo = (int64_t)(2 * g.nlx - 1) * (2 * g.nly - 1);
    const size_t smem = (size_t)nvo * sizeof(double2);
    if (smem > 200 * 1024) fail(SCMC_ERR_INVALID, "view grid too large for the offset reduction");
    double2 *sums = reinterpret_cast<double2 *>(c.offs.ensure((size_t)nvo * nlo * sizeof(double2)));
    CK(cudaMemsetAsync(sums, 0, (size_t)nvo * nlo * sizeof(double2), st));
    if (smem > 48 * 1024)
        CK(cudaFuncSetAttribute(offsets_sum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {
        StageScope sc(ST_FINAL, st);
        offsets_sum_kernel<<<(unsigned)((int64_t)nl * nl), 256, smem, st>>>(
            reinterpret_cast<const double2 *>(d_C1), reinterpret_cast<const double2 *>(d_C2), g, sums);
        CK(cudaGetLastError());
        LAUNCHED();
        offsets_finalize_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((nvo * nlo + 255) / 256, 4096)), 256, 0,
                                  st>>>(sums, g, reinterpret_cast<float2 *>(d_R));
        CK(cudaGetLastError());
        LAUNCHED();
    }
    (void)nv;
}

static OffsetGrid offsets_grid(int32_t nvx, int32_t nvy, int32_t nlx, int32_t nly)
{
    if (nvx < 1 || nvy < 1 || nlx < 1 || nly < 1) fail(SCMC_ERR_INVALID, "grid sizes must be positive");
    if ((int64_t)nvx * nvy > 65536 || (int64_t)nlx * nly > 65536) fail(SCMC_ERR_INVALID, "grid too large");
    return OffsetGrid{nvx, nvy, nlx, nly};
}

int scmc_cov_offsets_device(const double *d_C1, const double *d_C2, int32_t nvx, int32_t nvy, int32_t nlx,
                            int32_t nly, float *d_R, int32_t device, void *stream)
{
    return guarded([&] {
        if (!d_C1 || !d_R) fail(SCMC_ERR_INVALID, "null covariance or output");
        const OffsetGrid g = offsets_grid(nvx, nvy, nlx, nly);
        Ctx &c = context(device);
        std::lock_guard<std::mutex> lk(c.mu);
        CK(cudaSetDevice(device));
        offsets_run(c, d_C1, d_C2, g, d_R, reinterpret_cast<cudaStream_t>(stream));
    });
}

int scmc_cov_offsets(const double *C1, const double *C2, int32_t nvx, int32_t nvy, int32_t nlx, int32_t nly,
                     float *R, int32_t device)
{
    return guarded([&] {
        if (!C1 || !R) fail(SCMC_ERR_INVALID, "null covariance or output");
        const OffsetGrid g = offsets_grid(nvx, nvy, nlx, nly);
        Ctx &c = context(device);
        std::lock_guard<std::mutex> lk(c.mu);
        CK(cudaSetDevice(device));
        const int64_t nv = (int64_t)nvx * nvy, nl = (int64_t)nlx * nly;
        const size_t cb = (size_t)nv * nv * nl * nl * sizeof(double2);
        const int64_t nout = (int64_t)(2 * nvx - 1) * (2 * nvy - 1) * (2 * nlx - 1) * (2 * nly - 1);
        double *d1 = reinterpret_cast<double *>(c.acc_s.ensure(cb));
        double *d2 = C2 ? reinterpret_cast<double *>(c.acc_m.ensure(cb)) : nullptr;
        float *dR = reinterpret_cast<float *>(c.out0.ensure((size_t)nout * sizeof(float2)));
        CK(cudaMemcpy(d1, C1, cb, cudaMemcpyHostToDevice));
        if (C2) CK(cudaMemcpy(d2, C2, cb, cudaMemcpyHostToDevice));
        offsets_run(c, d1, d2, g, dR, 0);
        CK(cudaMemcpy(R, dR, (size_t)nout * sizeof(float2), cudaMemcpyDeviceToHost));
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// scmc_field_noalloc: the field path with every piece of device scratch in a
// fixed, file-scope device array instead of allocated memory.
//
// Some callers cannot allocate device memory while they call in: a host that
// runs under a pre-reserved memory budget (a serving process that sized its
// pools at start-up), a real-time caller that must not take the allocator's
// locks or let cudaFree synchronise the device, or an embedding runtime that
// forbids cudaMalloc/cudaFree on its threads.  This entry point serves them:
// it calls no cudaMalloc, cudaFree or allocating library routine; the caller
// passes the inputs (host struct) and the output (device memory).
//
// Limits (SCMC_ERR_INVALID beyond them): nv*nl <= 65536, each tabulated
// table <= 16384 entries, and no single path may have more scattering events
// than the scratch holds (~400k).  The scratch is 32 MiB per device and stays
// resident in every GPU that loads the library until the process exits.
// Every call shares it and it keeps the previous call's contents: the
// accumulators and counters are cleared at the start of each call.  Two calls
// whose work overlapped on the GPU would race on the array, so calls on one
// device are serialised: a per-device lock is held until the call's work on
// its stream has finished, on an error return too.  The accumulation is
// always the CUDA-core one (field_accum_kernel); in MIXED / FP16 mode with
// nv >= 64 and nl >= 32 scmc_field_device uses the tensor-core form instead,
// so there the two agree to the mixed tolerance, not bit for bit.
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture.
// ---------------------------------------------------------------------------
static constexpr size_t kFieldScratchBytes = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_field_scratch[kFieldScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_call_mu[kMaxDevices];  // one per device: calls on different GPUs run concurrently

unsigned char *field_scratch(int device)
{
    if (device < 0 || device >= kMaxDevices) fail(SCMC_ERR_INVALID, "invalid device ordinal");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_field_scratch));
        g_scratch_addr[device] = p;
    }
    return reinterpret_cast<unsigned char *>(g_scratch_addr[device]);
}

// [dim][n] column-major -> [n][3] (zero-padded), optionally also sign * the same.
__global__ void pack_dirs_kernel(const double *raw, int n, int dim, double sign, double *out, double *out_signed)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) {
            double x = k < dim ? raw[dim * j + k] : 0.0;
            out[3 * j + k] = x;
            if (out_signed) out_signed[3 * j + k] = sign * x;
        }
}

struct ScratchCarve {
    unsigned char *base;
    size_t off = 0, cap;
    template <typename T> T *take(size_t n)
    {
        off = (off + 255) & ~(size_t)255;
        T *p = reinterpret_cast<T *>(base + off);
        off += n * sizeof(T);
        if (off > cap) fail(SCMC_ERR_INVALID, "inputs exceed the fixed scratch of scmc_field_noalloc");
        return p;
    }
    size_t left() const { return cap > off ? cap - off : 0; }
};

constexpr int32_t kNoallocMaxTable = 16384;

// A tabulated function's evalAmp / sampleIcdf copied into the scratch.
void noalloc_table(const scmc_phase_function &pf, ScratchCarve &sc, cudaStream_t st, const double2 **amp,
                   const double **icdf)
{
    *amp = nullptr;
    *icdf = nullptr;
    if (pf.sct_type != SCMC_SCT_TABULATED) return;
    if (pf.table_n > kNoallocMaxTable)
        fail(SCMC_ERR_INVALID, "scmc_field_noalloc: tabulated tables are limited to 16384 entries");
    double2 *a = sc.take<double2>(pf.table_n);
    double *c = sc.take<double>(pf.table_n);
    CK(cudaMemcpyAsync(a, pf.eval_amp, pf.table_n * sizeof(double2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c, pf.sample_icdf, pf.table_n * sizeof(double), cudaMemcpyHostToDevice, st));
    *amp = a;
    *icdf = c;
}

template <int DIM, int POL, typename AccT>
void field_noalloc_run(const scmc_mc_args *a, double2 *d_u, cudaStream_t st)
{
    const int dim = DIM;
    ScratchCarve sc{field_scratch(a->device)};
    sc.cap = kFieldScratchBytes;
    const int nv = (int)a->nv, nl = (int)a->nl;

    // parameters as prepare() builds them, with the inputs placed in scratch
    Prepared P = host_params(a, 1);
    const double2 *amp0, *amp1 = nullptr;
    const double *icdf0, *icdf1 = nullptr;
    noalloc_table(a->ampfunc, sc, st, &amp0, &icdf0);
    if (a->has_ampfunc0) noalloc_table(a->ampfunc0, sc, st, &amp1, &icdf1);
    set_tables(P, a, amp0, icdf0, amp1, icdf1);
    WalkParams W = P.W;
    const NeeParams &Q = P.Q;

    // raw dim x n inputs into scratch, then packed to [n][3] on the device
    double *raw_l = sc.take<double>((size_t)dim * nl), *raw_v = sc.take<double>((size_t)dim * nv);
    CK(cudaMemcpyAsync(raw_l, a->l, (size_t)dim * nl * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(raw_v, a->v, (size_t)dim * nv * 8, cudaMemcpyHostToDevice, st));
    double *dl = sc.take<double>(3 * (size_t)nl), *dv = sc.take<double>(3 * (size_t)nv), *dvs = sc.take<double>(3 * (size_t)nv);
    pack_dirs_kernel<<<std::max(1, (nl + 255) / 256), 256, 0, st>>>(raw_l, nl, dim, 1.0, dl, nullptr);
    pack_dirs_kernel<<<std::max(1, (nv + 255) / 256), 256, 0, st>>>(raw_v, nv, dim, a->is_ff_v ? -1.0 : 1.0, dv, dvs);
    CK(cudaGetLastError());
    LAUNCHED();
    LAUNCHED();
    P.Q.l = dl;
    P.Q.v = dv;
    P.Q.vs = dvs;

    // accumulators, counters and the scan's temporary storage
    const int64_t n = (int64_t)nv * nl;
    AccT *Us = sc.take<AccT>(2 * n), *Um = sc.take<AccT>(2 * n);
    unsigned long long *ctr = sc.take<unsigned long long>(2);
    int *err = sc.take<int>(1);
    const int64_t max_batch = 8192;
    int32_t *counts = sc.take<int32_t>(max_batch);
    int64_t *mcnt = sc.take<int64_t>(max_batch);
    int64_t *moff = sc.take<int64_t>(max_batch + 1);
    size_t scan_bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, mcnt, moff, max_batch, st));
    unsigned char *scan_tmp = sc.take<unsigned char>(scan_bytes);
    SingleRec S{sc.take<double>(3 * max_batch), sc.take<double>(3 * max_batch), sc.take<double>(max_batch),
                sc.take<double>(max_batch), sc.take<int32_t>(max_batch)};
    const int64_t scap = max_batch;
    const size_t per_event = 8 * sizeof(double) + 2 * sizeof(int32_t);
    const int64_t mcap = (int64_t)(sc.left() / per_event) - 64;
    if (mcap < 1024) fail(SCMC_ERR_INVALID, "scmc_field_noalloc: scratch too small for these inputs");
    MultiRec Mr{sc.take<double>(3 * mcap), sc.take<double>(3 * mcap), sc.take<double>(mcap), sc.take<double>(mcap),
                sc.take<int32_t>(mcap), sc.take<int32_t>(mcap)};
    CK(cudaMemsetAsync(Us, 0, 2 * n * sizeof(AccT), st));
    CK(cudaMemsetAsync(Um, 0, 2 * n * sizeof(AccT), st));

    const int sms = sm_count(a->device);
    int tv = std::min(nv, 32), tl = std::min(nl, 32);
    while (tv * tl > kFieldMaxTile) tl /= 2;
    const int n_vtiles = (nv + tv - 1) / tv, n_ltiles = (nl + tl - 1) / tl;
    const int tiles = n_vtiles * n_ltiles;
    using R = typename std::conditional<POL == P64, double, float>::type;
    using C = typename cplx_t<R>::type;
    const size_t smem = sizeof(C) * (2 * kFieldEB * (tv + tl) + kFieldEB) + sizeof(EventView) * kFieldEB + 16;
    if (smem > 48 * 1024) {
        CK(cudaFuncSetAttribute(field_accum_kernel<DIM, POL, true, AccT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CK(cudaFuncSetAttribute(field_accum_kernel<DIM, POL, false, AccT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    auto accumulate = [&](bool single, int64_t n_ev) {
        if (n_ev <= 0) return;
        int64_t ranges = std::max<int64_t>(1, (int64_t)sms * 6 / tiles);
        int64_t per = std::max<int64_t>((n_ev + ranges - 1) / ranges, kFieldEB * 4);
        ranges = (n_ev + per - 1) / per;
        dim3 grid(tiles, (unsigned)ranges);
        if (single)
            field_accum_kernel<DIM, POL, true, AccT><<<grid, kFieldThreads, smem, st>>>(Q, S, scap, Mr, mcap, n_ev, tv, tl,
                                                                                        n_vtiles, per, Us, 1);
        else
            field_accum_kernel<DIM, POL, false, AccT><<<grid, kFieldThreads, smem, st>>>(Q, S, scap, Mr, mcap, n_ev, tv, tl,
                                                                                         n_vtiles, per, Um, 1);
        CK(cudaGetLastError());
        LAUNCHED();
    };

    int64_t batch = max_batch;
    for (int64_t done = 0; done < a->max_itr;) {
        const int64_t nb = std::min(batch, a->max_itr - done);
        W.path_base = a->path_offset + (uint64_t)done;
        W.n_paths = nb;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nb + 127) / 128, (int64_t)sms * 8));
        CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), st));
        CK(cudaMemsetAsync(err, 0, sizeof(int), st));
        walk_count_kernel<DIM><<<grid, 128, 0, st>>>(W, counts, ctr, err);
        CK(cudaGetLastError());
        LAUNCHED();
        count_to_multi_kernel<<<std::max(1, (int)((nb + 255) / 256)), 256, 0, st>>>(counts, nb, mcnt);
        CK(cudaGetLastError());
        LAUNCHED();
        size_t tb = scan_bytes;
        CK(cub::DeviceScan::ExclusiveSum(scan_tmp, tb, mcnt, moff, nb, st));
        LAUNCHED();
        int64_t last[2];
        int herr = 0;
        CK(cudaMemcpyAsync(&last[0], moff + nb - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&last[1], mcnt + nb - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr) fail(SCMC_ERR_LIMIT, "a path exceeded max_events_per_path");
        const int64_t n_multi = last[0] + last[1];
        if (n_multi > mcap) {
            if (nb == 1) fail(SCMC_ERR_INVALID, "scmc_field_noalloc: one path has more events than the fixed scratch holds");
            batch = std::max<int64_t>(1, nb / 2);
            continue;  // re-walk a smaller batch (Philox regenerates the same paths)
        }
        CK(cudaMemsetAsync(ctr + 1, 0, sizeof(unsigned long long), st));
        walk_record_kernel<DIM><<<grid, 128, 0, st>>>(W, moff, S, scap, Mr, mcap, ctr + 1);
        CK(cudaGetLastError());
        LAUNCHED();
        accumulate(true, nb);
        accumulate(false, n_multi);
        done += nb;
    }
    const double m = (double)(a->norm_itr > 0 ? a->norm_itr : a->max_itr);
    const double norm = m > 0 ? std::sqrt(1.0 / m * P.volume * a->sigt) : 0.0;  // MCfield.m:253-254
    const int fgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1024));
    field_finalize_kernel<DIM, AccT><<<fgrid, 256, 0, st>>>(Q, Us, Um, norm, d_u);
    CK(cudaGetLastError());
    LAUNCHED();
}

}  // namespace

extern "C" int scmc_field_noalloc(const scmc_mc_args *args, double *d_u, void *stream)
{
    return guarded([&] {
        if (!d_u) fail(SCMC_ERR_INVALID, "null output");
        validate(args);
        if (args->nv * args->nl > 65536)
            fail(SCMC_ERR_INVALID, "scmc_field_noalloc: nv*nl is limited to 65536 by its fixed scratch");
        int ndev = 0, major = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(SCMC_ERR_NODEVICE, "no CUDA device visible");
        if (args->device < 0 || args->device >= ndev || args->device >= kMaxDevices)
            fail(SCMC_ERR_INVALID, "invalid device ordinal");
        CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, args->device));
        if (major < 10) fail(SCMC_ERR_NODEVICE, "an sm_100 (Blackwell) device is required");
        CK(cudaSetDevice(args->device));
        std::lock_guard<std::mutex> lk(g_scratch_call_mu[args->device]);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        double2 *u = reinterpret_cast<double2 *>(d_u);
        try {
            if (args->dim == 3) {
                if (args->precision == SCMC_PREC_FP64) field_noalloc_run<3, P64, double>(args, u, st);
                else if (args->precision == SCMC_PREC_FP32) field_noalloc_run<3, P32, float>(args, u, st);
                else field_noalloc_run<3, PMIX, double>(args, u, st);
            } else {
                if (args->precision == SCMC_PREC_FP64) field_noalloc_run<2, P64, double>(args, u, st);
                else if (args->precision == SCMC_PREC_FP32) field_noalloc_run<2, P32, float>(args, u, st);
                else field_noalloc_run<2, PMIX, double>(args, u, st);
            }
        } catch (...) {
            // work this call already enqueued still uses the shared array:
            // let it finish before the lock is released
            (void)cudaStreamSynchronize(st);
            throw;
        }
        CK(cudaStreamSynchronize(st));
    });
}

// ---------------------------------------------------------------------------
// serving (scmc_server_*)
// ---------------------------------------------------------------------------
extern "C" int scmc_server_create(int32_t device, int32_t n_slots, int64_t hbm_budget_bytes, scmc_server **out)
{
    return guarded([&] {
        if (!out) fail(SCMC_ERR_INVALID, "null output");
        if (n_slots < 1 || n_slots > 64) fail(SCMC_ERR_INVALID, "n_slots must be between 1 and 64");
        context(device);  // checks the ordinal and the architecture
        CK(cudaSetDevice(device));
        if (hbm_budget_bytes <= 0) {
            size_t fr = 0, tot = 0;
            CK(cudaMemGetInfo(&fr, &tot));
            hbm_budget_bytes = (int64_t)(0.8 * (double)fr);
        }
        // keep freed slot memory cached in this process's pool up to the budget
        cudaMemPool_t pool;
        CK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thr = (uint64_t)hbm_budget_bytes;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        scmc_server *s = new scmc_server();
        s->impl.device = device;
        s->impl.n_slots = n_slots;
        s->impl.budget = hbm_budget_bytes;
        s->impl.start();
        *out = s;
    });
}

extern "C" int scmc_server_submit(scmc_server *s, int32_t kind, const scmc_mc_args *args, double *out0, double *out1,
                                  int64_t *ticket)
{
    return guarded([&] {
        if (!s || !ticket) fail(SCMC_ERR_INVALID, "null server or ticket");
        if (kind != SCMC_REQ_FIELD && kind != SCMC_REQ_COV) fail(SCMC_ERR_INVALID, "unknown request kind");
        validate(args);
        if (args->device != s->impl.device) fail(SCMC_ERR_INVALID, "request device differs from the server's device");
        if (kind == SCMC_REQ_FIELD && !out0) fail(SCMC_ERR_INVALID, "null output");
        Request *r = new Request();
        r->kind = kind;
        r->args.take(*args);
        r->out0 = out0;
        r->out1 = kind == SCMC_REQ_COV ? out1 : nullptr;
        r->estimate = request_estimate(kind, r->args.a, sm_count(s->impl.device), s->impl.chunk_bytes);
        if (r->estimate > s->impl.budget) {
            delete r;
            fail(SCMC_ERR_NOMEM, "request needs more device memory than the server's HBM budget");
        }
        {
            std::lock_guard<std::mutex> lk(s->impl.mu);
            if (s->impl.stopping) {
                delete r;
                fail(SCMC_ERR_CANCELLED, "server is shutting down");
            }
            r->ticket = s->impl.next_ticket++;
            r->submit_ms = s->impl.now_ms();
            s->impl.table[r->ticket] = r;
            s->impl.queue.push_back(r);
            *ticket = r->ticket;
        }
        s->impl.cv_work.notify_all();
    });
}

extern "C" int scmc_server_wait(scmc_server *s, int64_t ticket, int64_t timeout_ms, scmc_request_info *info)
{
    int result = SCMC_OK;
    const int g = guarded([&] {
        if (!s) fail(SCMC_ERR_INVALID, "null server");
        std::unique_lock<std::mutex> lk(s->impl.mu);
        auto it = s->impl.table.find(ticket);
        if (it == s->impl.table.end()) fail(SCMC_ERR_INVALID, "unknown ticket");
        Request *r = it->second;
        auto pred = [&] { return r->finished != 0; };
        if (timeout_ms < 0) s->impl.cv_done.wait(lk, pred);
        else s->impl.cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
        s->impl.info(*r, info);
        if (!r->finished) {
            result = SCMC_ERR_TIMEOUT;
            g_last_error = "request has not finished";
            return;
        }
        result = r->status;
        g_last_error = r->message;
        s->impl.table.erase(it);
        delete r;
    });
    return g != SCMC_OK ? g : result;
}

extern "C" int scmc_server_stats_read(scmc_server *s, scmc_server_stats *out)
{
    return guarded([&] {
        if (!s || !out) fail(SCMC_ERR_INVALID, "null server or output");
        std::lock_guard<std::mutex> lk(s->impl.mu);
        out->n_slots = s->impl.n_slots;
        out->busy_slots = s->impl.busy;
        out->queued = (int64_t)s->impl.queue.size();
        out->completed = s->impl.completed;
        out->failed = s->impl.failed;
        out->budget_bytes = s->impl.budget;
        out->reserved_bytes = s->impl.reserved;
        out->peak_reserved_bytes = s->impl.peak_reserved;
        out->paths_completed = s->impl.paths_completed;
    });
}

extern "C" int scmc_server_destroy(scmc_server *s)
{
    return guarded([&] {
        if (!s) return;
        s->impl.shutdown();
        delete s;
    });
}
