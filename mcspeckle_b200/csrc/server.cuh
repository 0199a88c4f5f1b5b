// server.cuh - request server behind scmc_server_* (included by scmc_capi.cu
// inside its private namespace, after the field and covariance runners).
//
// Continuous batching of MCfield / MCcov solves: n_slots worker threads, each
// with its own CUDA stream and its own scratch context (stream-ordered
// allocations, released after every request).  Admission: a slot that falls
// idle takes the oldest request whose memory estimate fits the HBM budget
// beside the reservations of the requests already running; a request that
// does not fit may be passed by younger ones at most kMaxPassed times, after
// which nothing is admitted before it (no starvation).  The estimate is an
// upper bound from the request's sizes and expected events per path; each
// request's real footprint is reported beside its reservation.  Small field
// requests on the CUDA-core accumulation (up to kPackPaths paths, same
// dimension and precision class) are packed: the slot takes up to kPackMax of
// them from the queue and runs them as one walk, one accumulation and one
// finalisation launch per round (field_pack_device); if a pack fails, its
// requests are rerun one by one so that a failure stays with its request.
// Requests on different slots share the device: their kernels interleave and
// overlap.
// The standard headers it needs (<chrono>, <condition_variable>, <deque>,
// <thread>, <unordered_map>) are included at the top of scmc_capi.cu.
#pragma once

using SteadyClock = std::chrono::steady_clock;

struct OwnedArgs {
    scmc_mc_args a{};
    std::vector<double> l, v, amp0, icdf0, amp1, icdf1;

    static void own_pf(scmc_phase_function &pf, std::vector<double> &amp, std::vector<double> &icdf)
    {
        if (pf.sct_type != SCMC_SCT_TABULATED) return;
        amp.assign(pf.eval_amp, pf.eval_amp + 2 * (size_t)pf.table_n);
        icdf.assign(pf.sample_icdf, pf.sample_icdf + (size_t)pf.table_n);
        pf.eval_amp = amp.data();
        pf.sample_icdf = icdf.data();
    }
    void take(const scmc_mc_args &src)
    {
        a = src;
        l.assign(src.l, src.l + (size_t)src.dim * src.nl);
        v.assign(src.v, src.v + (size_t)src.dim * src.nv);
        a.l = l.data();
        a.v = v.data();
        own_pf(a.ampfunc, amp0, icdf0);
        if (a.has_ampfunc0) own_pf(a.ampfunc0, amp1, icdf1);
    }
};

struct Request {
    int64_t ticket = 0;
    int kind = SCMC_REQ_FIELD;
    OwnedArgs args;
    double *out0 = nullptr, *out1 = nullptr;
    int64_t estimate = 0, reserved = 0, peak = 0;
    int slot = -1, status = SCMC_OK, finished = 0;
    std::string message;
    double submit_ms = 0, start_ms = 0, done_ms = 0, device_ms = 0;
    int passed = 0;   // times a younger request was admitted before it
    int packed = 0;   // requests in the pack it ran in (1: alone)
};

constexpr int kMaxPassed = 16;
constexpr int kPackMax = 64;
constexpr int64_t kPackPaths = (int64_t)1 << 20;       // per request
constexpr int64_t kPackTotalPaths = (int64_t)1 << 23;  // per pack

// Device memory a request will hold on its slot, from its sizes.  The walk
// term uses the expected events per path of a slab sigt*thickness optical
// depths thick (about 2 per optical depth plus a constant); the real count is
// known only after the walk, and the server tracks the real footprint.
int64_t request_estimate(int kind, const scmc_mc_args &a, int sms, size_t chunk_bytes)
{
    const scmc_tuning T = tuning_for(kind == SCMC_REQ_FIELD ? SCMC_TUNE_FIELD : SCMC_TUNE_COV, a.precision, a.nv * a.nl);
    const int64_t nb = std::max<int64_t>(1, std::min<int64_t>(a.max_itr, T.path_batch));
    const double depth = a.sigt * (a.box_max[a.dim - 1] - a.box_min[a.dim - 1]);
    const double ev = 4.0 + 2.0 * std::max(depth, 1.0);
    double walk = (double)nb * (4 + 8 + 8 + 68) + (double)nb * ev * 1.25 * 72;
    const double nv = (double)a.nv, nl = (double)a.nl;
    double acc = 0;
    if (kind == SCMC_REQ_FIELD) {
        const bool tc = use_field_tc(&a);
        if (tc) {
            FieldTcPlan p = field_tc_plan((int)a.nv, (int)a.nl, a.do_cbs ? 2 : 1, a.precision == SCMC_PREC_MIXED, sms,
                                          chunk_bytes, T.ksplit);
            acc = (double)field_tc_bytes(p) + 2.0 * p.ksplit * 2 * nv * nl * 8;
        } else {
            acc = 2.0 * 2 * nv * nl * 8;
        }
        acc += 2 * nv * nl * 8;  // device copy of u
    } else {
        const double N = nv * nl;
        const bool tc = a.precision == SCMC_PREC_MIXED || a.precision == SCMC_PREC_FP16;
        // tensor-core path: two accumulators each for Ms and Mm and three
        // operand buffers; CUDA-core path: one accumulator each and a row buffer;
        // both: device copies of Ms, Mm
        acc = (tc ? 4.0 : 2.0) * 2 * N * N * 8 + 2.0 * 2 * N * N * 8;
        if (tc)
            acc += 3.0 * (double)tc_operand_bytes(
                                 tc_plan((int)N, a.precision == SCMC_PREC_MIXED, chunk_bytes, T.chunk_events, T.stages));
        else acc += 256.0 * (1 << 20);
    }
    // every scratch buffer is allocated 1/8 above its request (DevBuf::ensure)
    return (int64_t)((walk + acc) * 1.125 * 1.05) + ((int64_t)16 << 20);
}

struct Server {
    int device = 0;
    int n_slots = 0;
    int64_t budget = 0;
    // the library's default operand memory per tensor-core chunk, so that a
    // request's chunks (and their FP32 sums) are the same on a slot as alone
    size_t chunk_bytes = (size_t)2 << 30;
    SteadyClock::time_point t0;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<int64_t, Request *> table;
    int64_t next_ticket = 1;
    int64_t reserved = 0, peak_reserved = 0, completed = 0, failed = 0, paths_completed = 0;
    int busy = 0;
    bool stopping = false;
    std::vector<std::thread> workers;
    std::vector<std::string> worker_error;

    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(SteadyClock::now() - t0).count();
    }

    void start()
    {
        t0 = SteadyClock::now();
        worker_error.assign(n_slots, std::string());
        for (int s = 0; s < n_slots; ++s) workers.emplace_back([this, s] { worker(s); });
    }

    // The queue index of the request to admit next, if any fits: the oldest
    // that fits the budget, younger ones passing an older one that does not fit
    // at most kMaxPassed times.  Called with mu held.
    bool admissible(size_t &pick)
    {
        for (size_t i = 0; i < queue.size(); ++i) {
            if (reserved + queue[i]->estimate <= budget) {
                pick = i;
                return true;
            }
            if (queue[i]->passed >= kMaxPassed) return false;  // its turn: wait for room
        }
        return false;
    }

    // Runs a pack of small field requests as one walk / accumulate / finalise
    // launch sequence per round and copies each result out.
    void run_pack(Ctx &c, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, std::vector<Request *> &batch)
    {
        size_t total = 0;
        for (Request *r : batch) total += (size_t)r->args.a.nv * r->args.a.nl * 2;
        CK(cudaEventRecord(e0, st));
        double *d = reinterpret_cast<double *>(c.out0.ensure(total * sizeof(double)));
        std::vector<PackItem> items;
        size_t o = 0;
        for (Request *r : batch) {
            items.push_back(PackItem{&r->args.a, d + o});
            o += (size_t)r->args.a.nv * r->args.a.nl * 2;
        }
        field_pack_device(c, items, st);
        o = 0;
        for (Request *r : batch) {
            const size_t n = (size_t)r->args.a.nv * r->args.a.nl * 2;
            CK(cudaMemcpyAsync(r->out0, d + o, n * sizeof(double), cudaMemcpyDeviceToHost, st));
            o += n;
        }
        CK(cudaEventRecord(e1, st));
        CK(cudaStreamSynchronize(st));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        for (Request *r : batch) r->device_ms = ms;
    }

    // Runs one request on a slot's stream and copies its result out.
    void run(Ctx &c, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, Request &r)
    {
        const scmc_mc_args *a = &r.args.a;
        CK(cudaEventRecord(e0, st));
        const size_t n_out = r.kind == SCMC_REQ_FIELD ? (size_t)a->nv * a->nl * 2 : (size_t)a->nv * a->nl * a->nv * a->nl * 2;
        if (r.kind == SCMC_REQ_FIELD) {
            double *d = reinterpret_cast<double *>(c.out0.ensure(n_out * sizeof(double)));
            field_device_locked(c, a, d, st);
            CK(cudaMemcpyAsync(r.out0, d, n_out * sizeof(double), cudaMemcpyDeviceToHost, st));
        } else {
            double *d0 = r.out0 ? reinterpret_cast<double *>(c.out0.ensure(n_out * sizeof(double))) : nullptr;
            double *d1 = r.out1 ? reinterpret_cast<double *>(c.out1.ensure(n_out * sizeof(double))) : nullptr;
            cov_device_locked(c, a, d0, d1, st);
            if (d0) CK(cudaMemcpyAsync(r.out0, d0, n_out * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (d1) CK(cudaMemcpyAsync(r.out1, d1, n_out * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        CK(cudaEventRecord(e1, st));
        CK(cudaStreamSynchronize(st));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        r.device_ms = ms;
    }

    void worker(int s)
    {
        cudaStream_t st = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        Ctx c;
        c.device = device;
        c.tc_chunk_bytes = chunk_bytes;
        if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            worker_error[s] = "slot set-up failed";
            return;
        }
        c.set_stream_ordered(st);
        for (;;) {
            std::vector<Request *> batch;
            {
                std::unique_lock<std::mutex> lk(mu);
                size_t pick = 0;
                cv_work.wait(lk, [&] { return stopping || admissible(pick); });
                if (stopping) break;  // shutdown has cancelled the queue
                Request *r = queue[pick];
                for (size_t i = 0; i < pick; ++i) ++queue[i]->passed;
                queue.erase(queue.begin() + (std::ptrdiff_t)pick);
                batch.push_back(r);
                // a small CUDA-core field request takes others of its class along
                const int cls = pack_class(r->kind, r->args.a, kPackPaths);
                int64_t paths = r->args.a.max_itr, res = reserved + r->estimate;
                if (cls >= 0) {
                    for (size_t i = 0; i < queue.size() && (int)batch.size() < kPackMax;) {
                        Request *q = queue[i];
                        if (pack_class(q->kind, q->args.a, kPackPaths) == cls && paths + q->args.a.max_itr <= kPackTotalPaths &&
                            res + q->estimate <= budget) {
                            paths += q->args.a.max_itr;
                            res += q->estimate;
                            batch.push_back(q);
                            queue.erase(queue.begin() + (std::ptrdiff_t)i);
                        } else {
                            ++i;
                        }
                    }
                }
                const double t = now_ms();
                for (Request *q : batch) {
                    q->slot = s;
                    q->reserved = q->estimate;
                    q->start_ms = t;
                    q->packed = (int)batch.size();
                    reserved += q->reserved;
                }
                peak_reserved = std::max(peak_reserved, reserved);
                ++busy;
            }
            std::vector<int> status(batch.size(), SCMC_OK);
            std::vector<std::string> msg(batch.size());
            auto attempt = [&](auto &&fn, size_t k) {
                try {
                    fn();
                } catch (const ScmcError &e) {
                    status[k] = e.code;
                    msg[k] = e.msg;
                } catch (const std::exception &e) {
                    status[k] = SCMC_ERR_CUDA;
                    msg[k] = e.what();
                }
            };
            if (batch.size() == 1) {
                attempt([&] { run(c, st, e0, e1, *batch[0]); }, 0);
            } else {
                attempt([&] { run_pack(c, st, e0, e1, batch); }, 0);
                if (status[0] != SCMC_OK) {  // rerun one by one: a failure stays with its request
                    try {
                        cudaStreamSynchronize(st);
                        c.release_all();
                    } catch (...) {
                    }
                    for (size_t k = 0; k < batch.size(); ++k) {
                        status[k] = SCMC_OK;
                        msg[k].clear();
                        batch[k]->packed = 1;
                        attempt([&] { run(c, st, e0, e1, *batch[k]); }, k);
                    }
                } else {
                    for (size_t k = 1; k < batch.size(); ++k) status[k] = SCMC_OK;
                }
            }
            const int64_t held = (int64_t)c.held();  // what the slot allocated for this request or pack
            try {
                c.release_all();
                cudaStreamSynchronize(st);
            } catch (...) {
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                const double t = now_ms();
                for (size_t k = 0; k < batch.size(); ++k) {
                    Request *r = batch[k];
                    r->peak = held;
                    reserved -= r->reserved;
                    r->status = status[k];
                    r->message = msg[k];
                    r->done_ms = t;
                    r->finished = 1;
                    if (status[k] == SCMC_OK) {
                        ++completed;
                        paths_completed += r->args.a.max_itr;
                    } else {
                        ++failed;
                    }
                }
                --busy;
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
        c.destroy_aux();
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(st);
    }

    void info(const Request &r, scmc_request_info *o) const
    {
        if (!o) return;
        o->ticket = r.ticket;
        o->kind = r.kind;
        o->slot = r.slot;
        o->status = r.status;
        o->finished = r.finished;
        o->submit_ms = r.submit_ms;
        o->start_ms = r.start_ms;
        o->done_ms = r.done_ms;
        o->device_ms = r.device_ms;
        o->reserved_bytes = r.reserved ? r.reserved : r.estimate;
        o->peak_bytes = r.peak;
        o->paths = r.args.a.max_itr;
        o->packed = r.packed;
    }

    void shutdown()
    {
        std::deque<Request *> cancelled;
        {
            std::lock_guard<std::mutex> lk(mu);
            stopping = true;
            cancelled.swap(queue);
            for (Request *r : cancelled) {
                r->status = SCMC_ERR_CANCELLED;
                r->message = "server destroyed before the request was admitted";
                r->finished = 1;
                r->done_ms = now_ms();
            }
        }
        cv_work.notify_all();
        for (auto &t : workers)
            if (t.joinable()) t.join();
        cv_done.notify_all();
        for (auto &kv : table) delete kv.second;
        table.clear();
    }
};
