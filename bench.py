#!/usr/bin/env python
"""Throughput of SCMC's Monte Carlo speckle path on B200.

Headline workload (the one the metric is quoted on that fits one GPU): the
far-field covariance - MCcov on a homogeneous box 20 x 20 x 5 MFP (MFP = 10
wavelengths, wavelength 1), Henyey-Greenstein g=0.8, sigma_s = 1,
sigma_a = 0.01 per MFP, 64 lights and 64 views on regular 8 x 8
(sin theta_x, sin theta_y) grids spanning +-5 degrees about +z / -z
(reflection, CBS on, exponential first-scatter sampling), 1e7 paths per GPU
per step, full 64x64x64x64 complex covariance.  Synthetic: every input is
generated from fixed seeds; each step walks a fresh Philox path range.

One step = one MCcov solve of --paths paths on every GPU (default precision
fp16: one FP16 tcgen05 product per term with FP32 accumulation, phases
reduced in FP64, FP64 cross-chunk sums; --precision mixed runs the FP16
hi+lo split), plus for N>1 an NCCL sum of the partial Ms / Mm.  `value` =
paths of all ranks / the max over ranks of the CUDA-event time of the K
timed steps, outputs in HBM.  `e2e` = the same through the host-buffer C ABI
call (scmc_cov: inputs from host, Ms / Mm copied back to host every step).

On one GPU the line also carries `workloads`: the other measured
configurations (field16, fq256, hetero128), each with its own device-timed
value, host-buffer e2e, roofline of its dominant kernel, error against the
FP64 oracle on a small sample and the CPU oracle's rate; and `serving`, the
served request stream.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mcspeckle_b200 import workloads as WL  # noqa: E402

METRIC = "MC paths/s at 1e-3 rel err vs FP64 (mixed vs FP32 GPU); p50/p99 request latency"
UNIT = "paths/s"
WORKLOAD = WL.COV64
workload_args = WL.cov64_args


# ---------------------------------------------------------------------------
# measurement helpers
# ---------------------------------------------------------------------------
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def load_traffic(name):
    """DRAM bytes per unit of work of a kernel, from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


def rel_err(x, ref, mask=None):
    """Relative Frobenius error of x (array or tuple of arrays) against ref."""
    x = x if isinstance(x, tuple) else (x,)
    ref = ref if isinstance(ref, tuple) else (ref,)
    num = den = 0.0
    for xa, ra in zip(x, ref):
        if mask is not None:
            m = np.broadcast_to(mask, ra.shape)
            xa, ra = xa[m], ra[m]
        num += float(np.linalg.norm((xa - ra).ravel())) ** 2
        den += float(np.linalg.norm(ra.ravel())) ** 2
    return math.sqrt(num / den)


def cpu_oracle_rate(args_fn, target_s=15.0, threads=None):
    """The FP64 oracle (C restatement of MCcov) on the host cores: paths/s on a
    bounded sample of the same workload."""
    from mcspeckle_b200 import mc as MC
    from oracle import oracle as O
    O.build()
    threads = threads or os.cpu_count() or 1
    n = 2
    while True:
        h = MC.mc_args(*args_fn(n), seed=99, precision="fp64")
        t0 = time.perf_counter()
        O.cov(h, O.Rng.philox(), threads=threads)
        dt = time.perf_counter() - t0
        if dt >= target_s or n >= 4096:
            return n / dt, n, dt, threads
        n = max(n + 1, int(n * min(8.0, 1.3 * target_s / max(dt, 1e-3))))


def run_reference(a):
    """--impl reference: the CPU oracle port of the reference's MCcov timed on
    the host cores (MATLAB / Octave are not available on this box)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    per_step = []
    sample = None
    for i in range(a.warmup + a.steps):
        rate, n, dt, thr = cpu_oracle_rate(workload_args, target_s=a.ref_seconds)
        if i >= a.warmup:
            per_step.append((rate, n, dt))
        sample = (n, thr)
    value = float(np.median([r for r, _, _ in per_step]))
    ms = 1000.0 * float(np.mean([n / r for r, n, _ in per_step]))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "paths_per_step": sample[0], "full_config_paths": 10_000_000},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": sample[1], "kind": "port",
                         "sample": f"{sample[0]} paths of the workload per step (oracle/scmc_oracle.c MCcov, FP64, "
                                   f"{sample[1]} threads; MATLAB/Octave absent on this box)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# served stream: uneven MCfield requests with Poisson arrivals
# ---------------------------------------------------------------------------
def serve(reqs, slots=8, rate=None, precision="mixed", device=0, budget=80e9):
    """Runs the requests through the request server.  rate None: all submitted
    at once (closed batch); else Poisson arrivals at `rate` requests/s.
    Returns per-request infos (server clock) and the results."""
    from mcspeckle_b200 import mc as MC
    from mcspeckle_b200.serving import Server
    holders = [MC.mc_args(*r["args"], seed=r["seed"], precision=precision, device=device) for r in reqs]
    gaps = np.random.default_rng(11).exponential(1.0 / rate, len(reqs)) if rate else np.zeros(len(reqs))
    arrive = np.cumsum(gaps) - gaps[0]
    tickets = [None] * len(reqs)
    with Server(device=device, slots=slots, hbm_budget=budget) as srv:
        def submitter():
            t0 = time.perf_counter()
            for i, h in enumerate(holders):
                dt = arrive[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                tickets[i] = srv.submit_field(h)

        th = threading.Thread(target=submitter)
        th.start()
        infos, results = [], []
        for i in range(len(reqs)):
            while tickets[i] is None:
                time.sleep(0.0005)
            u, info = srv.wait(tickets[i])
            infos.append(info)
            results.append(u)
        th.join()
        stats = srv.stats()
    return infos, results, stats


def served_summary(reqs, infos):
    lat = np.array([i["done_ms"] - i["submit_ms"] for i in infos])
    t0 = min(i["submit_ms"] for i in infos)
    t1 = max(i["done_ms"] for i in infos)
    paths = sum(r["paths"] for r in reqs)
    busy = sum(i["device_ms"] for i in infos)
    out = {"requests": len(reqs), "paths": int(paths), "makespan_s": (t1 - t0) / 1000.0,
           "paths_per_s": paths / ((t1 - t0) / 1000.0), "p50_ms": float(np.percentile(lat, 50)),
           "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
           "sum_device_ms": busy}
    # latency by request size (paths x (views + lights)): the small, medium and large thirds
    size = np.array([r["paths"] * (r["nv"] + r["nl"]) for r in reqs], dtype=float)
    if len(reqs) >= 6:
        cuts = np.quantile(size, [1 / 3, 2 / 3])
        buckets = {}
        for name, sel in (("small", size <= cuts[0]), ("medium", (size > cuts[0]) & (size <= cuts[1])),
                          ("large", size > cuts[1])):
            if sel.any():
                buckets[name] = {"requests": int(sel.sum()), "p50_ms": float(np.percentile(lat[sel], 50)),
                                 "p99_ms": float(np.percentile(lat[sel], 99)),
                                 "paths_range": [int(min(r["paths"] for r, s in zip(reqs, sel) if s)),
                                                 int(max(r["paths"] for r, s in zip(reqs, sel) if s))]}
        out["by_size"] = buckets
    return out


def run_served_leg(a, device):
    """Served stream: closed batch (capacity), then Poisson arrivals at 85% of
    that capacity (latency), then a plain FP32 one-request-at-a-time pass and
    the same requests served, on a prefix."""
    from mcspeckle_b200 import mc as MC
    lo, hi = a.served_paths_min, a.served_paths_max
    reqs = WL.served_requests(a.served_requests, paths=(lo, hi))
    infos, _, st_closed = serve(reqs, slots=a.slots, device=device)
    closed = served_summary(reqs, infos)
    rate = 0.85 * len(reqs) / closed["makespan_s"]
    infos, _, st_open = serve(reqs, slots=a.slots, rate=rate, device=device)
    opened = served_summary(reqs, infos)
    # plain FP32, one request at a time, on a prefix of the stream (bounded time)
    t0 = time.perf_counter()
    k = 0
    while k < len(reqs) and time.perf_counter() - t0 < a.served_fp32_seconds:
        r = reqs[k]
        MC.field_from_args(MC.mc_args(*r["args"], seed=r["seed"], precision="fp32", device=device))
        k += 1
    fp32_s = time.perf_counter() - t0
    prefix = reqs[:k]
    infos_p, _, _ = serve(prefix, slots=a.slots, device=device)
    served_prefix = served_summary(prefix, infos_p)
    fp32_rate = sum(r["paths"] for r in prefix) / fp32_s
    return {
        "workload": WL.SERVED, "requests": len(reqs), "paths_range": [lo, hi],
        "path_budget_note": f"the config's 10,000 requests at 1e5-1e8 paths run as {len(reqs)} requests at "
                            f"{lo:.0e}-{hi:.0e} so the leg ends in minutes",
        "slots": a.slots, "hbm_budget_gb": 80, "precision": "mixed",
        "closed_batch": closed, "poisson": dict(opened, offered_load=0.85, rate_per_s=rate),
        "peak_reserved_gb": max(st_closed["peak_reserved_bytes"], st_open["peak_reserved_bytes"]) / 1e9,
        "fp32_one_at_a_time": {"requests": k, "paths_per_s": fp32_rate, "seconds": fp32_s},
        "served_same_prefix": {"requests": k, "paths_per_s": served_prefix["paths_per_s"]},
        "speedup_vs_fp32_one_at_a_time": served_prefix["paths_per_s"] / fp32_rate,
    }


# ---------------------------------------------------------------------------
# the other configurations: field16, fq256, hetero128
# ---------------------------------------------------------------------------
class Leg:
    """One configuration: how to build a solve, run it on the device and from
    host buffers, its oracle, and the kernel whose roofline is reported."""

    def __init__(self, name):
        from mcspeckle_b200 import _lib
        from mcspeckle_b200 import fourier_quad as FQ
        from mcspeckle_b200 import hetero as H
        from mcspeckle_b200 import mc as MC
        L = _lib.lib()
        self.name = name
        self.mask = None
        self.device_compare = False
        if name == "field16":
            self.desc = WL.FIELD16 + ", phases reduced in FP64, CUDA-core accumulation"
            self.paths, self.acc_paths, self.cpu_paths = 1_000_000, 20_000, 4000
            self.make = lambda n, p, seed, off=0, norm=0: MC.mc_args(*WL.field16_args(n), seed=seed, precision=p,
                                                                     path_offset=off, norm_itr=norm)
            self.sizes = [2 * 16 * 16]
            self.dev = lambda h, outs, st: _lib.check(L.scmc_field_device(h.ref, outs[0].data_ptr(), st))
            self.host = MC.field_from_args
            self.oracle = lambda h, O: O.field(h, O.Rng.philox())
            self.kernel, self.bound, self.stage = "field_accum_kernel", "fp32", "rows"
            self.traffic_file, self.unit_name = "field_accum_kernel_field16_traffic.json", "event"
            self.h2d = 2 * 16 * 3 * 8
            self.cpu_threads = 1
        elif name == "fq256":
            self.desc = WL.fq256_desc(True)
            self.paths, self.acc_paths, self.cpu_paths = 10_000_000, 40, 40
            self.make = lambda n, p, seed, off=0, norm=0: WL.fq256_args(n, extended=True, seed=seed, precision=p,
                                                                        path_offset=off)
            self.sizes = [2 * 256 * 256]
            self.dev = lambda h, outs, st: _lib.check(L.scmc_field_fourier_quad_device(h.ref, outs[0].data_ptr(), st))
            self.host = FQ.field_fourier_quad_from_args
            self.oracle = lambda h, O: O.field_fourier_quad(h.args, O.Rng.philox(), h.nv0)
            self.mask = WL.fq256_propagating()
            self.kernel, self.bound, self.stage = "fq_pair_planes_kernel", "tensor", "contract"
            self.traffic_file, self.unit_name = "fq_pair_planes_kernel_fq256_traffic.json", "entry"
            self.h2d = 3 * 8 + 256 * 256 * 16 * 2
            self.cpu_threads = 1
        elif name == "hetero128":
            self.desc = WL.hetero128_desc()
            self.paths, self.acc_paths, self.cpu_paths = 100_000, 8, 8
            self.make = lambda n, p, seed, off=0, norm=0: WL.hetero128_args(n, seed=seed, precision=p,
                                                                            path_offset=off, norm_itr=norm)
            n2 = 128 * 128
            self.sizes = [2 * n2 * n2, 2 * n2 * n2, 2 * n2]
            self.dev = lambda h, outs, st: _lib.check(L.scmc_cov_hetero_device(
                h.ref, outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), st))
            self.host = lambda h: H.cov_hetero_from_args(h)[:2]
            self.oracle = lambda h, O: O.cov_hetero(h, O.Rng.philox(), threads=os.cpu_count() or 1)[:2]
            self.kernel, self.bound, self.stage = "herk_tc2_kernel", "tensor", "contract"
            self.traffic_file, self.unit_name = "herk_tc2_kernel_hetero128_traffic.json", "event"
            self.h2d = 128 ** 3 * 8 + 2 * 128 * 3 * 8 + 1024 * 24
            self.cpu_threads = os.cpu_count() or 1
            self.device_compare = True
        else:
            raise SystemExit(f"unknown workload {name}")


def _device_rel(outs, ref_dev):
    num = den = 0.0
    step = 1 << 27
    for x, r in zip(outs, ref_dev):
        for k in range(0, r.numel(), step):
            rr = r[k:k + step]
            num += float(((x[k:k + step] - rr) ** 2).sum())
            den += float((rr ** 2).sum())
    return math.sqrt(num / den)


def leg_accuracy(leg, precisions, O):
    """Error of each precision against the FP64 oracle on the same paths
    (a small sample; the oracle runs outside every timed region)."""
    import torch
    na = leg.acc_paths
    ho = leg.make(na, "fp64", 7)
    ref = leg.oracle(ho, O)
    out = {"paths": na, "tol": 1e-3, "reference": "FP64 oracle (C restatement of the reference) on the same "
                                                   "Philox paths"}
    if leg.mask is not None:
        out["mask"] = "propagating directions (vx^2 + vy^2 < 1)"
    if leg.device_compare:
        ref_dev = [torch.from_numpy(x.reshape(-1, order="F").view(np.float64)).cuda() for x in ref]
        del ref
        for p in precisions:
            outs = [torch.empty(n, dtype=torch.float64, device="cuda") for n in leg.sizes]
            leg.dev(leg.make(na, p, 7), outs, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            out[f"rel_err_{p}_vs_oracle"] = _device_rel(outs[:len(ref_dev)], ref_dev)
            del outs
        del ref_dev
        torch.cuda.empty_cache()
    else:
        for p in precisions:
            out[f"rel_err_{p}_vs_oracle"] = rel_err(leg.host(leg.make(na, p, 7)), ref, leg.mask)
    return out


def run_leg(leg, a, prec, peaks, peak_kind):
    """Device-timed steps of fresh path ranges (outputs in HBM), the
    host-buffer call, the roofline of the dominant kernel, accuracy against
    the oracle, plain FP32 and the CPU oracle."""
    import torch
    from mcspeckle_b200 import _lib
    from oracle import oracle as O
    O.build()
    P = int(a.leg_paths.get(leg.name, leg.paths))
    stream = torch.cuda.current_stream()
    outs = [torch.zeros(n, dtype=torch.float64, device="cuda") for n in leg.sizes]

    def step(i):
        leg.dev(leg.make(P, prec, 0, off=i * P, norm=P), outs, stream.cuda_stream)

    for i in range(a.warmup):
        step(i)
    torch.cuda.synchronize()
    clocks = ClockSampler(0).start()
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    l0 = _lib.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(a.steps):
        step(a.warmup + i)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = _lib.launch_count() - l0
    _lib.profile_enable(False)
    prof = _lib.profile_read(reset=True)
    clk = clocks.stop()
    del outs
    torch.cuda.empty_cache()
    value = P * a.steps / (ms / 1000.0)
    # e2e: the host-buffer call (inputs from host, results copied back every step)
    ke = min(a.steps, a.leg_e2e_steps)
    e2e = None
    if ke > 0:
        t0 = time.perf_counter()
        for i in range(ke):
            leg.host(leg.make(P, prec, 0, off=(a.warmup + a.steps + i) * P, norm=P))
        e2e = P * ke / (time.perf_counter() - t0)
    # roofline of the dominant kernel over its busy time (launches on several
    # streams overlap; each instant counts once)
    roof = None
    busy = prof[f"{leg.stage}_busy_ms"]
    if busy > 0:
        tj = load_traffic(leg.traffic_file)
        if leg.bound == "tensor":
            work = prof["contract_flops"]
            peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
            peak_src = f"bf16_tflops_sustained ({peak_kind})"
            units = work / (8.0 * 256 * 256) if leg.name == "fq256" else work / (4.0 * 16384 * 16385)
        else:
            # CUDA-core field accumulation: 8 nv nl flops per event and term
            # (single events 1 term, multiple-scattering events 2 with CBS)
            ev = prof["events"]
            paths = prof["paths"]
            work = 8.0 * 16 * 16 * (paths + 2.0 * (ev - paths))
            units = ev
            sms = torch.cuda.get_device_properties(0).multi_processor_count
            mhz = clk.get("sm_max_mhz") or 1965.0
            peak = sms * 128 * 2 * mhz * 1e6 / 1e12
            peak_src = f"nominal FP32 FMA peak ({sms} SMs x 128 lanes x 2 flops x {mhz:.0f} MHz)"
        n_launch = max(prof[f"{leg.stage}_launches"], 1)
        achieved = work / (busy / 1000.0) / 1e12
        traffic = None
        if tj is not None:
            traffic = tj[f"dram_bytes_per_{leg.unit_name}"] * units / n_launch
        roof = {"bound": leg.bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": leg.kernel, "peak_source": peak_src,
                "flops_per_launch": work / n_launch, "busy_ms_per_launch": busy / n_launch, "launches": n_launch,
                f"{leg.unit_name}s_per_launch": units / n_launch,
                "traffic_source": f"profiles/{leg.traffic_file}" if tj is not None else None}
    acc = None if a.no_accuracy else leg_accuracy(leg, [prec] + [p for p in ("mixed", "fp16", "fp32") if p != prec], O)
    # plain FP32 GPU on a smaller sample, and the same sample in the line's precision
    n32 = max(1, P // 10)
    fp32 = None
    if not a.no_fp32:
        t32 = time.perf_counter()
        leg.host(leg.make(n32, "fp32", 0))
        fp32_value = n32 / (time.perf_counter() - t32)
        tp = time.perf_counter()
        leg.host(leg.make(n32, prec, 0))
        same_value = n32 / (time.perf_counter() - tp)
        fp32 = {"paths": n32, "value": fp32_value, f"{prec}_same_sample": same_value,
                f"speedup_{prec}_over_fp32": same_value / fp32_value}
    cpu = None
    if not a.no_cpu_baseline:
        n = leg.cpu_paths
        h = leg.make(n, "fp64", 99)
        tc = time.perf_counter()
        r = leg.oracle(h, O)
        dt = time.perf_counter() - tc
        del r
        cpu = {"value": n / dt, "unit": UNIT, "cores": leg.cpu_threads, "kind": "port",
               "sample": f"{n} paths of the workload in {dt:.1f} s (FP64 oracle, {leg.cpu_threads} thread(s))"}
    return {"workload": leg.name, "description": leg.desc, "value": value, "unit": UNIT, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "paths_per_step": P, "precision": prec,
            "e2e": None if e2e is None else {"value": e2e, "unit": UNIT, "steps": ke, "h2d_bytes_per_step": int(leg.h2d),
                                             "d2h_bytes_per_step": int(sum(leg.sizes[:2]) * 8)},
            "gpu_launches": int(launches), "roofline": roof,
            "stages_ms": {k: prof[k] for k in ("walk_ms", "rows_ms", "contract_ms", "finalize_ms",
                                               "contract_busy_ms", "rows_busy_ms")},
            "accuracy": acc, "fp32_gpu": fp32, "cpu_baseline": cpu, "clocks": clk}


def run_workload(a):
    """--workload NAME: one configuration's leg alone, as one JSON line."""
    peaks, kind = load_peaks()
    r = run_leg(Leg(a.workload), a, a.precision, peaks, kind)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": a.precision, "data": "synthetic",
            "config": {"workload": a.workload, "description": r["description"], "paths_per_step": r["paths_per_step"],
                       "precision": a.precision},
            **{k: r[k] for k in ("e2e", "gpu_launches", "roofline", "stages_ms", "accuracy", "fp32_gpu",
                                 "cpu_baseline", "clocks")}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the headline: far-field covariance, 64 x 64
# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--paths", type=float, default=None, help="paths per GPU per step (cov64: 1e7)")
    ap.add_argument("--accuracy-paths", type=float, default=1e5,
                    help="cov64: regenerated paths for the error against the GPU's FP64 mode")
    ap.add_argument("--oracle-paths", type=int, default=100, help="cov64: paths for the error against the oracle")
    ap.add_argument("--fp32-paths", type=float, default=1e5)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp16", choices=["mixed", "fp16"],
                    help="mixed: FP16 hi+lo split (2 tensor products); fp16: one FP16 product")
    ap.add_argument("--served-requests", type=int, default=24)
    ap.add_argument("--served-paths-min", type=float, default=1e5)
    ap.add_argument("--served-paths-max", type=float, default=1e8)
    ap.add_argument("--served-fp32-seconds", type=float, default=10.0)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--legs", default="field16,fq256,hetero128",
                    help="configurations measured beside the headline on one GPU ('' for none)")
    ap.add_argument("--leg-paths", default="", help="per-leg path budgets, e.g. fq256=1e6,hetero128=2e4")
    ap.add_argument("--leg-e2e-steps", type=int, default=3, help="host-buffer solves per leg (0: none)")
    ap.add_argument("--no-accuracy", action="store_true", help="legs: skip the oracle comparison (profiling runs)")
    ap.add_argument("--no-fp32", action="store_true", help="legs: skip the plain FP32 comparison (profiling runs)")
    ap.add_argument("--workload", default="cov64", choices=["cov64", "field16", "fq256", "hetero128"],
                    help="cov64: the default line; the others print one line of their own (1 GPU)")
    a = ap.parse_args()
    a.leg_paths = {k: int(float(v)) for k, v in (kv.split("=") for kv in a.leg_paths.split(",") if kv)}
    if a.impl == "reference":
        return run_reference(a)
    if a.workload != "cov64":
        import torch
        torch.cuda.set_device(0)
        return run_workload(a)
    a.paths = 1e7 if a.paths is None else a.paths

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from mcspeckle_b200 import _lib
    from mcspeckle_b200 import mc as MC

    P = int(a.paths)
    N = 64 * 64
    n_out = N * N
    stream = torch.cuda.current_stream()
    Ms = torch.zeros(2 * n_out, dtype=torch.float64, device="cuda")
    Mm = torch.zeros(2 * n_out, dtype=torch.float64, device="cuda")
    seed = 0x5C3C0FFEE

    def step_args(step, n=P, precision=a.precision):
        off = (step * world + rank) * n
        return MC.mc_args(*workload_args(n), seed=seed, precision=precision, device=local, path_offset=off,
                          norm_itr=n * world)

    def device_step(step):
        h = step_args(step)
        _lib.check(_lib.lib().scmc_cov_device(h.ref, Ms.data_ptr(), Mm.data_ptr(), stream.cuda_stream))
        if world > 1:
            dist.all_reduce(Ms)
            dist.all_reduce(Mm)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    for s in range(a.warmup):
        device_step(s)
    barrier()

    # timed region (device-resident outputs)
    clocks = ClockSampler(local).start()
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    l0 = _lib.launch_count()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(a.steps):
        device_step(a.warmup + s)
    e1.record(stream)
    barrier()
    ms_total = e0.elapsed_time(e1)
    launches = _lib.launch_count() - l0
    _lib.profile_enable(False)
    prof = _lib.profile_read(reset=True)
    clk = clocks.stop()
    t = torch.tensor([ms_total], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = P * world * a.steps / (ms_max / 1000.0)

    # e2e: the host-buffer C ABI call, outputs copied to pinned host memory
    host_Ms = torch.empty(2 * n_out, dtype=torch.float64, pin_memory=True)
    host_Mm = torch.empty(2 * n_out, dtype=torch.float64, pin_memory=True)
    h_in = step_args(0)
    h2d = int(h_in.args.nl * 3 * 8 + h_in.args.nv * 3 * 8)
    barrier()
    t0 = time.perf_counter()
    for s in range(a.steps):
        h = step_args(a.warmup + a.steps + s)
        if world == 1:
            dp = ctypes.POINTER(ctypes.c_double)
            _lib.check(_lib.lib().scmc_cov(h.ref, ctypes.cast(host_Ms.data_ptr(), dp),
                                           ctypes.cast(host_Mm.data_ptr(), dp)))
        else:
            _lib.check(_lib.lib().scmc_cov_device(h.ref, Ms.data_ptr(), Mm.data_ptr(), stream.cuda_stream))
            dist.all_reduce(Ms)
            dist.all_reduce(Mm)
            host_Ms.copy_(Ms, non_blocking=True)
            host_Mm.copy_(Mm, non_blocking=True)
            torch.cuda.synchronize()
    barrier()
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = P * world * a.steps / float(t.item())

    # the memory-effect view of the last step's covariance (offset means, FP32), HBM bound
    n_off = 15 ** 4
    R = torch.empty(2 * n_off, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().scmc_cov_offsets_device(Ms.data_ptr(), Mm.data_ptr(), 8, 8, 8, 8, R.data_ptr(), local,
                                                  stream.cuda_stream))
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    _lib.check(_lib.lib().scmc_cov_offsets_device(Ms.data_ptr(), Mm.data_ptr(), 8, 8, 8, 8, R.data_ptr(), local,
                                                  stream.cuda_stream))
    f1.record(stream)
    torch.cuda.synchronize()
    off_ms = f0.elapsed_time(f1)
    Rh = R.cpu().numpy().view(np.complex64).reshape(15, 15, 15, 15, order="F")
    # along equal view and light tilts (dv = dl along one grid axis) relative to no offset
    curve = [float(abs(Rh[7 + d, 7, 7 + d, 7]) / abs(Rh[7, 7, 7, 7])) for d in range(8)]
    memory_effect = {"kernel_ms": off_ms, "hbm_gbs": 2 * 2 * n_out * 8 / (off_ms / 1000.0) / 1e9,
                     "output": "15x15x15x15 complex f32 (view offset x light offset on the 8x8 grids)",
                     "abs_R_dv_eq_dl_over_R0": curve}

    line = None
    if rank == 0:
        del host_Ms, host_Mm
        peaks, peak_kind = load_peaks()
        peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
        # Consecutive contraction launches run on two streams and overlap, so
        # the kernel's time is the union of its launch intervals (CUDA events
        # on each launching stream): achieved = algorithmic flops of all
        # launches / that busy time = flops per launch / busy time per launch.
        per_launch_ms = prof["contract_ms"] / max(prof["contract_launches"], 1)
        busy_per_launch_ms = prof["contract_busy_ms"] / max(prof["contract_launches"], 1)
        flops_per_launch = prof["contract_flops"] / max(prof["contract_launches"], 1)
        achieved = flops_per_launch / (busy_per_launch_ms / 1000.0) / 1e12
        traffic = None
        tj = load_traffic("herk_tc2_kernel_cov64x64_traffic.json")
        if tj is not None:
            # bytes per event measured by ncu, scaled to this run's events per launch
            ev_per_launch = flops_per_launch / (4.0 * N * (N + 1))
            traffic = tj["dram_bytes_per_event"] * ev_per_launch
        # accuracy on regenerated paths against the GPU's FP64 mode (1e5 paths)
        # and against the FP64 oracle (a small sample)
        na = int(a.accuracy_paths)
        other = "fp16" if a.precision == "mixed" else "mixed"
        M64 = MC.cov_from_args(MC.mc_args(*workload_args(na), seed=seed, precision="fp64", device=local))
        acc = {"paths": na, "tol": 1e-3, "norm": "Frobenius of (Ms, Mm)"}
        for p in (a.precision, other, "fp32"):
            acc[f"rel_err_{p}_vs_fp64"] = rel_err(
                MC.cov_from_args(MC.mc_args(*workload_args(na), seed=seed, precision=p, device=local)), M64)
        del M64
        from oracle import oracle as O
        O.build()
        no = int(a.oracle_paths)
        ho = MC.mc_args(*workload_args(no), seed=seed, precision="fp64", device=local)
        Mo = O.cov(ho, O.Rng.philox(), threads=os.cpu_count() or 1)
        acc["oracle_paths"] = no
        acc["rel_err_fp64_vs_oracle"] = rel_err(MC.cov_from_args(ho), Mo)
        for p in (a.precision, other):
            acc[f"rel_err_{p}_vs_oracle"] = rel_err(
                MC.cov_from_args(MC.mc_args(*workload_args(no), seed=seed, precision=p, device=local)), Mo)
        del Mo
        # the 5x comparison: plain FP32 GPU and both tensor-core precisions on the same sample
        nf = int(a.fp32_paths)
        t32 = time.perf_counter()
        MC.cov_from_args(MC.mc_args(*workload_args(nf), seed=seed, precision="fp32", device=local))
        fp32_s = time.perf_counter() - t32
        tmx = time.perf_counter()
        MC.cov_from_args(MC.mc_args(*workload_args(nf), seed=seed, precision=a.precision, device=local))
        prec_small_s = time.perf_counter() - tmx
        tot = time.perf_counter()
        MC.cov_from_args(MC.mc_args(*workload_args(nf), seed=seed, precision=other, device=local))
        other_small_s = time.perf_counter() - tot
        legs = None
        if world == 1 and a.legs:
            legs = {}
            for name in a.legs.split(","):
                legs[name] = run_leg(Leg(name), a, a.precision, peaks, peak_kind)
                torch.cuda.empty_cache()
        served = None if (a.no_served or world > 1) else run_served_leg(a, local)
        cpu = None
        if not a.no_cpu_baseline:
            rate, n, dt, thr = cpu_oracle_rate(workload_args, target_s=a.cpu_seconds)
            cpu = {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
                   "sample": f"{n} paths of the workload in {dt:.1f} s (oracle MCcov, FP64, {thr} threads)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("f16 hi+lo" if a.precision == "mixed" else "f16") + " x f16 -> f32 (phases f64-reduced f32, sums f64)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "paths_per_gpu_per_step": P, "lights": 64, "views": 64,
                       "output": "Ms, Mm: 64x64x64x64 complex f64", "precision": a.precision,
                       "parallelism": f"path-range shards x{world}" + (" + NCCL sum" if world > 1 else ""),
                       "l2": "working set > L2 (1 GiB operand per chunk, 2 x 268 MB accumulators)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(2 * n_out * 2 * 8)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "herk_tc2_kernel", "peak_source": f"bf16_tflops_sustained ({peak_kind})",
                         "flops_per_launch": flops_per_launch, "busy_ms_per_launch": busy_per_launch_ms,
                         "ms_per_launch_overlapped": per_launch_ms, "contract_busy_ms": prof["contract_busy_ms"],
                         "launches": prof["contract_launches"]},
            "stages_ms": {"walk": prof["walk_ms"], "rows": prof["rows_ms"], "contract": prof["contract_ms"],
                          "finalize": prof["finalize_ms"], "contract_busy": prof["contract_busy_ms"],
                          "rows_busy": prof["rows_busy_ms"], "timed_region": ms_max},
            "accuracy": acc,
            "other_precision": {"precision": other, "paths": nf, "value": nf / other_small_s},
            "fp32_gpu": {"paths": nf, "value": nf / fp32_s, f"{a.precision}_same_sample": nf / prec_small_s,
                         f"speedup_{a.precision}_over_fp32": fp32_s / prec_small_s},
            "memory_effect": memory_effect,
            "workloads": legs,
            "serving": served,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
