#!/usr/bin/env python
"""Throughput of SCMC's Monte Carlo covariance path on B200.

Workload: the far-field covariance configuration - MCcov on a homogeneous box
20 x 20 x 5 MFP (MFP = 10 wavelengths, wavelength 1), Henyey-Greenstein g=0.8,
sigma_s = 1, sigma_a = 0.01 per MFP, 64 lights and 64 views on regular 8 x 8
(sin theta_x, sin theta_y) grids spanning +-5 degrees about +z / -z
(reflection, CBS on, exponential first-scatter sampling), 1e7 paths per GPU
per step, full 64x64x64x64 complex covariance.  Synthetic: every input is
generated from fixed seeds; each step walks a fresh Philox path range.

One step = one MCcov solve of --paths paths on every GPU (mixed precision:
tcgen05 FP16 hi+lo contraction, FP64 cross-chunk sums), plus for N>1 an
NCCL sum of the partial Ms / Mm.  `value` = paths of all ranks / the max over
ranks of the CUDA-event time of the K timed steps, outputs in HBM.  `e2e` =
the same through the host-buffer C ABI call (scmc_cov: inputs from host,
Ms / Mm copied back to host every step).
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

METRIC = "MC paths/s at 1e-3 rel err vs FP64 (mixed vs FP32 GPU); p50/p99 request latency"
UNIT = "paths/s"
WORKLOAD = "MCcov far-field covariance, 64 lights x 64 views (8x8 grids, +-5 deg), HG g=0.8, box 20x20x5 MFP"


def grid_dirs(n_side, half_deg, zsign):
    s = math.sin(math.radians(half_deg))
    g = np.linspace(-s, s, n_side)
    sx, sy = np.meshgrid(g, g, indexing="ij")
    sx, sy = sx.reshape(-1), sy.reshape(-1)
    return np.stack([sx, sy, zsign * np.sqrt(1 - sx * sx - sy * sy)])


def workload_args(n_paths):
    mfp = 10.0
    sigt = 1.01 / mfp          # sigma_s + sigma_a = (1 + 0.01) / MFP
    albedo = 1.0 / 1.01
    box_min = np.array([-100.0, -100.0, 0.0])
    box_max = np.array([100.0, 100.0, 50.0])
    l = grid_dirs(8, 5.0, +1.0)
    v = grid_dirs(8, 5.0, -1.0)
    return [sigt, albedo, box_min, box_max, l, v, 1, 1, int(n_paths), 1.0, True, 2, 3, 0.8]


# ---------------------------------------------------------------------------
# served stream: uneven MCfield requests with Poisson arrivals
# ---------------------------------------------------------------------------
SERVED_WORKLOAD = ("served MCfield stream: lights 1-256, views 1-1024, paths log-uniform; box 5-50 MFP "
                   "(MFP 10 wavelengths, thickness 1/4 of the side), HG g~U(0,0.95), sigma_a~U(0,0.05), "
                   "isotropic/HG/tabulated 1:2:1, far field, CBS, Poisson arrivals")


def cap_dirs(n, half_deg, zsign, rng):
    """n directions uniform on the solid-angle cap <= half_deg about zsign*z."""
    c = rng.uniform(math.cos(math.radians(half_deg)), 1.0, n)
    phi = rng.uniform(0, 2 * math.pi, n)
    s = np.sqrt(1 - c * c)
    return np.stack([s * np.cos(phi), s * np.sin(phi), zsign * c])


def hg_table(g, n=1001):
    """A tabulated phase function (tabulatedAmplitudeScatter of an HG lobe)."""
    from mcspeckle_b200 import interface as I
    th = np.linspace(0, 1, n) * np.pi
    f = np.sqrt((1 - g * g) / (4 * np.pi * (1 + g * g - 2 * g * np.cos(th)) ** 1.5))
    t = I.tabulatedAmplitudeScatter(th, f)["ampfunc"]
    return {"evalAmp": t["evalAmp"], "sampleIcdf": t["sampleIcdf"]}


def served_requests(n, seed=5, paths=(1e5, 1e8), nv_max=1024, nl_max=256, side_mfp=(5.0, 50.0)):
    """The served stream: n MCfield requests with log-uniform sizes and budgets
    and media drawn per request.  Returns dicts with the positional MCfield
    arguments, the Philox key and the sizes."""
    rng = np.random.default_rng(seed)

    def logu(lo, hi):
        return math.exp(rng.uniform(math.log(lo), math.log(hi)))

    out = []
    mfp = 10.0
    for i in range(n):
        nl = max(1, min(nl_max, int(round(logu(1, nl_max)))))
        nv = max(1, min(nv_max, int(round(logu(1, nv_max)))))
        n_paths = int(round(logu(*paths)))
        side = logu(*side_mfp) * mfp
        g = float(rng.uniform(0.0, 0.95))
        sa = float(rng.uniform(0.0, 0.05))
        kind = ["iso", "hg", "hg", "tab"][int(rng.integers(0, 4))]
        sct, amp = {"iso": (1, 0), "hg": (3, g), "tab": (2, None)}[kind]
        if kind == "tab":
            amp = hg_table(g)
        l = cap_dirs(nl, 10.0, +1.0, rng)
        v = cap_dirs(nv, 10.0, -1.0, rng)
        args = [(1.0 + sa) / mfp, 1.0 / (1.0 + sa), np.array([-side / 2, -side / 2, 0.0]),
                np.array([side / 2, side / 2, side / 4]), l, v, 1, 1, n_paths, 1.0, True, 2, sct, amp]
        out.append({"args": args, "seed": 0x5E4E0000 + i, "paths": n_paths, "nv": nv, "nl": nl, "scatter": kind})
    return out


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
        ready = threading.Event()

        def submitter():
            t0 = time.perf_counter()
            for i, h in enumerate(holders):
                dt = arrive[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                tickets[i] = srv.submit_field(h)
                if i == 0:
                    ready.set()
            ready.set()

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
    return {"requests": len(reqs), "paths": int(paths), "makespan_s": (t1 - t0) / 1000.0,
            "paths_per_s": paths / ((t1 - t0) / 1000.0), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "sum_device_ms": busy}


def run_served_leg(a, device):
    """Served stream at reduced path budgets: closed batch (capacity), then
    Poisson arrivals at 85% of that capacity (latency), then a plain FP32
    one-request-at-a-time pass and the same requests served, on a prefix."""
    from mcspeckle_b200 import mc as MC
    lo, hi = a.served_paths_min, a.served_paths_max
    reqs = served_requests(a.served_requests, paths=(lo, hi))
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
        "workload": SERVED_WORKLOAD, "requests": len(reqs), "paths_range": [lo, hi],
        "path_budget_note": "config budgets 1e5-1e8 scaled to the stated range so the leg runs in about a minute",
        "slots": a.slots, "hbm_budget_gb": 80, "precision": "mixed",
        "closed_batch": closed, "poisson": dict(opened, offered_load=0.85, rate_per_s=rate),
        "peak_reserved_gb": max(st_closed["peak_reserved_bytes"], st_open["peak_reserved_bytes"]) / 1e9,
        "fp32_one_at_a_time": {"requests": k, "paths_per_s": fp32_rate, "seconds": fp32_s},
        "served_same_prefix": {"requests": k, "paths_per_s": served_prefix["paths_per_s"]},
        "speedup_vs_fp32_one_at_a_time": served_prefix["paths_per_s"] / fp32_rate,
    }


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


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
# the other configurations, one JSON line each (`--workload`); the default line
# above is the far-field covariance
# ---------------------------------------------------------------------------
def grid_rect(nx, ny, half_deg, zsign):
    """nx x ny directions on a regular (sin theta_x, sin theta_y) grid."""
    s = math.sin(math.radians(half_deg))
    sx, sy = np.meshgrid(np.linspace(-s, s, nx), np.linspace(-s, s, ny), indexing="ij")
    sx, sy = sx.reshape(-1), sy.reshape(-1)
    return np.stack([sx, sy, zsign * np.sqrt(1 - sx * sx - sy * sy)])


def hg_mixture_table(n_bins, seed):
    """Tabulated amplitude of a seeded mixture of 3 HG lobes (g in [-0.3, 0.95],
    weights from Dirichlet(1,1,1)) on n_bins angles in [0, pi]."""
    from mcspeckle_b200 import interface as I
    g_rng = np.random.default_rng(seed)
    gs = g_rng.uniform(-0.3, 0.95, 3)
    w = g_rng.dirichlet([1.0, 1.0, 1.0])
    th = np.linspace(0, 1, n_bins) * np.pi
    c = np.cos(th)
    pdf = sum(wk * (1 - gk * gk) / (4 * np.pi * (1 + gk * gk - 2 * gk * c) ** 1.5) for wk, gk in zip(w, gs))
    t = I.tabulatedAmplitudeScatter(th, np.sqrt(pdf))["ampfunc"]
    return {"evalAmp": t["evalAmp"], "sampleIcdf": t["sampleIcdf"]}, gs.tolist(), w.tolist()


ACC_MASK = None  # entries excluded from the accuracy comparison of a workload


def workload_spec(name):
    """(description, make(n, precision, seed, offset, norm) -> holder, device solve,
    host solve, output doubles, oracle solve, the tensor-core kernel whose
    roofline is reported or None)."""
    from mcspeckle_b200 import _lib
    from mcspeckle_b200 import mc as MC
    from mcspeckle_b200 import fourier_quad as FQ
    from mcspeckle_b200 import hetero as H
    L = _lib.lib()
    if name == "field16":
        rng = np.random.default_rng(0)
        l16 = cap_dirs(16, 10.0, +1.0, rng)
        v16 = cap_dirs(16, 10.0, -1.0, rng)
        base = [0.1, 1.0, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]), l16, v16, 1, 1, 0,
                1.0, True, 2, 1, 0]

        def make(n, prec, seed, off=0, norm=0):
            b = list(base)
            b[8] = int(n)
            return MC.mc_args(*b, seed=seed, precision=prec, path_offset=off, norm_itr=norm)

        def dev(h, outs, stream):
            _lib.check(L.scmc_field_device(h.ref, outs[0].data_ptr(), stream))

        def oracle(h, O):
            return O.field(h, O.Rng.philox())
        return ("MCfield far field, 16 lights x 16 views within 10 deg of +z / -z, isotropic, box 20x20x5 MFP "
                "(MFP 10 wavelengths), CBS, 1e5 paths per step", make, dev, MC.field_from_args, [2 * 16 * 16],
                oracle, None)
    if name == "fq256":
        mfp = 100.0
        base = dict(sigt=1.005 / mfp, albedo=1 / 1.005, box_min=[-25 * mfp, -25 * mfp, 0.0],
                    box_max=[25 * mfp, 25 * mfp, 10 * mfp], l=np.array([[0.0], [0.0], [1.0]]),
                    v_max=255.0 / 256.0, v_stp=1.0 / 128.0)

        def make(n, prec, seed, off=0, norm=0):
            return FQ.fq_args(base["sigt"], base["albedo"], base["box_min"], base["box_max"], base["l"],
                              base["v_max"], base["v_stp"], int(n), 1.0, True, 2, None, -1, seed=seed,
                              precision=prec, path_offset=off)

        def dev(h, outs, stream):
            _lib.check(L.scmc_field_fourier_quad_device(h.ref, outs[0].data_ptr(), stream))

        def oracle(h, O):
            return O.field_fourier_quad(h.args, O.Rng.philox(), h.nv0)
        th = -base["v_max"] + np.arange(256) * base["v_stp"]
        # accuracy over the propagating directions only: where vx^2 + vy^2 > 1 the
        # reference's plane factor grows exponentially with depth (evanescent)
        global ACC_MASK
        ACC_MASK = (th[:, None] ** 2 + th[None, :] ** 2 < 1.0)[:, :, None]
        return ("MCfieldFourierQuad, box 50x50x10 MFP (MFP 100 wavelengths), sigma_a 0.005 per MFP, plane wave "
                "along +z, 256x256 angular grid (v_max 255/256, v_stp 1/128: 0.5-wavelength lateral pitch), CBS; "
                "isotropic as the reference (HG g=0.9 and the point source are not built)",
                make, dev, FQ.field_fourier_quad_from_args, [2 * 256 * 256], oracle, "fq_planes_tc_kernel")
    if name == "hetero128":
        mfp = 10.0
        g = np.random.default_rng(4)
        sig = np.exp(g.normal(0.0, 0.5, (128, 128, 128))) / mfp
        table, gs, ws = hg_mixture_table(1024, 5)
        bmin, bmax = np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0])
        bbin = (bmax - bmin) / 128.0
        l = grid_rect(16, 8, 5.0, +1.0)
        v = grid_rect(16, 8, 5.0, -1.0)

        def make(n, prec, seed, off=0, norm=0):
            return H.hetero_args(True, sig, 1.0, bmin, bmax, bbin, l, v, 1, 1, int(n), 1.0, True, 2, 2, table,
                                 seed=seed, precision=prec, path_offset=off, norm_itr=norm)

        def dev(h, outs, stream):
            _lib.check(L.scmc_cov_hetero_device(h.ref, outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                                stream))

        def oracle(h, O):
            return O.cov_hetero(h, O.Rng.philox(), threads=os.cpu_count() or 1)[:2]
        n2 = 128 * 128
        return (f"MCCovHetro, sigma_s on a 128^3 grid log-normal(0, 0.5) per MFP (MFP 10 wavelengths, nearest "
                f"voxel as the reference), box 20x20x5 MFP, Woodcock tracking, tabulated phase function on 1024 "
                f"theta bins from 3 HG lobes g={[round(x, 3) for x in gs]} w={[round(x, 3) for x in ws]}, "
                f"128 lights x 128 views (16x8 grids of +-5 deg), CBS",
                make, dev, lambda h: H.cov_hetero_from_args(h)[:2], [2 * n2 * n2, 2 * n2 * n2, 2 * n2], oracle,
                "herk_tc2_kernel")
    raise SystemExit(f"unknown workload {name}")


def run_workload(a):
    """One JSON line for a non-default configuration, 1 GPU: device-timed
    steps of fresh path ranges (outputs in HBM), the host-buffer call, stage
    times, accuracy against FP64 on a smaller sample, the CPU oracle on a
    bounded sample."""
    import torch
    from mcspeckle_b200 import _lib
    desc, make, dev, host, sizes, oracle_fn, bound = workload_spec(a.workload)
    prec = a.precision
    P = int(a.paths if a.paths is not None else {"field16": 1e5, "fq256": 1e5, "hetero128": 2e4}[a.workload])
    stream = torch.cuda.current_stream()
    outs = [torch.zeros(n, dtype=torch.float64, device="cuda") for n in sizes]
    seed = 0

    def step(i):
        dev(make(P, prec, seed, off=i * P, norm=P), outs, stream.cuda_stream)

    for i in range(a.warmup):
        step(i)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
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
    value = P * a.steps / (ms / 1000.0)
    # e2e: the host-buffer call (results copied to host every step)
    t0 = time.perf_counter()
    for i in range(a.steps):
        host(make(P, prec, seed, off=(a.warmup + a.steps + i) * P, norm=P))
    e2e = P * a.steps / (time.perf_counter() - t0)
    # accuracy on a smaller sample, same paths in every precision
    na = int(a.accuracy_paths if a.accuracy_paths is not None else
             {"field16": 1e5, "fq256": 2e4, "hetero128": 1e3}[a.workload])
    ref = host(make(na, "fp64", 7))
    ref = ref if isinstance(ref, tuple) else (ref,)

    def rel(x):
        x = x if isinstance(x, tuple) else (x,)
        num = den = 0.0
        for xa, ra in zip(x, ref):
            m = np.isfinite(ra) if ACC_MASK is None else np.broadcast_to(ACC_MASK, ra.shape)
            num += float(np.linalg.norm((xa - ra)[m])) ** 2
            den += float(np.linalg.norm(ra[m])) ** 2
        return math.sqrt(num / den)
    acc = {"paths": na, "tol": 1e-3}
    for pz in ("mixed", "fp16", "fp32"):
        acc[f"rel_err_{pz}_vs_fp64"] = rel(host(make(na, pz, 7)))
    # plain FP32 GPU, one solve, same paths as one timed step
    t32 = time.perf_counter()
    host(make(P, "fp32", seed))
    fp32_value = P / (time.perf_counter() - t32)
    roof = None
    if bound is not None and prof["contract_launches"]:
        peaks, peak_kind = load_peaks()
        peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
        achieved = prof["contract_flops"] / (prof["contract_busy_ms"] / 1000.0) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "kernel": bound, "peak_source": f"bf16_tflops_sustained ({peak_kind})",
                "flops": prof["contract_flops"], "contract_busy_ms": prof["contract_busy_ms"]}
    cpu = None
    if not a.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        n = {"field16": 2000, "fq256": 20, "hetero128": 16}[a.workload]
        h = make(n, "fp64", 99)
        tc = time.perf_counter()
        oracle_fn(h, O)
        dt = time.perf_counter() - tc
        thr = (os.cpu_count() or 1) if a.workload == "hetero128" else 1
        cpu = {"value": n / dt, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"{n} paths of the workload in {dt:.1f} s (FP64 oracle, {thr} thread(s))"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": prec, "data": "synthetic",
            "config": {"workload": a.workload, "description": desc, "paths_per_step": P, "precision": prec},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": None,
                    "d2h_bytes_per_step": int(sum(sizes) * 8)},
            "gpu_launches": int(launches), "roofline": roof,
            "stages_ms": {k: prof[k] for k in ("walk_ms", "rows_ms", "contract_ms", "finalize_ms",
                                               "contract_busy_ms", "rows_busy_ms")},
            "accuracy": acc, "fp32_gpu": {"paths": P, "value": fp32_value}, "cpu_baseline": cpu, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--paths", type=float, default=None, help="paths per GPU per step (cov64: 1e7)")
    ap.add_argument("--accuracy-paths", type=float, default=None, help="(cov64: 1e5)")
    ap.add_argument("--fp32-paths", type=float, default=1e5)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp16", choices=["mixed", "fp16"],
                    help="mixed: FP16 hi+lo split (2 tensor products); fp16: one FP16 product")
    ap.add_argument("--served-requests", type=int, default=200)
    ap.add_argument("--served-paths-min", type=float, default=1e4)
    ap.add_argument("--served-paths-max", type=float, default=1e7)
    ap.add_argument("--served-fp32-seconds", type=float, default=20.0)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--workload", default="cov64", choices=["cov64", "field16", "fq256", "hetero128"],
                    help="cov64: the far-field covariance (the default line); the others print one line of "
                         "their own (1 GPU): field16, fq256, hetero128")
    a = ap.parse_args()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload != "cov64":
        import torch
        torch.cuda.set_device(0)
        return run_workload(a)
    a.paths = 1e7 if a.paths is None else a.paths
    a.accuracy_paths = 1e5 if a.accuracy_paths is None else a.accuracy_paths

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
    clocks = ClockSampler(local)
    clocks.start()
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

    line = None
    if rank == 0:
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
        tf = os.path.join(ROOT, "profiles", "herk_tc2_kernel_cov64x64_traffic.json")
        if os.path.exists(tf):
            with open(tf) as f:
                tj = json.load(f)
            # bytes per event measured by ncu, scaled to this run's events per launch
            ev_per_launch = flops_per_launch / (4.0 * N * (N + 1))
            traffic = tj["dram_bytes_per_event"] * ev_per_launch
        # accuracy on regenerated paths: mixed and plain FP32 against FP64
        na = int(a.accuracy_paths)
        ha = MC.mc_args(*workload_args(na), seed=seed, precision="fp64", device=local)
        M64 = MC.cov_from_args(ha)
        Mmx = MC.cov_from_args(MC.mc_args(*workload_args(na), seed=seed, precision=a.precision, device=local))
        other = "fp16" if a.precision == "mixed" else "mixed"
        Moth = MC.cov_from_args(MC.mc_args(*workload_args(na), seed=seed, precision=other, device=local))
        t32 = time.perf_counter()
        M32 = MC.cov_from_args(MC.mc_args(*workload_args(int(a.fp32_paths)), seed=seed, precision="fp32",
                                          device=local))
        fp32_s = time.perf_counter() - t32
        if int(a.fp32_paths) != na:
            M32 = MC.cov_from_args(MC.mc_args(*workload_args(na), seed=seed, precision="fp32", device=local))
        C64 = M64[0] + M64[1]

        def rel(x, y):
            return float(np.linalg.norm((x - y).ravel()) / np.linalg.norm(y.ravel()))

        err_mixed = rel(Mmx[0] + Mmx[1], C64)
        err_fp32 = rel(M32[0] + M32[1], C64)
        err_other = rel(Moth[0] + Moth[1], C64)
        tmx = time.perf_counter()
        MC.cov_from_args(MC.mc_args(*workload_args(int(a.fp32_paths)), seed=seed, precision=a.precision,
                                    device=local))
        mixed_small_s = time.perf_counter() - tmx
        tot = time.perf_counter()
        MC.cov_from_args(MC.mc_args(*workload_args(int(a.fp32_paths)), seed=seed, precision=other, device=local))
        other_small_s = time.perf_counter() - tot
        served = None if a.no_served else run_served_leg(a, local)
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
            "accuracy": {"paths": na, f"rel_err_{a.precision}_vs_fp64": err_mixed,
                         f"rel_err_{other}_vs_fp64": err_other, "rel_err_fp32_vs_fp64": err_fp32,
                         "tol": 1e-3, "norm": "Frobenius of C = Ms + Mm"},
            "other_precision": {"precision": other, "paths": int(a.fp32_paths),
                                "value": int(a.fp32_paths) / other_small_s},
            "fp32_gpu": {"paths": int(a.fp32_paths), "value": int(a.fp32_paths) / fp32_s,
                         "mixed_same_sample": int(a.fp32_paths) / mixed_small_s,
                         "speedup_mixed_over_fp32": (int(a.fp32_paths) / mixed_small_s) / (int(a.fp32_paths) / fp32_s)},
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
