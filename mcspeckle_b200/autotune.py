"""The project's autotuner: launch parameters chosen by timing on the GPU.

For one solve shape (kind, precision, size) it times candidate values of the
library's tunables - path-batch size, covariance chunk size and CTA-pair
pipeline stages, split-K of the tensor-core field, FourierQuad plane-group
size - one parameter at a time (coordinate descent from the built-in
choice), each candidate as the median of a few device-timed solves (CUDA
events on the launching stream, after a warm-up solve), and writes the best
values as entries of the tuning file the library reads at its first use
(scmc_tuning.txt beside libscmc_gpu.so, or the file named by
SCMC_TUNING_FILE).  Candidates never exceed the accuracy caps the library
keeps (the covariance chunk), so tuning changes speed, not the error bound.

    python -m mcspeckle_b200.autotune [--out PATH] [--quick]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import _abi, _lib
from . import workloads as WL

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_FILE = os.path.join(HERE, "scmc_tuning.txt")
KIND_NAME = {_abi.SCMC_TUNE_FIELD: "field", _abi.SCMC_TUNE_COV: "cov", _abi.SCMC_TUNE_FQ: "fq"}
PREC_NAME = {v: k for k, v in _abi.PRECISIONS.items()}
FIELDS = ("path_batch", "chunk_events", "stages", "ksplit", "group_entries")


def set_entry(kind, prec, n_lo, n_hi, **vals):
    t = _abi.Tuning(kind=kind, precision=prec, n_lo=n_lo, n_hi=n_hi, **vals)
    _lib.check(_lib.lib().scmc_tuning_set(C.byref(t)))


def clear():
    _lib.check(_lib.lib().scmc_tuning_clear())


def resolved(kind, prec, n):
    t = _abi.Tuning()
    _lib.check(_lib.lib().scmc_tuning_get(kind, prec, n, C.byref(t)))
    return {f: getattr(t, f) for f in FIELDS}


class Shape:
    """One solve shape to tune: a device solve and its size key."""

    def __init__(self, name, kind, prec, n, run, candidates):
        self.name, self.kind, self.prec, self.n, self.run, self.candidates = name, kind, prec, n, run, candidates


def shapes(quick=False):
    import torch
    from . import mc as MC
    L = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    out = []
    n2 = 4096
    Ms = torch.empty(2 * n2 * n2, dtype=torch.float64, device="cuda")
    Mm = torch.empty_like(Ms)
    cov_paths = 1_000_000 if quick else 3_000_000

    def cov_run(prec):
        def run(i):
            h = MC.mc_args(*WL.cov64_args(cov_paths), seed=11, precision=prec, path_offset=i * cov_paths)
            _lib.check(L.scmc_cov_device(h.ref, Ms.data_ptr(), Mm.data_ptr(), st))
        return run
    for prec in ("fp16", "mixed"):
        p = _abi.PRECISIONS[prec]
        # hi+lo: chunks up to the 4096-event default only (its error grows with the chunk)
        cand = {"chunk_events": [16384, 32768, 65536] if prec == "fp16" else [2048, 4096],
                "path_batch": [1 << 19, 1 << 20, 1 << 21]}
        if prec == "fp16":
            cand["stages"] = [2, 3]
        out.append(Shape(f"cov64_{prec}", _abi.SCMC_TUNE_COV, p, n2, cov_run(prec), cand))
    # the tensor-core field at the served stream's large end (1024 views x 256 lights)
    rng = np.random.default_rng(3)
    l = WL.cap_dirs(256, 10.0, +1.0, rng)
    v = WL.cap_dirs(1024, 10.0, -1.0, rng)
    u = torch.empty(2 * 1024 * 256, dtype=torch.float64, device="cuda")
    fpaths = 100_000 if quick else 300_000

    def field_run(i):
        base = [0.101, 1 / 1.01, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]), l, v, 1, 1, fpaths,
                1.0, True, 2, 3, 0.8]
        h = MC.mc_args(*base, seed=12, precision="fp16", path_offset=i * fpaths)
        _lib.check(L.scmc_field_device(h.ref, u.data_ptr(), st))
    out.append(Shape("field1024x256_fp16", _abi.SCMC_TUNE_FIELD, _abi.PRECISIONS["fp16"], 1024 * 256, field_run,
                     {"ksplit": [1, 2, 4, 8], "path_batch": [1 << 18, 1 << 20]}))
    uq = torch.empty(2 * 256 * 256, dtype=torch.float64, device="cuda")
    qpaths = 1_000_000 if quick else 4_000_000

    def fq_run(i):
        h = WL.fq256_args(qpaths, extended=True, seed=13, precision="fp16", path_offset=i * qpaths)
        _lib.check(L.scmc_field_fourier_quad_device(h.ref, uq.data_ptr(), st))
    out.append(Shape("fq256_fp16", _abi.SCMC_TUNE_FQ, _abi.PRECISIONS["fp16"], 256 * 256, fq_run,
                     {"group_entries": [1 << 19, 1 << 20, 1 << 21], "path_batch": [1 << 19, 1 << 20, 1 << 21]}))
    return out


def time_shape(shape, vals, reps):
    import torch
    clear()
    set_entry(shape.kind, shape.prec, shape.n, shape.n, **vals)
    shape.run(0)  # warm-up (allocations grow here)
    torch.cuda.synchronize()
    ts = []
    for i in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        shape.run(i + 1)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def tune(shape, reps=3, log=print):
    """Coordinate descent over the shape's candidates from the built-in choice."""
    best = {k: v for k, v in resolved(shape.kind, shape.prec, shape.n).items() if k in shape.candidates}
    best_ms = time_shape(shape, best, reps)
    trials = [dict(best, ms=best_ms)]
    for name, values in shape.candidates.items():
        for val in values:
            if val == best.get(name):
                continue
            trial = dict(best, **{name: val})
            ms = time_shape(shape, trial, reps)
            trials.append(dict(trial, ms=ms))
            log(f"  {shape.name} {trial} {ms:.2f} ms")
            if ms < best_ms * 0.98:  # keep a change only when it is clearly faster
                best, best_ms = trial, ms
    return best, best_ms, trials


def write_file(path, results):
    lines = ["# scmc tuning entries written by mcspeckle_b200.autotune on the GPU that ran it",
             "# kind precision n_lo n_hi path_batch chunk_events stages ksplit group_entries"]
    for shape, best, ms in results:
        vals = [int(best.get(f, 0)) for f in FIELDS]
        lines.append(f"{KIND_NAME[shape.kind]} {PREC_NAME[shape.prec]} {shape.n} {shape.n} " +
                     " ".join(str(v) for v in vals) + f"   # {shape.name}: {ms:.2f} ms per solve")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_FILE)
    ap.add_argument("--quick", action="store_true", help="smaller solves (a first pass)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--json", default=None, help="also write every trial here")
    a = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    results, report = [], []
    t0 = time.perf_counter()
    for shape in shapes(a.quick):
        best, ms, trials = tune(shape, a.reps)
        print(f"{shape.name}: best {best} {ms:.2f} ms", flush=True)
        results.append((shape, best, ms))
        report.append({"shape": shape.name, "best": best, "best_ms": ms, "trials": trials})
    clear()
    write_file(a.out, results)
    if a.json:
        with open(a.json, "w") as f:
            json.dump({"seconds": time.perf_counter() - t0, "shapes": report}, f, indent=1)
    print(f"wrote {a.out} in {time.perf_counter() - t0:.0f} s")


if __name__ == "__main__":
    main()
