"""ctypes mirror of include/scmc_gpu.h (structs and status codes).

The structs carry the positional arguments of MCfield / MCcov /
MCfieldFourierQuad (code/MCfield.m:1, code/MCcov.m:1,
code/MCfieldFourierQuad.m:1) plus execution controls.  `McArgs.build`
keeps every numpy buffer it points at alive on the returned object.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

SCMC_OK = 0
SCMC_ERR_INVALID = 1
SCMC_ERR_CUDA = 2
SCMC_ERR_NOMEM = 3
SCMC_ERR_NODEVICE = 4
SCMC_ERR_TIMEOUT = 5
SCMC_ERR_CANCELLED = 6
SCMC_ERR_LIMIT = 7

SCT_ISOTROPIC, SCT_TABULATED, SCT_HG = 1, 2, 3
PREC_FP64, PREC_MIXED, PREC_FP32, PREC_FP16 = 0, 1, 2, 3
PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED, "fp32": PREC_FP32, "fp16": PREC_FP16}

_dp = C.POINTER(C.c_double)


class PhaseFunction(C.Structure):
    _fields_ = [
        ("sct_type", C.c_int32),
        ("g", C.c_double),
        ("table_n", C.c_int32),
        ("eval_amp", _dp),
        ("sample_icdf", _dp),
        ("table_in_cos", C.c_int32),
    ]


class McArgs(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("sigt", C.c_double),
        ("albedo", C.c_double),
        ("box_min", C.c_double * 3),
        ("box_max", C.c_double * 3),
        ("l", _dp),
        ("nl", C.c_int64),
        ("v", _dp),
        ("nv", C.c_int64),
        ("is_ff_l", C.c_int32),
        ("is_ff_v", C.c_int32),
        ("max_itr", C.c_int64),
        ("lambda_", C.c_double),
        ("do_cbs", C.c_int32),
        ("smp_flg", C.c_int32),
        ("ampfunc", PhaseFunction),
        ("has_ampfunc0", C.c_int32),
        ("ampfunc0", PhaseFunction),
        ("has_lmean0", C.c_int32),
        ("lmean0", C.c_double * 3),
        ("seed", C.c_uint64),
        ("path_offset", C.c_uint64),
        ("norm_itr", C.c_int64),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("max_events_per_path", C.c_int64),
    ]


class FqArgs(C.Structure):
    _fields_ = [
        ("sigt", C.c_double),
        ("albedo", C.c_double),
        ("box_min", C.c_double * 3),
        ("box_max", C.c_double * 3),
        ("l", _dp),
        ("nl", C.c_int64),
        ("v_max", C.c_double),
        ("v_stp", C.c_double),
        ("max_itr", C.c_int64),
        ("lambda_", C.c_double),
        ("do_cbs", C.c_int32),
        ("smp_flg", C.c_int32),
        ("has_lmean0", C.c_int32),
        ("lmean0", C.c_double * 3),
        ("vsign", C.c_double),
        ("seed", C.c_uint64),
        ("path_offset", C.c_uint64),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("light_point", C.c_int32),
        ("sct_type", C.c_int32),
        ("g", C.c_double),
    ]


SCMC_TUNE_FIELD, SCMC_TUNE_COV, SCMC_TUNE_FQ = 0, 1, 2


class Tuning(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("precision", C.c_int32),
        ("n_lo", C.c_int64),
        ("n_hi", C.c_int64),
        ("path_batch", C.c_int64),
        ("chunk_events", C.c_int64),
        ("stages", C.c_int32),
        ("ksplit", C.c_int32),
        ("group_entries", C.c_int64),
    ]


class HeteroArgs(C.Structure):
    _fields_ = [
        ("mc", McArgs),
        ("sigt_grid", _dp),
        ("albedo_grid", _dp),
        ("box_bin", C.c_double * 3),
        ("has_lrad", C.c_int32),
        ("lrad", C.c_double),
        ("null_basis", C.c_double * 6),
        ("trilinear", C.c_int32),
    ]


class StageTimes(C.Structure):
    _fields_ = [
        ("walk_launches", C.c_int64),
        ("walk_ms", C.c_double),
        ("rows_launches", C.c_int64),
        ("rows_ms", C.c_double),
        ("contract_launches", C.c_int64),
        ("contract_ms", C.c_double),
        ("finalize_launches", C.c_int64),
        ("finalize_ms", C.c_double),
        ("paths", C.c_int64),
        ("events", C.c_int64),
        ("contract_flops", C.c_double),
        ("contract_busy_ms", C.c_double),
        ("rows_busy_ms", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


SCMC_REQ_FIELD = 0
SCMC_REQ_COV = 1


class RequestInfo(C.Structure):
    """scmc_request_info: one served request's timeline and memory."""
    _fields_ = [
        ("ticket", C.c_int64),
        ("kind", C.c_int32),
        ("slot", C.c_int32),
        ("status", C.c_int32),
        ("finished", C.c_int32),
        ("submit_ms", C.c_double),
        ("start_ms", C.c_double),
        ("done_ms", C.c_double),
        ("device_ms", C.c_double),
        ("reserved_bytes", C.c_int64),
        ("peak_bytes", C.c_int64),
        ("paths", C.c_int64),
        ("packed", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    """scmc_server_stats."""
    _fields_ = [
        ("n_slots", C.c_int32),
        ("busy_slots", C.c_int32),
        ("queued", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("budget_bytes", C.c_int64),
        ("reserved_bytes", C.c_int64),
        ("peak_reserved_bytes", C.c_int64),
        ("paths_completed", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class ScatterSpec:
    """One (sct_type, ampfunc) pair in C form.

    `ampfunc` is 0 (isotropic), a scalar g (HG) or a mapping with the
    `evalAmp` and `sampleIcdf` tables of tabulatedAmplitudeScatter.m:78-99
    (with `cosBins` true: tables on cos(theta) bins, the extension of
    interface.tabulatedAmplitudeScatterCos).
    """

    def __init__(self, sct_type: int, ampfunc):
        self.sct_type = int(sct_type)
        self.g = 0.0
        self.eval_amp = None
        self.sample_icdf = None
        self.cos_bins = 0
        if self.sct_type == SCT_HG:
            self.g = float(np.asarray(ampfunc).reshape(-1)[0])
        elif self.sct_type == SCT_TABULATED:
            ea = np.asarray(_field(ampfunc, "evalAmp")).reshape(-1).astype(np.complex128)
            ic = np.asarray(_field(ampfunc, "sampleIcdf"), dtype=np.float64).reshape(-1)
            if ea.size != ic.size or ea.size < 2:
                raise ValueError("tabulated ampfunc needs evalAmp and sampleIcdf of equal length >= 2")
            self.eval_amp = np.ascontiguousarray(ea.view(np.float64))
            self.sample_icdf = np.ascontiguousarray(ic)
            try:
                self.cos_bins = int(bool(np.asarray(_field(ampfunc, "cosBins")).reshape(-1)[0]))
            except (KeyError, AttributeError, TypeError, IndexError):
                self.cos_bins = 0
        elif self.sct_type != SCT_ISOTROPIC:
            raise ValueError("sct_type must be 1, 2 or 3")

    def fill(self, pf: PhaseFunction) -> None:
        pf.sct_type = self.sct_type
        pf.g = self.g
        if self.eval_amp is not None:
            pf.table_n = self.sample_icdf.size
            pf.eval_amp = _ptr(self.eval_amp)
            pf.sample_icdf = _ptr(self.sample_icdf)
            pf.table_in_cos = self.cos_bins
        else:
            pf.table_n = 0


def _field(obj, name):
    if isinstance(obj, dict):
        return obj[name]
    return getattr(obj, name)


class ArgsHolder:
    """An McArgs plus the numpy buffers it points into."""

    def __init__(self, args, keep):
        self.args = args
        self._keep = keep

    @property
    def ref(self):
        return C.byref(self.args)


def build_mc_args(*, dim, sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v,
                  max_itr, lam, do_cbs, smp_flg, scatter: ScatterSpec,
                  scatter0: ScatterSpec | None = None, lmean0=None, seed=0,
                  path_offset=0, norm_itr=0, precision=PREC_FP64, device=0,
                  max_events_per_path=0) -> ArgsHolder:
    a = McArgs()
    l = _f64(np.asarray(l, dtype=np.float64).reshape(dim, -1, order="F").T.copy())  # row per column
    v = _f64(np.asarray(v, dtype=np.float64).reshape(dim, -1, order="F").T.copy())
    a.dim = dim
    a.sigt = float(sigt)
    a.albedo = float(albedo)
    bmin = np.asarray(box_min, dtype=np.float64).reshape(-1)
    bmax = np.asarray(box_max, dtype=np.float64).reshape(-1)
    for k in range(dim):
        a.box_min[k] = bmin[k]
        a.box_max[k] = bmax[k]
    a.l = _ptr(l)
    a.nl = l.shape[0]
    a.v = _ptr(v)
    a.nv = v.shape[0]
    a.is_ff_l = int(bool(is_ff_l))
    a.is_ff_v = int(bool(is_ff_v))
    a.max_itr = int(max_itr)
    a.lambda_ = float(lam)
    a.do_cbs = int(bool(do_cbs))
    a.smp_flg = int(smp_flg)
    scatter.fill(a.ampfunc)
    keep = [l, v, scatter]
    if scatter0 is not None:
        a.has_ampfunc0 = 1
        scatter0.fill(a.ampfunc0)
        keep.append(scatter0)
    if lmean0 is not None:
        lm = np.asarray(lmean0, dtype=np.float64).reshape(-1)
        a.has_lmean0 = 1
        for k in range(dim):
            a.lmean0[k] = lm[k]
    a.seed = int(seed) & (2**64 - 1)
    a.path_offset = int(path_offset)
    a.norm_itr = int(norm_itr)
    a.precision = int(precision)
    a.device = int(device)
    a.max_events_per_path = int(max_events_per_path)
    return ArgsHolder(a, keep)
