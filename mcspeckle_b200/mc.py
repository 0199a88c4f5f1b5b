"""MCfield / MCcov with the reference's positional signatures, on the GPU.

    u       = MCfield(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v,
                      maxItr, lambda_, doCBS, smpFlg, sct_type, ampfunc
                      [, ampfunc0 [, lmean0]])               (code/MCfield.m:1)
    Ms, Mm  = MCcov(... same 14 [, ampfunc0])                 (code/MCcov.m:1)

Argument checks and conversions follow code/MCfield.m:41-69 (box size, 2-D
angle rows converted to [sin; cos], error strings verbatim).  The Philox key
is drawn from this module's global stream, which `rng(seed)` resets, so a
seeded call is reproducible as `rng(seed)` makes a MATLAB run (scmc.m:328-330).
GPU knobs (precision, device, event cap) are keyword-only; they have no slot
in the reference's positional lists.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _lib
from ._abi import ArgsHolder, ScatterSpec, build_mc_args

_MISSING = object()
_stream = np.random.default_rng()
DEFAULT_PRECISION = "mixed"


class MatlabStyleError(ValueError):
    """Input validation error; the message is the reference's error() text."""


def rng(seed) -> None:
    """Seed the stream the Philox keys are drawn from (MATLAB's rng(seed))."""
    global _stream
    _stream = np.random.default_rng(int(seed))


def draw_seed() -> int:
    return int(_stream.integers(0, 2**63 - 1, dtype=np.int64))


def _as_matrix(a) -> np.ndarray:
    """numpy value -> 2-D array with MATLAB's row-vector convention for 1-D."""
    x = np.asarray(a)
    if x.ndim == 0:
        return x.reshape(1, 1)
    if x.ndim == 1:
        return x.reshape(1, -1)
    return x


def _box(box_min, box_max):
    bmin = _as_matrix(np.asarray(box_min, dtype=float))
    bmax = _as_matrix(np.asarray(box_max, dtype=float))
    # a 1-D box is accepted as the column MATLAB code passes
    if np.asarray(box_min).ndim == 1:
        bmin = bmin.T
    if np.asarray(box_max).ndim == 1:
        bmax = bmax.T
    if (bmax.size not in (2, 3)) or bmax.shape[1] != 1 or bmax.shape != bmin.shape:
        raise MatlabStyleError("Invalid box size")  # MCfield.m:44-47
    return bmin[:, 0].copy(), bmax[:, 0].copy()


def _sources(a, dim, what):
    x = _as_matrix(np.asarray(a, dtype=float))
    if x.shape[0] != dim:
        if dim == 2 and x.shape[0] == 1:
            x = np.vstack([np.sin(x), np.cos(x)])  # MCfield.m:52-58
        else:
            raise MatlabStyleError(f"Invalid {what} source input")
    return x


def _scatter(sct_type, ampfunc) -> ScatterSpec:
    st = int(np.asarray(sct_type).reshape(-1)[0])
    if st == 1:
        return ScatterSpec(1, 0)
    if st == 3:
        return ScatterSpec(3, ampfunc)
    if st == 2:
        return ScatterSpec(2, ampfunc)
    raise MatlabStyleError("sct_type must be 1, 2 or 3")


def mc_args(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, maxItr, lambda_, doCBS, smpFlg,
            sct_type, ampfunc, ampfunc0=_MISSING, lmean0=_MISSING, *, seed=None, precision=DEFAULT_PRECISION,
            device=0, path_offset=0, norm_itr=0, max_events_per_path=0) -> ArgsHolder:
    """Validate and convert MCfield/MCcov arguments into the C argument struct."""
    bmin, bmax = _box(box_min, box_max)
    dim = bmin.size
    L = _sources(l, dim, "light")
    V = _sources(v, dim, "view")
    sc = _scatter(sct_type, ampfunc)
    sc0 = None if ampfunc0 is _MISSING else _scatter(sct_type, ampfunc0)
    lm = None if lmean0 is _MISSING or lmean0 is None else np.asarray(lmean0, dtype=float).reshape(-1)
    prec = _abi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    return build_mc_args(dim=dim, sigt=float(np.asarray(sigt).reshape(-1)[0]),
                         albedo=float(np.asarray(albedo).reshape(-1)[0]), box_min=bmin, box_max=bmax,
                         l=L, v=V, is_ff_l=bool(np.asarray(is_ff_l).reshape(-1)[0]),
                         is_ff_v=bool(np.asarray(is_ff_v).reshape(-1)[0]),
                         max_itr=int(np.asarray(maxItr).reshape(-1)[0]),
                         lam=float(np.asarray(lambda_).reshape(-1)[0]),
                         do_cbs=bool(np.asarray(doCBS).reshape(-1)[0]),
                         smp_flg=int(np.asarray(smpFlg).reshape(-1)[0]), scatter=sc, scatter0=sc0,
                         lmean0=lm, seed=draw_seed() if seed is None else seed, path_offset=path_offset,
                         norm_itr=norm_itr, precision=prec, device=device,
                         max_events_per_path=max_events_per_path)


def field_from_args(h: ArgsHolder) -> np.ndarray:
    a = h.args
    u = np.zeros(2 * a.nv * a.nl)
    _lib.check(_lib.lib().scmc_field(h.ref, u.ctypes.data_as(C.POINTER(C.c_double))))
    return u.view(np.complex128).reshape(a.nv, a.nl, order="F")


def field_onwave_from_args(h: ArgsHolder, Wl) -> np.ndarray:
    a = h.args
    w = np.ascontiguousarray(np.asarray(Wl, dtype=np.complex128).reshape(-1))
    if w.size != a.nl:
        raise MatlabStyleError("Wl needs one weight per light")
    u = np.zeros(2 * a.nv)
    dp = C.POINTER(C.c_double)
    _lib.check(_lib.lib().scmc_field_onwave(h.ref, w.view(np.float64).ctypes.data_as(dp), u.ctypes.data_as(dp)))
    return u.view(np.complex128).reshape(a.nv, 1)


def cov_from_args(h: ArgsHolder):
    a = h.args
    n = a.nv * a.nv * a.nl * a.nl
    Ms = np.zeros(2 * n)
    Mm = np.zeros(2 * n)
    dp = C.POINTER(C.c_double)
    _lib.check(_lib.lib().scmc_cov(h.ref, Ms.ctypes.data_as(dp), Mm.ctypes.data_as(dp)))
    shp = (a.nv, a.nv, a.nl, a.nl)
    return Ms.view(np.complex128).reshape(shp, order="F"), Mm.view(np.complex128).reshape(shp, order="F")


def MCfield(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, maxItr, lambda_, doCBS, smpFlg,
            sct_type, ampfunc, ampfunc0=_MISSING, lmean0=_MISSING, **gpu):
    """Speckle field u (Nv x Nl), as code/MCfield.m:1-254."""
    return field_from_args(mc_args(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, maxItr, lambda_,
                                   doCBS, smpFlg, sct_type, ampfunc, ampfunc0, lmean0, **gpu))


def MCcov(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, maxItr, lambda_, doCBS, smpFlg,
          sct_type, ampfunc, ampfunc0=_MISSING, **gpu):
    """Single- and multiple-scattering covariances Ms, Mm (Nv x Nv x Nl x Nl), as code/MCcov.m:1-299."""
    return cov_from_args(mc_args(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, maxItr, lambda_,
                                 doCBS, smpFlg, sct_type, ampfunc, ampfunc0, **gpu))


def MCfieldOnWave(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, maxItr, lambda_, doCBS, smpFlg,
                  sct_type, ampfunc, ampfunc0, lmean0, Wl, **gpu) -> np.ndarray:
    """Field of the lights combined with complex weights Wl (MCfieldOnWave.m:1-267): Nv x 1."""
    return field_onwave_from_args(mc_args(sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, maxItr, lambda_,
                                          doCBS, smpFlg, sct_type, ampfunc, ampfunc0, lmean0, **gpu), Wl)


class Records:
    """Per-event path records exported from the GPU walk (scmc_export_records)."""

    def __init__(self, cap):
        self.x = np.zeros(3 * cap)
        self.ow = np.zeros(3 * cap)
        self.x1 = np.zeros(3 * cap)
        self.w1 = np.zeros(3 * cap)
        self.wpx = np.zeros(cap)
        self.xi = np.zeros(cap)
        self.plen = np.zeros(cap, dtype=np.int32)
        self.path = np.zeros(cap, dtype=np.int64)
        self.n = 0

    def pointers(self):
        dp = C.POINTER(C.c_double)
        return (self.x.ctypes.data_as(dp), self.ow.ctypes.data_as(dp), self.x1.ctypes.data_as(dp),
                self.w1.ctypes.data_as(dp), self.wpx.ctypes.data_as(dp), self.xi.ctypes.data_as(dp),
                self.plen.ctypes.data_as(C.POINTER(C.c_int32)), self.path.ctypes.data_as(C.POINTER(C.c_int64)))

    def truncate(self, n):
        self.n = n
        for k in ("x", "ow", "x1", "w1"):
            setattr(self, k, getattr(self, k)[: 3 * n].copy())
        for k in ("wpx", "xi", "plen", "path"):
            setattr(self, k, getattr(self, k)[:n].copy())
        return self


def export_records(h: ArgsHolder, want_phase: bool, capacity: int) -> Records:
    r = Records(capacity)
    n = C.c_int64(0)
    st = _lib.lib().scmc_export_records(h.ref, int(want_phase), capacity, *r.pointers(), C.byref(n))
    if st == _abi.SCMC_ERR_LIMIT and n.value > capacity:
        return export_records(h, want_phase, int(n.value))
    _lib.check(st)
    return r.truncate(n.value)


def philox_stream(seed: int, path: int, tag: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    _lib.check(_lib.lib().scmc_philox_stream(seed, path, tag, n, out.ctypes.data_as(C.POINTER(C.c_double))))
    return out
