"""ctypes front end of oracle/libscmc_oracle.so (test infrastructure only).

The C library restates code/MCfield.m, code/MCcov.m and
code/MCfieldFourierQuad.m in FP64.  Random numbers come either from tapes
(the draws a MATLAB run consumed, in order) or from the per-path Philox
streams the GPU walk uses.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mcspeckle_b200._abi import ArgsHolder, FqArgs, HeteroArgs

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libscmc_oracle.so")
_lib = None

TAPE, PHILOX = 0, 1


class RngSpec(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("utape", C.POINTER(C.c_double)),
        ("un", C.c_int64),
        ("ntape", C.POINTER(C.c_double)),
        ("nn", C.c_int64),
        ("used_u", C.c_int64),
        ("used_n", C.c_int64),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        lp = C.POINTER(C.c_int64)
        _lib.oracle_field.argtypes = [C.c_void_p, C.POINTER(RngSpec), dp]
        _lib.oracle_cov.argtypes = [C.c_void_p, C.POINTER(RngSpec), dp, dp, C.c_int]
        _lib.oracle_field_onwave.argtypes = [C.c_void_p, dp, C.POINTER(RngSpec), dp]
        _lib.oracle_records.argtypes = [C.c_void_p, C.POINTER(RngSpec), C.c_int32, C.c_int64,
                                        dp, dp, dp, dp, dp, dp, ip, lp, lp]
        _lib.oracle_field_from_records.argtypes = [C.c_void_p, C.c_int64, dp, dp, dp, dp, dp, dp, ip, dp]
        _lib.oracle_cov_from_records.argtypes = [C.c_void_p, C.c_int64, dp, dp, dp, dp, dp, ip,
                                                 dp, dp, C.c_int]
        _lib.oracle_cov_hetero.argtypes = [C.POINTER(HeteroArgs), C.POINTER(RngSpec), dp, dp, dp, C.c_int]
        _lib.oracle_field_hetero.argtypes = [C.POINTER(HeteroArgs), C.POINTER(RngSpec), dp]
        _lib.oracle_field_fourier_quad.argtypes = [C.POINTER(FqArgs), C.POINTER(RngSpec), dp]
        _lib.oracle_field_fourier_quad_onwave.argtypes = [C.POINTER(FqArgs), dp, C.c_int32, C.POINTER(RngSpec), dp]
        _lib.oracle_refocus_grid.argtypes = [C.c_int32, dp, dp, dp, lp]
        _lib.oracle_refocus_grid.restype = C.c_int64
        _lib.oracle_refocus.argtypes = [dp, dp, C.c_int64, C.c_int32, dp, dp, dp, dp, C.c_double, C.c_int32, dp]
        _lib.oracle_sample_cov.argtypes = [dp, C.c_int64, C.c_int64, dp, dp]
        _lib.oracle_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                              C.POINTER(C.c_uint32)]
        _lib.oracle_philox_stream.argtypes = [C.c_uint64, C.c_uint64, C.c_int32, C.c_int64, dp]
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Rng:
    """Random source for one oracle call; keeps its tapes alive."""

    def __init__(self, mode=PHILOX, utape=None, ntape=None):
        self.spec = RngSpec()
        self.spec.mode = mode
        self._u = None if utape is None else np.ascontiguousarray(utape, dtype=np.float64)
        self._n = None if ntape is None else np.ascontiguousarray(ntape, dtype=np.float64)
        if self._u is not None:
            self.spec.utape = _dp(self._u)
            self.spec.un = self._u.size
        if self._n is not None:
            self.spec.ntape = _dp(self._n)
            self.spec.nn = self._n.size

    @classmethod
    def tape(cls, utape, ntape):
        return cls(TAPE, utape, ntape)

    @classmethod
    def philox(cls):
        return cls(PHILOX)


def _check(rc, what):
    if rc == -1:
        raise RuntimeError(f"{what}: random tape exhausted")
    if rc == -3:
        raise RuntimeError(f"{what}: path exceeded max_events_per_path")
    if rc != 0:
        raise RuntimeError(f"{what}: oracle returned {rc}")


def field(h: ArgsHolder, rng: Rng) -> np.ndarray:
    a = h.args
    u = np.zeros(2 * a.nv * a.nl)
    _check(lib().oracle_field(C.addressof(a), C.byref(rng.spec), _dp(u)), "oracle_field")
    return u.view(np.complex128).reshape(a.nv, a.nl, order="F")


def field_onwave(h: ArgsHolder, Wl, rng: Rng) -> np.ndarray:
    """MCfieldOnWave.m: the field of the lights combined with weights Wl (nl complex)."""
    a = h.args
    w = np.ascontiguousarray(np.asarray(Wl, dtype=np.complex128).reshape(-1))
    if w.size != a.nl:
        raise ValueError("Wl needs one weight per light")
    wd = w.view(np.float64)
    u = np.zeros(2 * a.nv)
    _check(lib().oracle_field_onwave(C.addressof(a), _dp(wd), C.byref(rng.spec), _dp(u)), "oracle_field_onwave")
    return u.view(np.complex128).reshape(a.nv, 1)


def cov(h: ArgsHolder, rng: Rng, threads: int = 1):
    a = h.args
    n = a.nv * a.nv * a.nl * a.nl
    Ms = np.zeros(2 * n)
    Mm = np.zeros(2 * n)
    _check(lib().oracle_cov(C.addressof(a), C.byref(rng.spec), _dp(Ms), _dp(Mm), threads), "oracle_cov")
    shp = (a.nv, a.nv, a.nl, a.nl)
    return (Ms.view(np.complex128).reshape(shp, order="F"),
            Mm.view(np.complex128).reshape(shp, order="F"))


class Records:
    """Per-event path records (layout of scmc_export_records)."""

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

    def truncate(self, n):
        self.n = n
        for k in ("x", "ow", "x1", "w1"):
            setattr(self, k, getattr(self, k)[: 3 * n].copy())
        for k in ("wpx", "xi", "plen", "path"):
            setattr(self, k, getattr(self, k)[:n].copy())
        return self

    def pointers(self):
        ip = C.POINTER(C.c_int32)
        lp = C.POINTER(C.c_int64)
        return (_dp(self.x), _dp(self.ow), _dp(self.x1), _dp(self.w1), _dp(self.wpx), _dp(self.xi),
                self.plen.ctypes.data_as(ip), self.path.ctypes.data_as(lp))


def records(h: ArgsHolder, rng: Rng, want_phase: bool, capacity: int) -> Records:
    r = Records(capacity)
    n = C.c_int64(0)
    rc = lib().oracle_records(C.addressof(h.args), C.byref(rng.spec), int(want_phase), capacity,
                              *r.pointers(), C.byref(n))
    if rc == -2:
        raise RuntimeError(f"oracle_records: {n.value} events exceed capacity {capacity}")
    _check(rc, "oracle_records")
    return r.truncate(n.value)


def field_from_records(h: ArgsHolder, r: Records) -> np.ndarray:
    a = h.args
    u = np.zeros(2 * a.nv * a.nl)
    p = r.pointers()
    lib().oracle_field_from_records(C.addressof(a), r.n, p[0], p[1], p[2], p[3], p[4], p[5], p[6], _dp(u))
    return u.view(np.complex128).reshape(a.nv, a.nl, order="F")


def cov_from_records(h: ArgsHolder, r: Records, threads: int = 1):
    a = h.args
    n = a.nv * a.nv * a.nl * a.nl
    Ms = np.zeros(2 * n)
    Mm = np.zeros(2 * n)
    p = r.pointers()
    lib().oracle_cov_from_records(C.addressof(a), r.n, p[0], p[1], p[2], p[3], p[4], p[6],
                                  _dp(Ms), _dp(Mm), threads)
    shp = (a.nv, a.nv, a.nl, a.nl)
    return (Ms.view(np.complex128).reshape(shp, order="F"),
            Mm.view(np.complex128).reshape(shp, order="F"))


def philox_block(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().oracle_philox4x32_10(c, k, o)
    return list(o)


def philox_stream(seed, path, tag, n):
    out = np.zeros(n)
    lib().oracle_philox_stream(seed, path, tag, n, _dp(out))
    return out


def field_fourier_quad(fa: FqArgs, rng: Rng, nv0: int) -> np.ndarray:
    """MCfieldFourierQuad on the oracle: nv0 x nv0 x nl complex."""
    u = np.zeros(2 * nv0 * nv0 * fa.nl)
    _check(lib().oracle_field_fourier_quad(C.byref(fa), C.byref(rng.spec), _dp(u)), "oracle_field_fourier_quad")
    return u.view(np.complex128).reshape(nv0, nv0, fa.nl, order="F")


def field_fourier_quad_onwave(fa: FqArgs, Wl, rng: Rng, nv0: int, as_written: bool = False) -> np.ndarray:
    """MCfieldFourierQuadOnWave on the oracle: nv0 x nv0 complex.  as_written:
    the reference's lines 282-292 exactly (light weight of a plane's j3-th
    vertex taken at the j3-th vertex of the whole sorted list)."""
    w = np.ascontiguousarray(np.asarray(Wl, dtype=np.complex128).reshape(-1))
    if w.size != fa.nl:
        raise ValueError("Wl needs one weight per light")
    u = np.zeros(2 * nv0 * nv0)
    _check(lib().oracle_field_fourier_quad_onwave(C.byref(fa), _dp(w.view(np.float64)), int(bool(as_written)),
                                                  C.byref(rng.spec), _dp(u)),
           "oracle_field_fourier_quad_onwave")
    return u.view(np.complex128).reshape(nv0, nv0, order="F")


def cov_hetero(h, rng: Rng, threads: int = 1):
    """MCCovHetro on the oracle -> Ms, Mm, mean1."""
    n = h.nv * h.nv * h.nl * h.nl
    Ms, Mm, m1 = np.zeros(2 * n), np.zeros(2 * n), np.zeros(2 * h.nv * h.nl)
    _check(lib().oracle_cov_hetero(C.byref(h.args), C.byref(rng.spec), _dp(Ms), _dp(Mm), _dp(m1), threads),
           "oracle_cov_hetero")
    shp = (h.nv, h.nv, h.nl, h.nl)
    return (Ms.view(np.complex128).reshape(shp, order="F"), Mm.view(np.complex128).reshape(shp, order="F"),
            m1.view(np.complex128).reshape(h.nv, h.nl, order="F"))


def field_hetero(h, rng: Rng) -> np.ndarray:
    """MCsampleHetro on the oracle -> u."""
    u = np.zeros(2 * h.nv * h.nl)
    _check(lib().oracle_field_hetero(C.byref(h.args), C.byref(rng.spec), _dp(u)), "oracle_field_hetero")
    return u.view(np.complex128).reshape(h.nv, h.nl, order="F")


def refocus(u, v, l, box_min, box_max, box_stp, lambda_, as_written=True):
    """refocus.m on the oracle: rU shaped like the reference's ndgrid."""
    v = np.asarray(v, dtype=np.float64)
    dim = v.shape[0]
    f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))  # noqa: E731
    bmin, bmax, bstp, lv = f(box_min), f(box_max), f(box_stp), f(l)
    dims = np.zeros(3, dtype=np.int64)
    n = lib().oracle_refocus_grid(dim, _dp(bmin), _dp(bmax), _dp(bstp), dims.ctypes.data_as(C.POINTER(C.c_int64)))
    uc = np.ascontiguousarray(np.asarray(u, dtype=np.complex128).reshape(-1))
    vc = np.ascontiguousarray(v.T)
    out = np.zeros(2 * n)
    _check(lib().oracle_refocus(_dp(uc.view(np.float64)), _dp(vc), v.shape[1], dim, _dp(lv), _dp(bmin), _dp(bmax),
                                _dp(bstp), float(lambda_), int(bool(as_written)), _dp(out)), "oracle_refocus")
    return out.view(np.complex128).reshape(tuple(dims[:dim]), order="F")


def sample_cov(C_mat, normals):
    """samplingFromCovMatrix.m:47-64 on the oracle: one complex N-vector per row of normals (2N each)."""
    Cm = np.ascontiguousarray(np.asarray(C_mat, dtype=np.complex128).reshape(-1, order="F"))
    N = int(round(np.sqrt(Cm.size)))
    g = np.ascontiguousarray(np.asarray(normals, dtype=np.float64).reshape(-1, 2 * N))
    Z = np.zeros(2 * N * g.shape[0])
    rc = lib().oracle_sample_cov(_dp(Cm.view(np.float64)), N, g.shape[0], _dp(g), _dp(Z))
    if rc == -1:
        raise ValueError("Sigma is not positive definite")
    _check(rc, "oracle_sample_cov")
    return Z.view(np.complex128).reshape(N, g.shape[0], order="F")
