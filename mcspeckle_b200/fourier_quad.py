"""MCfieldFourierQuad with the reference's positional signature, on the GPU.

    u = MCfieldFourierQuad(sigt, albedo, box_min, box_max, l, v_max, v_stp,
                           maxItr, lambda_, doCBS, smpFlg, lmean0=[], vsign=-1)
                                              (code/MCfieldFourierQuad.m:1)

u is Nv0 x Nv0 x Nl complex on the angular grid -v_max:v_stp:v_max
(uniform in sin(theta)).  The first-scatter direction defaults to +z
(MCfieldFourierQuad.m:59-64), the walk is isotropic, and the normalisation
counts vertices, as in the reference (MCfieldFourierQuad.m:214, 302-303).
Keyword-only extensions (fq_args): point sources and HG scattering.

The reference's FFT needs integer padding, which holds only for an odd grid
length; for even lengths it stops.  The GPU evaluates the same centred-DFT
formula with half-integer offsets there (an extension, unpinned).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi, _lib
from .mc import DEFAULT_PRECISION, MatlabStyleError, _as_matrix, draw_seed


def colon_count(a: float, s: float, b: float) -> int:
    """Element count of MATLAB's a:s:b."""
    if s == 0 or (s > 0 and a > b) or (s < 0 and a < b):
        return 0
    q = (b - a) / s
    return int(math.floor(q + 1e-10 * max(1.0, abs(q)))) + 1


def grid_length(v_max: float, v_stp: float) -> int:
    return colon_count(-v_max, v_stp, v_max)


class FqHolder:
    def __init__(self, args, keep, nv0):
        self.args = args
        self._keep = keep
        self.nv0 = nv0

    @property
    def ref(self):
        return C.byref(self.args)


def fq_args(sigt, albedo, box_min, box_max, l, v_max, v_stp, maxItr, lambda_, doCBS, smpFlg, lmean0=None,
            vsign=-1, *, seed=None, precision=DEFAULT_PRECISION, device=0, path_offset=0, light_point=False,
            hg_g=None) -> FqHolder:
    """The C argument struct.  Two extensions beyond the reference, off by
    default: light_point=True takes the columns of l as point-source
    positions (the near-field light factor of evalphaseatt.m:10-16 instead of
    the plane wave of MCfieldFourierQuad.m:272); hg_g=g samples the walk's
    scattering directions from HG(g) (the smpampfunc_general call the
    reference leaves commented out at line 208)."""
    bmin = np.asarray(box_min, dtype=float).reshape(-1)
    bmax = np.asarray(box_max, dtype=float).reshape(-1)
    if bmin.size != 3 or bmax.size != 3:
        raise MatlabStyleError("Invalid box size")  # MCfieldFourierQuad.m:41-44 (3-D only here)
    L = _as_matrix(np.asarray(l, dtype=float))
    if L.shape[0] != 3:
        raise MatlabStyleError("Invalid light source input")
    a = _abi.FqArgs()
    a.sigt = float(sigt)
    a.albedo = float(albedo)
    for k in range(3):
        a.box_min[k] = bmin[k]
        a.box_max[k] = bmax[k]
    lc = np.ascontiguousarray(L.T)  # [nl][3]
    a.l = lc.ctypes.data_as(C.POINTER(C.c_double))
    a.nl = lc.shape[0]
    a.v_max = float(v_max)
    a.v_stp = float(v_stp)
    a.max_itr = int(maxItr)
    a.lambda_ = float(lambda_)
    a.do_cbs = int(bool(doCBS))
    a.smp_flg = int(smpFlg)
    lm = None if lmean0 is None else np.asarray(lmean0, dtype=float).reshape(-1)
    if lm is not None and lm.size == 3:
        a.has_lmean0 = 1
        for k in range(3):
            a.lmean0[k] = lm[k]
    a.vsign = float(vsign)
    a.seed = (draw_seed() if seed is None else int(seed)) & (2**64 - 1)
    a.path_offset = int(path_offset)
    a.precision = _abi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    a.device = int(device)
    a.light_point = int(bool(light_point))
    if hg_g is not None:
        if not abs(float(hg_g)) <= 1.0:
            raise MatlabStyleError("Invalid g input")
        a.sct_type = 3
        a.g = float(hg_g)
    return FqHolder(a, [lc], grid_length(a.v_max, a.v_stp))


def field_fourier_quad_from_args(h: FqHolder) -> np.ndarray:
    a = h.args
    u = np.zeros(2 * h.nv0 * h.nv0 * a.nl)
    _lib.check(_lib.lib().scmc_field_fourier_quad(h.ref, u.ctypes.data_as(C.POINTER(C.c_double))))
    return u.view(np.complex128).reshape(h.nv0, h.nv0, a.nl, order="F")


def MCfieldFourierQuad(sigt, albedo, box_min, box_max, l, v_max, v_stp, maxItr, lambda_, doCBS, smpFlg,
                       lmean0=None, vsign=-1, **gpu):
    """Speckle field on an angular grid by z-plane quadrature (MCfieldFourierQuad.m:1-303)."""
    return field_fourier_quad_from_args(fq_args(sigt, albedo, box_min, box_max, l, v_max, v_stp, maxItr, lambda_,
                                                doCBS, smpFlg, lmean0, vsign, **gpu))


def field_fourier_quad_onwave_from_args(h: FqHolder, Wl) -> np.ndarray:
    a = h.args
    w = np.ascontiguousarray(np.asarray(Wl, dtype=np.complex128).reshape(-1))
    if w.size != a.nl:
        raise MatlabStyleError("Wl needs one weight per light")
    u = np.zeros(2 * h.nv0 * h.nv0)
    dp = C.POINTER(C.c_double)
    _lib.check(_lib.lib().scmc_field_fourier_quad_onwave(h.ref, w.view(np.float64).ctypes.data_as(dp),
                                                         u.ctypes.data_as(dp)))
    return u.view(np.complex128).reshape(h.nv0, h.nv0, order="F")


def MCfieldFourierQuadOnWave(sigt, albedo, box_min, box_max, l, v_max, v_stp, maxItr, lambda_, doCBS, smpFlg,
                             lmean0, Wl, vsign=-1, **gpu):
    """The lights combined with complex weights Wl (MCfieldFourierQuadOnWave.m:1-337): Nv0 x Nv0."""
    return field_fourier_quad_onwave_from_args(fq_args(sigt, albedo, box_min, box_max, l, v_max, v_stp, maxItr,
                                                       lambda_, doCBS, smpFlg, lmean0, vsign, **gpu), Wl)
