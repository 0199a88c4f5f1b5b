"""Post-processing of rendered fields and covariances (refocus.m and the
samplingFromCovMatrix example), on the GPU through the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _lib

_dp = C.POINTER(C.c_double)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


def refocus(u, v, l, box_min, box_max, box_stp, lambda_, *, as_written=True, precision="fp64", device=0):
    """rU = refocus(u, v, l, box_min, box_max, box_stp, lambda) (refocus.m:1-34):
    the views' field u back-propagated onto an ndgrid of points with light
    direction l; shaped like the grid.  as_written: the first grid point stays
    0 as in the reference (its chunk indices start at j+1)."""
    v = np.asarray(v, dtype=np.float64)
    if v.ndim == 1:
        v = v.reshape(-1, 1)
    dim = v.shape[0]
    bmin, bmax, bstp = _f64(box_min), _f64(box_max), _f64(box_stp)
    if bmin.size != dim or bmax.size != dim or bstp.size != dim:
        raise ValueError("box and views must have the same dimension")
    uc = np.ascontiguousarray(np.asarray(u, dtype=np.complex128).reshape(-1, order="F"))
    if uc.size != v.shape[1]:
        raise ValueError("u needs one value per view")
    vc = np.ascontiguousarray(v.T)
    dims = np.zeros(3, dtype=np.int64)
    n = C.c_int64()
    L = _lib.lib()
    _lib.check(L.scmc_refocus_grid(dim, bmin.ctypes.data_as(_dp), bmax.ctypes.data_as(_dp), bstp.ctypes.data_as(_dp),
                                   dims.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(n)))
    out = np.zeros(2 * n.value)
    prec = _abi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    lv = _f64(l)
    _lib.check(L.scmc_refocus(uc.view(np.float64).ctypes.data_as(_dp), vc.ctypes.data_as(_dp), uc.size, dim,
                              lv.ctypes.data_as(_dp), bmin.ctypes.data_as(_dp), bmax.ctypes.data_as(_dp),
                              bstp.ctypes.data_as(_dp), float(lambda_), int(bool(as_written)), prec, int(device),
                              out.ctypes.data_as(_dp)))
    return out.view(np.complex128).reshape(tuple(dims[:dim]), order="F")


def united_cov(Cmat) -> np.ndarray:
    """scmc's C(v1, v2, l1, l2) joined into the N x N matrix of the
    samplingFromCovMatrix example ([C(:,:,1,1) C(:,:,1,2); ...]), N = nv*nl."""
    Cm = np.asarray(Cmat)
    if Cm.ndim == 2:
        return Cm
    nv, nl = Cm.shape[0], Cm.shape[2]
    return Cm.transpose(0, 2, 1, 3).reshape(nv * nl, nv * nl, order="F")


def sample_from_cov(Cmat, n_samples=1, seed=0, *, device=0):
    """Field samples with covariance C (samplingFromCovMatrix.m:47-64):
    z = s(1:N) + i s(N+1:2N), s = g chol(0.5 [Re C, -Im C; Im C, Re C]),
    g the Philox normal stream (seed, path t) of sample t.  A 4-D scmc C
    gives samples shaped nv x nl x n_samples, an N x N one N x n_samples."""
    Cm = np.asarray(Cmat)
    shape4 = Cm.ndim == 4
    U = np.ascontiguousarray(united_cov(Cm).astype(np.complex128).reshape(-1, order="F"))
    N = int(round(np.sqrt(U.size)))
    Z = np.zeros(2 * N * int(n_samples))
    _lib.check(_lib.lib().scmc_sample_cov(U.view(np.float64).ctypes.data_as(_dp), N, int(n_samples),
                                          int(seed) & (2**64 - 1), int(device), Z.ctypes.data_as(_dp)))
    z = Z.view(np.complex128).reshape(N, int(n_samples), order="F")
    if shape4:
        return z.reshape(Cm.shape[0], Cm.shape[2], int(n_samples), order="F")
    return z


def memory_effect_offsets(C1, C2=None, *, views_grid, lights_grid, device=0):
    """The memory-effect view of scmc's covariance C(v1, v2, l1, l2) (+ C2,
    e.g. Ms + Mm): the mean over all entries with the same view offset
    v1 - v2 and light offset l1 - l2 on the views' (nvx, nvy) and the lights'
    (nlx, nly) grids (flat index x fastest), the diagonal means that
    examples/memoryEffectMeasurements/memoryEffectMeasurements.m:72-86 takes.
    Returns complex64 R[dvx, dvy, dlx, dly], offset d at index d + n - 1."""
    nvx, nvy = (int(x) for x in views_grid)
    nlx, nly = (int(x) for x in lights_grid)
    c1 = np.ascontiguousarray(np.asarray(C1, dtype=np.complex128).reshape(-1, order="F"))
    if c1.size != (nvx * nvy) ** 2 * (nlx * nly) ** 2:
        raise ValueError("C does not match the grids")
    c2 = None
    if C2 is not None:
        c2 = np.ascontiguousarray(np.asarray(C2, dtype=np.complex128).reshape(-1, order="F"))
        if c2.size != c1.size:
            raise ValueError("C1 and C2 differ in size")
    shape = (2 * nvx - 1, 2 * nvy - 1, 2 * nlx - 1, 2 * nly - 1)
    out = np.zeros(2 * int(np.prod(shape)), dtype=np.float32)
    _lib.check(_lib.lib().scmc_cov_offsets(c1.view(np.float64).ctypes.data_as(_dp),
                                           None if c2 is None else c2.view(np.float64).ctypes.data_as(_dp),
                                           nvx, nvy, nlx, nly, out.ctypes.data_as(C.POINTER(C.c_float)),
                                           int(device)))
    return out.view(np.complex64).reshape(shape, order="F")


def memory_effect_offsets_numpy(Cmat, views_grid, lights_grid):
    """The same reduction in NumPy (FP64), for checks."""
    nvx, nvy = views_grid
    nlx, nly = lights_grid
    Cm = np.asarray(Cmat).reshape(nvx, nvy, nvx, nvy, nlx, nly, nlx, nly, order="F")
    R = np.zeros((2 * nvx - 1, 2 * nvy - 1, 2 * nlx - 1, 2 * nly - 1), dtype=np.complex128)
    cnt = np.zeros(R.shape)
    ix = np.arange(nvx)
    iy = np.arange(nvy)
    jx = np.arange(nlx)
    jy = np.arange(nly)
    dvx = (ix[:, None] - ix[None, :]) + nvx - 1      # (v1x, v2x)
    dvy = (iy[:, None] - iy[None, :]) + nvy - 1
    dlx = (jx[:, None] - jx[None, :]) + nlx - 1
    dly = (jy[:, None] - jy[None, :]) + nly - 1
    a = dvx[:, None, :, None, None, None, None, None]
    b = dvy[None, :, None, :, None, None, None, None]
    c = dlx[None, None, None, None, :, None, :, None]
    d = dly[None, None, None, None, None, :, None, :]
    A, B, Cc, D = np.broadcast_arrays(a, b, c, d)
    np.add.at(R, (A.ravel(), B.ravel(), Cc.ravel(), D.ravel()), Cm.ravel())
    np.add.at(cnt, (A.ravel(), B.ravel(), Cc.ravel(), D.ravel()), 1.0)
    return R / cnt
