"""MCCovHetro / MCsampleHetro (voxel medium) with the reference's signatures.

    [Ms, Mm, mean1] = MCCovHetro(sigt, albedo, box_min, box_max, box_bin, l, v,
                                 is_ff_l, is_ff_v, maxItr, lambda_, doCBS,
                                 smpFlg, sct_type, ampfunc[, ampfunc0[, lrad]])
                                                      (code/MCCovHetro.m:1)
    u = MCsampleHetro(sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l,
                      is_ff_v, maxItr, lambda_, doCBS, smpFlg, sct_type,
                      ampfunc[, ampfunc0[, lmean0]])    (code/MCsampleHetro.m:1)

sigt (and optionally albedo) are voxel grids, x fastest (findBin.m order).
Unlike MCcov the result is normalised by maxItr only: the first-scatter
density px carries the medium's volume (MCCovHetro.m:64, 262-276).

The plane launch of smpFlg = 2 (expSmpXHetro.m:8) uses null(meanl') as its
lateral axes; they are computed here the way MATLAB's null() does, from the
SVD of the 1 x dim row (the right singular vectors past the rank).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _lib
from .mc import DEFAULT_PRECISION, _MISSING, _as_matrix, _scatter, draw_seed


def null_basis(meanl: np.ndarray) -> np.ndarray:
    """Orthonormal basis of the null space of the row vector meanl'."""
    a = np.asarray(meanl, dtype=float).reshape(1, -1)
    _, s, vh = np.linalg.svd(a)
    tol = max(a.shape) * (s[0] if s.size else 0.0) * np.finfo(float).eps
    r = int(np.sum(s > tol))
    return vh[r:].conj().T


class HeteroHolder:
    def __init__(self, args, keep, nv, nl):
        self.args = args
        self._keep = keep
        self.nv, self.nl = nv, nl

    @property
    def ref(self):
        return C.byref(self.args)


def hetero_args(cov: bool, sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l, is_ff_v, maxItr, lambda_,
                doCBS, smpFlg, sct_type, ampfunc, ampfunc0=_MISSING, extra=_MISSING, *, seed=None,
                precision=DEFAULT_PRECISION, device=0, path_offset=0, norm_itr=0, max_events_per_path=0,
                basis=None, trilinear=False) -> HeteroHolder:
    """The C argument struct.  trilinear=True (an extension, off by default)
    interpolates sigt trilinearly between voxel centres instead of the
    reference's nearest voxel (findBin.m)."""
    bmin = np.asarray(box_min, dtype=float).reshape(-1)
    bmax = np.asarray(box_max, dtype=float).reshape(-1)
    bbin = np.asarray(box_bin, dtype=float).reshape(-1)
    dim = bmin.size
    L = _as_matrix(np.asarray(l, dtype=float))
    V = _as_matrix(np.asarray(v, dtype=float))
    if L.shape[0] == 1:
        L = np.vstack([np.sin(L), np.cos(L)])  # MCCovHetro.m:20-25
    if V.shape[0] == 1:
        V = np.vstack([np.sin(V), np.cos(V)])
    sg = np.asarray(sigt, dtype=float)
    nb = np.rint((bmax - bmin) / bbin).astype(int)
    if sg.size != int(np.prod(nb)):
        raise ValueError(f"sigt has {sg.size} voxels, the box has {int(np.prod(nb))}")
    sg_flat = np.ascontiguousarray(sg.reshape(-1, order="F"))
    al = np.asarray(albedo, dtype=float)
    al_flat = None if al.size == 1 else np.ascontiguousarray(al.reshape(-1, order="F"))
    sc = _scatter(sct_type, ampfunc)
    has0 = ampfunc0 is not _MISSING and not (isinstance(ampfunc0, np.ndarray) and ampfunc0.size == 0)
    sc0 = _scatter(sct_type, ampfunc0) if has0 else None
    lrad = None
    lmean0 = None
    if extra is not _MISSING and extra is not None:
        if cov:
            lrad = float(np.asarray(extra).reshape(-1)[0])
        else:
            lmean0 = np.asarray(extra, dtype=float).reshape(-1)
    prec = _abi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    h = _abi.build_mc_args(dim=dim, sigt=1.0, albedo=float(al.reshape(-1)[0]), box_min=bmin, box_max=bmax, l=L,
                           v=V, is_ff_l=bool(np.asarray(is_ff_l).reshape(-1)[0]),
                           is_ff_v=bool(np.asarray(is_ff_v).reshape(-1)[0]), max_itr=int(maxItr),
                           lam=float(lambda_), do_cbs=bool(np.asarray(doCBS).reshape(-1)[0]), smp_flg=int(smpFlg),
                           scatter=sc, scatter0=sc0, lmean0=lmean0, seed=draw_seed() if seed is None else seed,
                           path_offset=path_offset, norm_itr=norm_itr, precision=prec, device=device,
                           max_events_per_path=max_events_per_path)
    a = _abi.HeteroArgs()
    a.mc = h.args
    a.sigt_grid = sg_flat.ctypes.data_as(C.POINTER(C.c_double))
    a.albedo_grid = al_flat.ctypes.data_as(C.POINTER(C.c_double)) if al_flat is not None else None
    for k in range(dim):
        a.box_bin[k] = bbin[k]
    if lrad is not None:
        a.has_lrad = 1
        a.lrad = lrad
    a.trilinear = int(bool(trilinear))
    # meanl as the reference forms it (MCCovHetro.m:38-39, MCsampleHetro.m:35-41)
    um = lmean0 if lmean0 is not None else L.mean(axis=1)
    meanl = um / np.linalg.norm(um)
    B = null_basis(meanl) if basis is None else np.asarray(basis, dtype=float).reshape(dim, dim - 1)
    flat = B.reshape(-1, order="F")
    for k in range(flat.size):
        a.null_basis[k] = flat[k]
    return HeteroHolder(a, [h, sg_flat, al_flat], V.shape[1], L.shape[1])


def cov_hetero_from_args(h: HeteroHolder):
    n = h.nv * h.nv * h.nl * h.nl
    Ms, Mm, m1 = np.zeros(2 * n), np.zeros(2 * n), np.zeros(2 * h.nv * h.nl)
    dp = C.POINTER(C.c_double)
    _lib.check(_lib.lib().scmc_cov_hetero(h.ref, Ms.ctypes.data_as(dp), Mm.ctypes.data_as(dp),
                                          m1.ctypes.data_as(dp)))
    shp = (h.nv, h.nv, h.nl, h.nl)
    return (Ms.view(np.complex128).reshape(shp, order="F"), Mm.view(np.complex128).reshape(shp, order="F"),
            m1.view(np.complex128).reshape(h.nv, h.nl, order="F"))


def field_hetero_from_args(h: HeteroHolder):
    u = np.zeros(2 * h.nv * h.nl)
    _lib.check(_lib.lib().scmc_field_hetero(h.ref, u.ctypes.data_as(C.POINTER(C.c_double))))
    return u.view(np.complex128).reshape(h.nv, h.nl, order="F")


def MCCovHetro(sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l, is_ff_v, maxItr, lambda_, doCBS, smpFlg,
               sct_type, ampfunc, ampfunc0=_MISSING, lrad=_MISSING, **gpu):
    """Voxel-medium covariance Ms, Mm and the single-scattering mean (MCCovHetro.m:1-276)."""
    return cov_hetero_from_args(hetero_args(True, sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l, is_ff_v,
                                            maxItr, lambda_, doCBS, smpFlg, sct_type, ampfunc, ampfunc0, lrad, **gpu))


def MCsampleHetro(sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l, is_ff_v, maxItr, lambda_, doCBS, smpFlg,
                  sct_type, ampfunc, ampfunc0=_MISSING, lmean0=_MISSING, **gpu):
    """Voxel-medium speckle field (MCsampleHetro.m:1-227)."""
    return field_hetero_from_args(hetero_args(False, sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l,
                                              is_ff_v, maxItr, lambda_, doCBS, smpFlg, sct_type, ampfunc, ampfunc0,
                                              lmean0, **gpu))
