"""Data formats around the Monte Carlo path.

* Tabulated scattering amplitudes stored as MATLAB .mat files (the
  reference ships examples/buildFarFieldCovMatrix/scatteringAmplitude.mat
  with variables `theta` and `farField`): `load_amplitude_table` reads one
  and builds the scatter structure with tabulatedAmplitudeScatter
  (tabulatedAmplitudeScatter.m:1-99).

* Path records on disk: the per-event records of the walk
  (scmc_export_records: x, ow, x1, w1, weight/px, xi, pL, path) together with
  the MCfield arguments they belong to, in one .npz file.  Records written on
  one machine replay on another (`replay_field`, on the GPU through
  scmc_field_from_records) and can be fed to any FP64 accumulation for
  parity checks.  Format "scmc-path-records", version 1:
      arrays  x, ow, x1, w1   (n, 3) float64   event, incoming direction,
                                                first scatterer, first direction
              wpx, xi         (n,)   float64   weight/px, random-phase uniform
              plen            (n,)   int32     1-based event index in its path
              path            (n,)   int64     path index (relative to path_offset)
              l, v            (dim, nl), (dim, nv) float64
              ampfunc_evalAmp, ampfunc_sampleIcdf, ampfunc0_* (tabulated only)
              lmean0          (dim,) float64 (when given)
      meta    JSON string: format, version, n_events, dim, sigt, albedo,
              box_min, box_max, is_ff_l, is_ff_v, max_itr, lambda, do_cbs,
              smp_flg, ampfunc_type, ampfunc_g (and ampfunc0_* when given),
              has_ampfunc0, has_lmean0, seed, path_offset, norm_itr, want_phase
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import _abi, _lib
from . import interface as I
from . import mc as MC

FORMAT = "scmc-path-records"
VERSION = 1


def load_amplitude_table(path, theta_key="theta", f_key="farField", *albedo):
    """tabulatedAmplitudeScatter(theta, f[, albedo]) from a .mat file."""
    import scipy.io as sio
    m = sio.loadmat(path)
    if theta_key not in m or f_key not in m:
        raise KeyError(f"{path} has no '{theta_key}' / '{f_key}' variables")
    return I.tabulatedAmplitudeScatter(np.asarray(m[theta_key]), np.asarray(m[f_key]), *albedo)


def _pf_meta(prefix, meta, arrays, cstruct: _abi.PhaseFunction):
    meta[prefix + "_type"] = int(cstruct.sct_type)
    meta[prefix + "_g"] = float(cstruct.g)
    if cstruct.sct_type == 2:
        n = int(cstruct.table_n)
        amp = np.ctypeslib.as_array(cstruct.eval_amp, shape=(2 * n,)).copy()
        arrays[prefix + "_evalAmp"] = amp.view(np.complex128)
        arrays[prefix + "_sampleIcdf"] = np.ctypeslib.as_array(cstruct.sample_icdf, shape=(n,)).copy()


def save_records(path, records: MC.Records, h: _abi.ArgsHolder, want_phase=True):
    """Write records and the arguments of the solve that produced them."""
    a = h.args
    dim = int(a.dim)
    meta = {"format": FORMAT, "version": VERSION, "n_events": int(records.n), "dim": dim, "sigt": a.sigt,
            "albedo": a.albedo, "box_min": list(a.box_min)[:dim], "box_max": list(a.box_max)[:dim],
            "is_ff_l": bool(a.is_ff_l), "is_ff_v": bool(a.is_ff_v), "max_itr": int(a.max_itr),
            "lambda": a.lambda_, "do_cbs": bool(a.do_cbs), "smp_flg": int(a.smp_flg),
            "has_ampfunc0": bool(a.has_ampfunc0), "has_lmean0": bool(a.has_lmean0), "seed": int(a.seed),
            "path_offset": int(a.path_offset), "norm_itr": int(a.norm_itr), "want_phase": bool(want_phase)}
    n = records.n
    arrays = {"x": records.x.reshape(n, 3), "ow": records.ow.reshape(n, 3), "x1": records.x1.reshape(n, 3),
              "w1": records.w1.reshape(n, 3), "wpx": records.wpx, "xi": records.xi, "plen": records.plen,
              "path": records.path,
              "l": np.ctypeslib.as_array(a.l, shape=(int(a.nl) * dim,)).reshape(dim, -1, order="F").copy(),
              "v": np.ctypeslib.as_array(a.v, shape=(int(a.nv) * dim,)).reshape(dim, -1, order="F").copy()}
    _pf_meta("ampfunc", meta, arrays, a.ampfunc)
    if a.has_ampfunc0:
        _pf_meta("ampfunc0", meta, arrays, a.ampfunc0)
    if a.has_lmean0:
        arrays["lmean0"] = np.array(list(a.lmean0)[:dim])
    np.savez_compressed(path, meta=json.dumps(meta), **arrays)


def load_records(path):
    """(Records, meta dict, arrays dict) from a record file."""
    z = np.load(path, allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    if meta.get("format") != FORMAT or meta.get("version") != VERSION:
        raise ValueError(f"{path}: not a {FORMAT} v{VERSION} file")
    arrays = {k: z[k] for k in z.files if k != "meta"}
    n = int(meta["n_events"])
    r = MC.Records(n)
    for k in ("x", "ow", "x1", "w1"):
        setattr(r, k, np.ascontiguousarray(arrays[k], dtype=np.float64).reshape(-1))
    r.wpx = np.ascontiguousarray(arrays["wpx"], dtype=np.float64)
    r.xi = np.ascontiguousarray(arrays["xi"], dtype=np.float64)
    r.plen = np.ascontiguousarray(arrays["plen"], dtype=np.int32)
    r.path = np.ascontiguousarray(arrays["path"], dtype=np.int64)
    r.n = n
    return r, meta, arrays


def args_from_records(meta, arrays, precision="fp64", device=0):
    """The MCfield argument holder the records were written with."""
    def amp(prefix):
        if meta[prefix + "_type"] == 2:
            return {"evalAmp": arrays[prefix + "_evalAmp"], "sampleIcdf": arrays[prefix + "_sampleIcdf"]}
        return meta[prefix + "_g"] if meta[prefix + "_type"] == 3 else 0
    pos = [meta["sigt"], meta["albedo"], np.array(meta["box_min"]), np.array(meta["box_max"]), arrays["l"],
           arrays["v"], meta["is_ff_l"], meta["is_ff_v"], meta["max_itr"], meta["lambda"], meta["do_cbs"],
           meta["smp_flg"], meta["ampfunc_type"], amp("ampfunc")]
    if meta["has_ampfunc0"]:
        pos.append(amp("ampfunc0"))
    if meta["has_lmean0"]:
        if not meta["has_ampfunc0"]:
            pos.append(MC._MISSING)
        pos.append(arrays["lmean0"])
    return MC.mc_args(*pos, seed=meta["seed"], precision=precision, device=device, path_offset=meta["path_offset"],
                      norm_itr=meta.get("norm_itr", 0))


def replay_field(path, precision="fp64", device=0):
    """The field of a record file, accumulated on the GPU (MCfield.m:207-254)."""
    r, meta, arrays = load_records(path)
    h = args_from_records(meta, arrays, precision, device)
    a = h.args
    u = np.zeros(2 * a.nv * a.nl)
    dp = C.POINTER(C.c_double)
    _lib.check(_lib.lib().scmc_field_from_records(h.ref, r.n, *r.pointers()[:6], r.plen.ctypes.data_as(
        C.POINTER(C.c_int32)), r.path.ctypes.data_as(C.POINTER(C.c_int64)), u.ctypes.data_as(dp)))
    return u.view(np.complex128).reshape(a.nv, a.nl, order="F")
