"""scmc - the Speckle Covariance Monte Carlo entry point (scmc.m:1-429).

    mulRes = scmc(targetArea, views, lights, scatter, iterations, 'opt', val, ...)
    mulRes = scmc(Config)

Validation, option parsing, Config building and the MCcov / MCfield dispatch
follow scmc.m line by line; the error strings are the reference's.  The
kernels run on the GPU through libscmc_gpu.so.

`parforIters` replicas (scmc.m:343-368, 398-423) are independent Philox path
ranges of one launch: the mean of P covariance replicas and the
sqrt-weighted sum of P field replicas equal one run of P*iterations paths,
which is what runs.

Behaviour that differs from the published file, on purpose:
* tabulated scatter: scmc.m:259-269 reads `Config.scatter.ampfunc0`, a field
  tabulatedAmplitudeScatter never sets, so the published file stops with
  "Reference to non-existent field".  A missing ampfunc0 is treated like
  `inf` (no first-event table), which is how the published example PDFs ran.
  scmc.m:259 also reads the local `scatter` rather than `Config.scatter`;
  here the Config's struct is used, so scmc(Config) works for tables too.
"""
from __future__ import annotations

import math

import numpy as np

from . import mc as _mc


class ScmcInputError(ValueError):
    """scmc input validation error (reference message text)."""


def _is_scalar(x) -> bool:
    return not isinstance(x, str) and np.asarray(x).size == 1


def _is_logical_scalar(x) -> bool:
    return isinstance(x, (bool, np.bool_)) or (isinstance(x, np.ndarray) and x.dtype == bool and x.size == 1)


class _GpuKernels:
    """MCcov / MCfield on the GPU with the given execution controls."""

    def __init__(self, **gpu):
        self.gpu = gpu

    def MCcov(self, *args, seed, n_total):
        return _mc.cov_from_args(_mc.mc_args(*args, seed=seed, norm_itr=n_total, **self.gpu))

    def MCfield(self, *args, seed, n_total):
        return _mc.field_from_args(_mc.mc_args(*args, seed=seed, norm_itr=n_total, **self.gpu))


def build_config(targetArea, views, lights, scatter, iterations, *varargin) -> dict:
    """scmc.m:59-235: validate the inputs and build the Config struct."""
    if len(varargin) % 2 != 0:
        raise ScmcInputError("Parameters must be in struct of option and value")
    if targetArea.get("type") != "targetArea":
        raise ScmcInputError("Invalid target area input")
    if views.get("type") != "source":
        raise ScmcInputError("Invalid views input")
    if lights.get("type") != "source":
        raise ScmcInputError("Invalid lights input")
    if scatter.get("type") != "scatter":
        raise ScmcInputError("Invalid scatter input")
    if not _is_scalar(iterations) or float(np.asarray(iterations).reshape(-1)[0]) < 1:
        raise ScmcInputError("Invalid photons number")
    if scatter.get("function") == "measuredFarField" and targetArea["D"] == 3:
        raise ScmcInputError("Measured scattering of far field is used only in 2D")
    views = dict(views)
    lights = dict(lights)
    sfx = "3D" if targetArea["D"] == 3 else "2D"
    for src in (views, lights):
        for key in ("directions", "positions"):
            if key + sfx in src:
                src[key] = src[key + sfx]
    cfg = {"targetArea": targetArea, "views": views, "lights": lights, "scatter": scatter,
           "render": {"iterations": float(np.asarray(iterations).reshape(-1)[0]), "singleScattering": False,
                      "cov": True, "multipleScattering": True, "field": False},
           "parforIters": 1, "rng": -1, "CBS": True, "uniformFirstScatter": False}
    for k in range(0, len(varargin), 2):
        opt, val = str(varargin[k]), varargin[k + 1]
        if opt == "parforIters":
            if not _is_scalar(val) or float(np.asarray(val).reshape(-1)[0]) < 0:
                raise ScmcInputError("invalid parfor iterations number")
            if cfg["rng"] != -1:
                raise ScmcInputError("rng can not be used while using parfor")
            cfg["parforIters"] = float(np.asarray(val).reshape(-1)[0])
        elif opt == "rng":
            if not _is_scalar(val) or float(np.asarray(val).reshape(-1)[0]) < 0:
                raise ScmcInputError("invalid rng number")
            if cfg["parforIters"] != 1:
                raise ScmcInputError("rng can not be used while using parfor")
            cfg["rng"] = float(np.asarray(val).reshape(-1)[0])
        elif opt in ("CBS", "uniformFirstScatter", "renderCov", "singleScattering", "multipleScattering",
                     "renderField"):
            if not _is_logical_scalar(val):
                raise ScmcInputError({
                    "CBS": "CBS must be logical scalar",
                    "uniformFirstScatter": "uniformFirstScatter must be logical scalar",
                    "renderCov": "renderCov must be logical scalar",
                    "singleScattering": "Single scattering option must be logical scalar",
                    "multipleScattering": "Multiple scattering option must be logical scalar",
                    "renderField": "renderField must be logical scalar"}[opt])
            v = bool(val)
            if opt == "CBS":
                cfg["CBS"] = v
            elif opt == "uniformFirstScatter":
                cfg["uniformFirstScatter"] = v
            elif opt == "renderCov":
                cfg["render"]["cov"] = v
            elif opt == "singleScattering":
                cfg["render"]["singleScattering"] = v
            elif opt == "multipleScattering":
                cfg["render"]["multipleScattering"] = v
            else:
                cfg["render"]["field"] = v
        else:
            raise ScmcInputError("Invalid option value")
    return cfg


def kernel_arguments(cfg: dict):
    """scmc.m:244-323: the positional MCcov / MCfield argument list."""
    ta, sc = cfg["targetArea"], cfg["scatter"]
    sigt = 1.0 / ta["MFP"]
    albedo = sc["albedo"]
    fn = sc["function"]
    extra = []
    if fn == "isotropic":
        sct_type, ampfunc = 1, 0
    elif fn == "tabulated":
        sct_type, ampfunc = 2, sc["ampfunc"]
        a0 = sc.get("ampfunc0", math.inf)
        if not (np.isscalar(a0) and math.isinf(a0)):
            extra = [a0]
    elif fn == "HG":
        sct_type, ampfunc = 3, sc["g"]
        if not math.isinf(sc["g0"]):
            extra = [sc["g0"]]
    else:
        raise ScmcInputError("Invalid scatter input")
    if ta["D"] == 3:
        box_min = np.array([ta["x"][0], ta["y"][0], ta["z"][0]], dtype=float)
        box_max = np.array([ta["x"][1], ta["y"][1], ta["z"][1]], dtype=float)
    else:
        box_min = np.array([ta["x"][0], ta["z"][0]], dtype=float)
        box_max = np.array([ta["x"][1], ta["z"][1]], dtype=float)
    lt, vw = cfg["lights"], cfg["views"]
    is_ff_l = 1 if lt["farField"] == 1 else 0
    l = lt["directions"] if is_ff_l else lt["positions"]
    is_ff_v = 1 if vw["farField"] == 1 else 0
    v = vw["directions"] if is_ff_v else vw["positions"]
    max_itr = cfg["render"]["iterations"]
    smp_flg = 1 if cfg["uniformFirstScatter"] else 2
    args = [sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, max_itr, ta["wavelength"],
            cfg["CBS"], smp_flg, sct_type, ampfunc] + extra
    return args


def run_config(cfg: dict, kernels) -> dict:
    """scmc.m:241-427 with the replicas of parforIters folded into one run."""
    mul = {"Config": cfg}
    args = kernel_arguments(cfg)
    reps = int(cfg["parforIters"])
    max_itr = int(args[8])
    total = max_itr * max(reps, 1)
    run_args = list(args)
    run_args[8] = total
    if cfg["render"]["cov"]:
        if reps == 1 and cfg["rng"] != -1:
            _mc.rng(cfg["rng"])
        Ms, Mm = kernels.MCcov(*run_args, seed=_mc.draw_seed(), n_total=total)
        if cfg["render"]["singleScattering"]:
            mul["Csingle"] = Ms
        if cfg["render"]["multipleScattering"]:
            mul["C"] = Ms + Mm
    if cfg["render"]["field"]:
        if reps == 1 and cfg["rng"] != -1:
            _mc.rng(cfg["rng"])
        fargs = run_args[:15] if len(run_args) > 14 else run_args
        mul["field"] = kernels.MCfield(*fargs, seed=_mc.draw_seed(), n_total=total)
    return mul


def scmc(targetArea, views=None, lights=None, scatter=None, iterations=None, *varargin, **gpu):
    """Run SCMC; keyword-only `precision`, `device`, `max_events_per_path` select GPU controls."""
    if views is None and lights is None and scatter is None and iterations is None:
        cfg = targetArea  # scmc(Config), scmc.m:236-239
    else:
        if iterations is None:
            raise ScmcInputError("Not enough input arguments.")
        cfg = build_config(targetArea, views, lights, scatter, iterations, *varargin)
    return run_config(cfg, _GpuKernels(**gpu))
