"""Parameter-struct constructors of SCMC's interface/ folder.

Each returns a dict with the reference struct's field names, so code written
against the MATLAB structs reads the same.  Validation and error strings
follow the reference files cited on each function.
"""
from __future__ import annotations

import math

import numpy as np


class InterfaceError(ValueError):
    """Invalid constructor input; the message is the reference's error() text."""


def _is_scalar(x) -> bool:
    return np.asarray(x).size == 1


def _scalar(x) -> float:
    return float(np.asarray(x).reshape(-1)[0])


def boxArea(wavelength, MFP, z, x, *y):
    """interface/targetArea/boxArea.m:1-65 (2-D with 4 args, 3-D with 5)."""
    if len(y) > 1:
        raise InterfaceError("Too many input arguments.")
    if not _is_scalar(wavelength) or not _is_scalar(MFP):
        raise InterfaceError("wavelength and MFP are scalars")
    z = np.asarray(z, dtype=float).reshape(-1)
    x = np.asarray(x, dtype=float).reshape(-1)
    yy = np.asarray(y[0], dtype=float).reshape(-1) if y else None
    if z.size != 2 or x.size != 2 or (yy is not None and yy.size != 2):
        raise InterfaceError("x, y and z defined as 2 elements vectors")
    if z[0] > z[1]:
        raise InterfaceError("z(1) must be smaller than z(2)")
    if x[0] > x[1]:
        raise InterfaceError("x(1) must be smaller than x(2)")
    if yy is not None and yy[0] > yy[1]:
        raise InterfaceError("y(1) must be smaller than y(2)")
    t = {"type": "targetArea", "wavelength": _scalar(wavelength), "MFP": _scalar(MFP), "z": z, "x": x}
    if yy is None:
        t["D"] = 2
    else:
        t["D"] = 3
        t["y"] = yy
    return t


def farFieldSource(in1, *rest):
    """interface/source/farFieldSource.m:1-57.

    farFieldSource(directions) normalises the 2xN / 3xN columns;
    farFieldSource(theta, 0) builds [sin; cos] (2-D) and [sin; 0; cos] (3-D).
    """
    if len(rest) > 1:
        raise InterfaceError("Too many input arguments.")
    src = {"type": "source", "farField": 1}
    if not rest:
        d = np.asarray(in1, dtype=float)
        if d.ndim == 1:
            d = d.reshape(-1, 1) if d.size in (2, 3) else d.reshape(1, -1)
        if d.shape[0] not in (2, 3):
            raise InterfaceError("Invalid positions elements number")
        src["count"] = d.shape[1]
        src["directions"] = d / np.sqrt(np.sum(np.abs(d) ** 2, axis=0))
    else:
        th = np.asarray(in1, dtype=float)
        if not (th.ndim <= 1 or min(th.shape) == 1):
            raise InterfaceError("theta must be vector of directions")
        th = th.reshape(-1)
        src["count"] = th.size
        src["directions2D"] = np.stack([np.sin(th), np.cos(th)])
        src["directions3D"] = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)])
    return src


def nearFieldSource(in1, *rest):
    """interface/source/nearFieldSource.m:1-91 (positions / (r, theta) / (X, Y, N))."""
    if len(rest) > 2:
        raise InterfaceError("Too many input arguments.")
    src = {"type": "source", "farField": 0}
    if not rest:
        p = np.asarray(in1, dtype=float)
        if p.ndim == 1:
            p = p.reshape(-1, 1)
        if p.shape[0] not in (2, 3):
            raise InterfaceError("Invalid positions elements number")
        src["count"] = p.shape[1]
        src["positions"] = p
    elif len(rest) == 1:
        r, th = in1, np.asarray(rest[0], dtype=float)
        if not (_is_scalar(r) and _scalar(r) > 0):
            raise InterfaceError("r must be positive scalar")
        if not (th.ndim <= 1 or min(th.shape) == 1):
            raise InterfaceError("theta must be vector of directions")
        th = th.reshape(-1)
        r = _scalar(r)
        src["count"] = th.size
        src["positions2D"] = r * np.stack([np.sin(th), np.cos(th)])
        src["positions3D"] = r * np.stack([np.sin(th), np.zeros_like(th), np.cos(th)])
    else:
        X = np.asarray(in1, dtype=float)
        Y = np.asarray(rest[0], dtype=float)
        n = rest[1]
        X = X.reshape(-1, 1) if X.ndim == 1 else X
        Y = Y.reshape(-1, 1) if Y.ndim == 1 else Y
        if X.shape[0] not in (2, 3) or X.shape[1] != 1:
            raise InterfaceError("Invalid X position")
        if Y.shape[0] not in (2, 3) or Y.shape[1] != 1:
            raise InterfaceError("Invalid Y position")
        if X.shape[0] != Y.shape[0]:
            raise InterfaceError("Both points must have the same diamentions")
        if not (_is_scalar(n) and float(n) == int(float(n)) and float(n) > 0):
            raise InterfaceError("Number of input points must be positive integer")
        n = int(float(n))
        src["count"] = n
        src["positions"] = np.stack([np.linspace(X[k, 0], Y[k, 0], n) for k in range(X.shape[0])])
    return src


def isotropicScatter(*albedo):
    """interface/scatter/isotropicScatter.m:1-33."""
    if len(albedo) > 1:
        raise InterfaceError("Too many input arguments.")
    s = {"type": "scatter", "function": "isotropic", "albedo": 1.0}
    if albedo:
        a = albedo[0]
        if not _is_scalar(a) or _scalar(a) < 0 or _scalar(a) > 1:
            raise InterfaceError("Invalid albedo input")
        s["albedo"] = _scalar(a)
    return s


def HGScatter(g, *rest):
    """interface/scatter/HGScatter.m:1-56: HGScatter(g[, g0[, albedo]])."""
    if len(rest) > 4:
        raise InterfaceError("Too many input arguments.")
    s = {"type": "scatter", "function": "HG", "albedo": 1.0, "g0": math.inf}
    if len(rest) >= 2:
        a = rest[1]
        if not _is_scalar(a) or _scalar(a) < 0 or _scalar(a) > 1:
            raise InterfaceError("Invalid albedo input")
        s["albedo"] = _scalar(a)
    if len(rest) >= 1:
        g0 = rest[0]
        if not _is_scalar(g0) or _scalar(g0) < -1 or _scalar(g0) > 1:
            raise InterfaceError("Invalid g0 input")
        s["g0"] = _scalar(g0)
    if not _is_scalar(g) or _scalar(g) < -1 or _scalar(g) > 1:
        raise InterfaceError("Invalid g input")
    s["g"] = _scalar(g)
    return s


def invCDF(cdf, dim):
    """code/coreFunctions/invCDF.m:1-18: nearest-grid inverse CDF, as angles."""
    cdf = np.asarray(cdf, dtype=float).reshape(-1)
    n = cdf.size
    grid = np.arange(n) * (1.0 / (n - 1))
    # [~, icdf(j)] = min(abs(cdf - grid(j))): first index of the minimum
    icdf = np.empty(n)
    for j in range(n):
        icdf[j] = np.argmin(np.abs(cdf - grid[j])) + 1
    if dim == 2:
        icdf = icdf / n * 2 * math.pi
    if dim == 3:
        icdf = icdf / n * math.pi
    return icdf


def _strictly_monotonic(x) -> bool:
    d = np.diff(np.asarray(x, dtype=float).reshape(-1))
    return bool(np.all(d > 0) or np.all(d < 0))


def tabulatedAmplitudeScatter(theta, f, *albedo):
    """interface/scatter/tabulatedAmplitudeScatter.m:1-101.

    Builds the cross section, the sampling pdf / cdf / inverse cdf and the
    normalised complex amplitude table from a measured amplitude f(theta).
    """
    if len(albedo) > 1:
        raise InterfaceError("Too many input arguments.")
    s = {"albedo": _scalar(albedo[0]) if albedo else 1.0, "type": "scatter", "function": "tabulated"}
    th = np.asarray(theta, dtype=float)
    fv = np.asarray(f)
    if not (th.ndim <= 1 or min(th.shape) == 1) or not (fv.ndim <= 1 or min(fv.shape) == 1):
        raise InterfaceError("theta and f must be vectors")
    th = th.reshape(-1)
    fv = fv.reshape(-1)
    if th.size != fv.size:
        raise InterfaceError("theta and f must have same elements number")
    if not _strictly_monotonic(th):
        raise InterfaceError("theta must be monotonic increasing")
    if th[0] == 0 and th[-1] == 2 * math.pi:
        s["D"] = 2
    elif th[0] == 0 and th[-1] == math.pi:
        s["D"] = 3
    else:
        raise InterfaceError("theta must be from 0 to 2pi in 2D or -1 to 1 in 3D")
    a2 = np.abs(fv) ** 2
    amp = {"theta": th.copy()}
    if s["D"] == 2:
        amp["cs"] = np.mean(a2) * 2 * math.pi
        amp["samplePdf"] = a2 / np.sum(a2)
    else:
        amp["cs"] = np.mean(a2 * np.sin(th)) * 2 * math.pi ** 2
        amp["samplePdf"] = a2 * np.sin(th) / np.sum(a2 * np.sin(th))
    amp["sampleCdf"] = np.cumsum(amp["samplePdf"])
    amp["sampleIcdf"] = invCDF(amp["sampleCdf"], s["D"])
    amp["evalPdf"] = a2 / amp["cs"]
    amp["evalAmp"] = amp["evalPdf"] ** 0.5 * np.exp(1j * np.angle(fv))
    s["ampfunc"] = amp
    return s


def tabulatedAmplitudeScatterCos(cs, f, *albedo):
    """Extension (3-D): a measured amplitude f tabulated on cos(theta) bins
    cs = 1 - 2i/(n-1), i = 0 .. n-1 (forward first), the form of the
    tabulated phase function of the heterogeneous configuration.  Built as
    tabulatedAmplitudeScatter.m:75-99 builds the angle-bin tables, with the
    measure dOmega = 2 pi dcos: cross section 4 pi mean(|f|^2), sampling pdf
    |f|^2 / sum |f|^2 over the bins, the inverse CDF by the nearest-grid
    search of invCDF.m returning the bin's cosine, evalAmp = sqrt(|f|^2 / cs)
    with f's phase.  The tables carry cosBins = True."""
    if len(albedo) > 1:
        raise InterfaceError("Too many input arguments.")
    c = np.asarray(cs, dtype=float).reshape(-1)
    fv = np.asarray(f).reshape(-1)
    n = c.size
    if fv.size != n or n < 2:
        raise InterfaceError("cs and f must have same elements number")
    if not np.allclose(c, 1.0 - 2.0 * np.arange(n) / (n - 1), rtol=0, atol=1e-12):
        raise InterfaceError("cs must be the bins 1 - 2i/(n-1)")
    a2 = np.abs(fv) ** 2
    amp = {"cosBins": True, "cs_bins": c.copy(), "cs": float(np.mean(a2)) * 4 * math.pi}
    amp["samplePdf"] = a2 / np.sum(a2)
    amp["sampleCdf"] = np.cumsum(amp["samplePdf"])
    grid = np.arange(n) * (1.0 / (n - 1))
    idx = np.array([np.argmin(np.abs(amp["sampleCdf"] - grid[j])) for j in range(n)])
    amp["sampleIcdf"] = c[idx]
    amp["evalPdf"] = a2 / amp["cs"]
    amp["evalAmp"] = amp["evalPdf"] ** 0.5 * np.exp(1j * np.angle(fv))
    return {"albedo": _scalar(albedo[0]) if albedo else 1.0, "type": "scatter", "function": "tabulated", "D": 3,
            "ampfunc": amp}
