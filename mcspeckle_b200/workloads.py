"""Seeded synthetic inputs of the five measured configurations.

Each builder returns the arguments of one solve in the reference's own
calling form (the positional lists of MCfield / MCcov / MCfieldFourierQuad /
MCCovHetro), so the same media and directions serve the benchmark and the
parity tests.  Every random choice comes from a fixed seed.

  field16    MCfield far field, 16 lights x 16 views within 10 deg of +z / -z,
             isotropic, box 20 x 20 x 5 MFP (MFP 10 wavelengths), CBS.
  cov64      MCcov far-field covariance, 64 lights x 64 views on 8 x 8
             (sin theta_x, sin theta_y) grids of +-5 deg, HG g = 0.8,
             sigma_s = 1, sigma_a = 0.01 per MFP, same box.
  fq256      MCfieldFourierQuad, box 50 x 50 x 10 MFP (MFP 100 wavelengths),
             sigma_a = 0.005 per MFP, 256 x 256 angular grid at a
             0.5-wavelength lateral pitch, CBS; the reference's isotropic
             plane-wave form, or HG g = 0.9 with a point source 2 MFP deep.
  hetero128  MCCovHetro, sigma_s on a 128^3 grid, log-normal(0, 0.5) per MFP,
             box 20 x 20 x 5 MFP, tabulated phase function on 1024 bins from a
             seeded mixture of 3 HG lobes, 128 lights x 128 views; trilinear
             sigma and cos(theta) bins as the configuration states them, or
             the reference's nearest voxel and angle bins.
  served     uneven MCfield requests (lights 1-256, views 1-1024, log-uniform
             path budgets, media drawn per request).
"""
from __future__ import annotations

import math

import numpy as np


def cap_dirs(n, half_deg, zsign, rng):
    """n directions uniform on the solid-angle cap <= half_deg about zsign*z."""
    c = rng.uniform(math.cos(math.radians(half_deg)), 1.0, n)
    phi = rng.uniform(0, 2 * math.pi, n)
    s = np.sqrt(1 - c * c)
    return np.stack([s * np.cos(phi), s * np.sin(phi), zsign * c])


def grid_rect(nx, ny, half_deg, zsign):
    """nx x ny directions on a regular (sin theta_x, sin theta_y) grid."""
    s = math.sin(math.radians(half_deg))
    sx, sy = np.meshgrid(np.linspace(-s, s, nx), np.linspace(-s, s, ny), indexing="ij")
    sx, sy = sx.reshape(-1), sy.reshape(-1)
    return np.stack([sx, sy, zsign * np.sqrt(1 - sx * sx - sy * sy)])


def hg_table(g, n=1001):
    """A tabulated phase function (tabulatedAmplitudeScatter of one HG lobe)."""
    from . import interface as I
    th = np.linspace(0, 1, n) * np.pi
    f = np.sqrt((1 - g * g) / (4 * np.pi * (1 + g * g - 2 * g * np.cos(th)) ** 1.5))
    t = I.tabulatedAmplitudeScatter(th, f)["ampfunc"]
    return {"evalAmp": t["evalAmp"], "sampleIcdf": t["sampleIcdf"]}


def hg_mixture_table(n_bins, seed, cos_bins=False):
    """Tabulated amplitude of a seeded mixture of 3 HG lobes (g in [-0.3, 0.95],
    weights from Dirichlet(1,1,1)) on n_bins angles in [0, pi] (the
    reference's tables), or on n_bins cos(theta) bins (the extension)."""
    from . import interface as I
    g_rng = np.random.default_rng(seed)
    gs = g_rng.uniform(-0.3, 0.95, 3)
    w = g_rng.dirichlet([1.0, 1.0, 1.0])
    if cos_bins:
        c = 1.0 - 2.0 * np.arange(n_bins) / (n_bins - 1)
    else:
        th = np.linspace(0, 1, n_bins) * np.pi
        c = np.cos(th)
    pdf = sum(wk * (1 - gk * gk) / (4 * np.pi * (1 + gk * gk - 2 * gk * c) ** 1.5) for wk, gk in zip(w, gs))
    if cos_bins:
        t = I.tabulatedAmplitudeScatterCos(c, np.sqrt(pdf))["ampfunc"]
        return {"evalAmp": t["evalAmp"], "sampleIcdf": t["sampleIcdf"], "cosBins": True}, gs.tolist(), w.tolist()
    t = I.tabulatedAmplitudeScatter(th, np.sqrt(pdf))["ampfunc"]
    return {"evalAmp": t["evalAmp"], "sampleIcdf": t["sampleIcdf"]}, gs.tolist(), w.tolist()


# ---------------------------------------------------------------------------
# field16 and cov64: positional MCfield / MCcov lists
# ---------------------------------------------------------------------------
FIELD16 = ("MCfield far field, 16 lights x 16 views within 10 deg of +z / -z, isotropic, box 20x20x5 MFP "
           "(MFP 10 wavelengths), CBS")
COV64 = "MCcov far-field covariance, 64 lights x 64 views (8x8 grids, +-5 deg), HG g=0.8, box 20x20x5 MFP"


def field16_args(n_paths):
    rng = np.random.default_rng(0)
    l16 = cap_dirs(16, 10.0, +1.0, rng)
    v16 = cap_dirs(16, 10.0, -1.0, rng)
    return [0.1, 1.0, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]), l16, v16, 1, 1,
            int(n_paths), 1.0, True, 2, 1, 0]


def cov64_args(n_paths):
    mfp = 10.0
    sigt = 1.01 / mfp          # sigma_s + sigma_a = (1 + 0.01) / MFP
    albedo = 1.0 / 1.01
    box_min = np.array([-100.0, -100.0, 0.0])
    box_max = np.array([100.0, 100.0, 50.0])
    l = grid_rect(8, 8, 5.0, +1.0)
    v = grid_rect(8, 8, 5.0, -1.0)
    return [sigt, albedo, box_min, box_max, l, v, 1, 1, int(n_paths), 1.0, True, 2, 3, 0.8]


# ---------------------------------------------------------------------------
# fq256: MCfieldFourierQuad
# ---------------------------------------------------------------------------
FQ_MFP = 100.0
FQ_V_MAX = 255.0 / 256.0
FQ_V_STP = 1.0 / 128.0


def fq256_desc(extended):
    base = ("MCfieldFourierQuad, box 50x50x10 MFP (MFP 100 wavelengths), sigma_a 0.005 per MFP, 256x256 angular "
            "grid (v_max 255/256, v_stp 1/128: 0.5-wavelength lateral pitch), CBS")
    if extended:
        return base + ", HG g=0.9 direction sampling, point source 2 MFP deep (near-field light factor)"
    return base + ", isotropic plane wave along +z (the reference's form)"


def fq256_args(n, *, extended, seed, precision, path_offset=0):
    from . import fourier_quad as FQ
    mfp = FQ_MFP
    sigt, albedo = 1.005 / mfp, 1 / 1.005
    bmin, bmax = [-25 * mfp, -25 * mfp, 0.0], [25 * mfp, 25 * mfp, 10 * mfp]
    if extended:
        src = np.array([[0.0], [0.0], [2 * mfp]])  # a point source 2 MFP deep
        return FQ.fq_args(sigt, albedo, bmin, bmax, src, FQ_V_MAX, FQ_V_STP, int(n), 1.0, True, 2, None, -1,
                          seed=seed, precision=precision, path_offset=path_offset, light_point=True, hg_g=0.9)
    l = np.array([[0.0], [0.0], [1.0]])
    return FQ.fq_args(sigt, albedo, bmin, bmax, l, FQ_V_MAX, FQ_V_STP, int(n), 1.0, True, 2, None, -1, seed=seed,
                      precision=precision, path_offset=path_offset)


def fq256_propagating():
    """Mask of the grid directions with vx^2 + vy^2 < 1 (256 x 256 x 1): where
    it is 1 or more the reference's plane factor exp(zexp0 tz) grows with depth
    (evanescent directions), so errors are measured over this mask."""
    th = -FQ_V_MAX + np.arange(256) * FQ_V_STP
    return (th[:, None] ** 2 + th[None, :] ** 2 < 1.0)[:, :, None]


# ---------------------------------------------------------------------------
# hetero128: MCCovHetro
# ---------------------------------------------------------------------------
_HGRID = {}


def hetero128_medium(extended=False):
    """(sigma grid 128^3, tabulated table, lobe g's, lobe weights); cached.
    extended: the table on cos(theta) bins instead of angle bins."""
    key = "ext" if extended else "ref"
    if key not in _HGRID:
        mfp = 10.0
        g = np.random.default_rng(4)
        sig = np.exp(g.normal(0.0, 0.5, (128, 128, 128))) / mfp
        table, gs, ws = hg_mixture_table(1024, 5, cos_bins=extended)
        _HGRID[key] = (sig, table, gs, ws)
    return _HGRID[key]


def hetero128_desc(extended=True):
    _, _, gs, ws = hetero128_medium(extended)
    lookup = "trilinear between voxel centres" if extended else "nearest voxel as the reference"
    bins = "cos(theta)" if extended else "theta"
    return (f"MCCovHetro, sigma_s on a 128^3 grid log-normal(0, 0.5) per MFP (MFP 10 wavelengths, {lookup}), box "
            f"20x20x5 MFP, Woodcock tracking, tabulated phase function on 1024 {bins} bins from 3 HG lobes "
            f"g={[round(x, 3) for x in gs]} w={[round(x, 3) for x in ws]}, 128 lights x 128 views (16x8 grids of "
            f"+-5 deg), CBS")


def hetero128_args(n, *, seed, precision, path_offset=0, norm_itr=0, extended=True):
    """extended: trilinear sigma and the cos(theta)-bin table (the
    configuration as stated); False: the reference's nearest voxel and angle
    bins."""
    from . import hetero as H
    sig, table, _, _ = hetero128_medium(extended)
    bmin, bmax = np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0])
    bbin = (bmax - bmin) / 128.0
    l = grid_rect(16, 8, 5.0, +1.0)
    v = grid_rect(16, 8, 5.0, -1.0)
    return H.hetero_args(True, sig, 1.0, bmin, bmax, bbin, l, v, 1, 1, int(n), 1.0, True, 2, 2, table, seed=seed,
                         precision=precision, path_offset=path_offset, norm_itr=norm_itr, trilinear=extended)


# ---------------------------------------------------------------------------
# served stream
# ---------------------------------------------------------------------------
SERVED = ("served MCfield stream: lights 1-256, views 1-1024, paths log-uniform; box 5-50 MFP "
          "(MFP 10 wavelengths, thickness 1/4 of the side), HG g~U(0,0.95), sigma_a~U(0,0.05), "
          "isotropic/HG/tabulated 1:2:1, far field, CBS, Poisson arrivals")


def served_requests(n, seed=5, paths=(1e5, 1e8), nv_max=1024, nl_max=256, side_mfp=(5.0, 50.0)):
    """n MCfield requests with log-uniform sizes and budgets and media drawn per
    request.  Returns dicts with the positional MCfield arguments, the Philox
    key and the sizes."""
    rng = np.random.default_rng(seed)

    def logu(lo, hi):
        return math.exp(rng.uniform(math.log(lo), math.log(hi)))

    out = []
    mfp = 10.0
    for i in range(n):
        nl = max(1, min(nl_max, int(round(logu(1, nl_max)))))
        nv = max(1, min(nv_max, int(round(logu(1, nv_max)))))
        n_paths = int(round(logu(*paths)))
        side = logu(*side_mfp) * mfp
        g = float(rng.uniform(0.0, 0.95))
        sa = float(rng.uniform(0.0, 0.05))
        kind = ["iso", "hg", "hg", "tab"][int(rng.integers(0, 4))]
        sct, amp = {"iso": (1, 0), "hg": (3, g), "tab": (2, None)}[kind]
        if kind == "tab":
            amp = hg_table(g)
        l = cap_dirs(nl, 10.0, +1.0, rng)
        v = cap_dirs(nv, 10.0, -1.0, rng)
        args = [(1.0 + sa) / mfp, 1.0 / (1.0 + sa), np.array([-side / 2, -side / 2, 0.0]),
                np.array([side / 2, side / 2, side / 4]), l, v, 1, 1, n_paths, 1.0, True, 2, sct, amp]
        out.append({"args": args, "seed": 0x5E4E0000 + i, "paths": n_paths, "nv": nv, "nl": nl, "scatter": kind})
    return out
