"""Seeded MCfield / MCcov argument sets shared by the parity tests."""
import numpy as np

from mcspeckle_b200 import interface as I


def cap_dirs(n, half_deg, zsign, seed):
    """n directions uniform on the solid-angle cap <= half_deg about zsign*z."""
    g = np.random.default_rng(seed)
    c = g.uniform(np.cos(np.deg2rad(half_deg)), 1.0, n)
    phi = g.uniform(0, 2 * np.pi, n)
    s = np.sqrt(1 - c * c)
    return np.stack([s * np.cos(phi), s * np.sin(phi), zsign * c])


def grid_dirs(n_side, half_deg, zsign):
    """n_side^2 directions on a regular (sin theta_x, sin theta_y) grid."""
    s = np.sin(np.deg2rad(half_deg))
    g = np.linspace(-s, s, n_side)
    sx, sy = np.meshgrid(g, g, indexing="ij")
    sx, sy = sx.reshape(-1), sy.reshape(-1)
    return np.stack([sx, sy, zsign * np.sqrt(1 - sx * sx - sy * sy)])


def hg_table_3d(g=0.7, n=1001):
    th = np.linspace(0, 1, n) * np.pi
    th[-1] = np.pi
    c = np.cos(th)
    f = np.sqrt((1 - g * g) / (4 * np.pi * (1 + g * g - 2 * g * c) ** 1.5))
    s = I.tabulatedAmplitudeScatter(th, f)
    return {"evalAmp": s["ampfunc"]["evalAmp"], "sampleIcdf": s["ampfunc"]["sampleIcdf"]}


def hg_table_2d(g=0.5, n=2001):
    th = np.linspace(0, 1, n) * 2 * np.pi
    th[-1] = 2 * np.pi
    c = np.cos(th)
    f = np.sqrt((1 - g * g) / (2 * np.pi * (1 + g * g - 2 * g * c)))
    s = I.tabulatedAmplitudeScatter(th, f)
    return {"evalAmp": s["ampfunc"]["evalAmp"], "sampleIcdf": s["ampfunc"]["sampleIcdf"]}


BOX3 = ([-20.0, -20.0, 0.0], [20.0, 20.0, 15.0])
BOX2 = ([-20.0, 0.0], [20.0, 15.0])
NF_V = np.array([[-5.0, 0.0, 6.0, 2.0], [1.0, -3.0, 2.0, 0.5], [-30.0, -30.0, -28.0, 40.0]])
NF_L = np.array([[0.0, 4.0, -6.0], [2.0, -1.0, 3.0], [-35.0, -40.0, -30.0]])


def small_cases(n_paths=300):
    """(name, positional MCfield/MCcov args without ampfunc0/lmean0 extras, extras)."""
    L3 = cap_dirs(3, 10, +1, 11)
    V3r = cap_dirs(4, 10, -1, 12)
    V3t = cap_dirs(4, 10, +1, 13)
    t3 = hg_table_3d()
    t2 = hg_table_2d()
    c = dict(sigt=0.2, albedo=0.9, lam=1.0)

    def args(box, l, v, ffl, ffv, cbs, smp, sct, amp, sigt=c["sigt"], albedo=c["albedo"], lam=c["lam"], n=n_paths):
        return [sigt, albedo, np.asarray(box[0]), np.asarray(box[1]), l, v, ffl, ffv, n, lam, cbs, smp, sct, amp]

    return [
        ("3d_iso_ff_refl_cbs_exp", args(BOX3, L3, V3r, 1, 1, True, 2, 1, 0), []),
        ("3d_hg_ff_trans_nocbs_unif", args(BOX3, L3, V3t, 1, 1, False, 1, 3, 0.8), []),
        ("3d_hg_nfv_cbs_exp_g0", args(BOX3, L3, NF_V, 1, 0, True, 2, 3, 0.6), [0.3]),
        ("3d_tab_nfl_nfv_cbs_exp", args(BOX3, NF_L, NF_V, 0, 0, True, 2, 2, t3), []),
        ("3d_tab_ff_refl_cbs_unif_t0", args(BOX3, L3, V3r, 1, 1, True, 1, 2, t3), [t3]),
        ("3d_iso_lowalbedo", args(BOX3, L3, V3r, 1, 1, True, 2, 1, 0, sigt=0.3, albedo=0.5, lam=0.7), []),
        ("2d_iso_angles_cbs_exp", args(BOX2, np.deg2rad([[0.0, 3.0, -4.0]]), np.deg2rad([[180.0, 170.0, 185.0, 200.0]]),
                                       1, 1, True, 2, 1, 0), []),
        ("2d_hg_nocbs_unif", args(BOX2, np.array([[0.1, -0.2], [1.0, 1.0]]) / np.hypot([0.1, -0.2], 1.0),
                                  np.array([[0.0, 0.3, -0.1], [1.0, 1.0, 1.0]]) / np.hypot([0.0, 0.3, -0.1], 1.0),
                                  1, 1, False, 1, 3, -0.4), []),
        ("2d_tab_cbs_exp", args(BOX2, np.deg2rad([[0.0, 20.0]]), np.deg2rad([[0.0, 90.0, 180.0, 270.0]]),
                                1, 1, True, 2, 2, t2), []),
    ]
