"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own .m files (read in place from the reference tree,
never copied) through the MATLAB-subset interpreter in mlite.py, with
`rand` / `randn` served from seeded tapes, and stores for every case the
arguments, the consumed prefix of each tape and the outputs.  The oracle,
fed the same tapes, must reproduce these outputs (tests/test_oracle_golden.py).

Usage (in a container that has the reference tree; the path is required,
as an argument or in SCMC_REFERENCE_TREE):
    python tests/golden/make_golden.py /path/to/mcspeckle
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import mlite as ml  # noqa: E402

M = ml.M
TAPE_LEN = 200_000


def tapes(seed):
    g = np.random.default_rng(seed)
    return g.random(TAPE_LEN), g.standard_normal(TAPE_LEN)


def norm_cols(a):
    a = np.asarray(a, dtype=float)
    return a / np.linalg.norm(a, axis=0, keepdims=True)


def cap_dirs(n, half_deg, zsign, seed):
    """n directions uniform on the solid-angle cap <= half_deg about zsign*z."""
    g = np.random.default_rng(seed)
    c = g.uniform(np.cos(np.deg2rad(half_deg)), 1.0, n)
    phi = g.uniform(0, 2 * np.pi, n)
    s = np.sqrt(1 - c * c)
    return np.stack([s * np.cos(phi), s * np.sin(phi), zsign * c])


def to_m(x):
    if isinstance(x, dict):
        st = ml.MStruct()
        for k, v in x.items():
            st[k] = to_m(v)
        return st
    if isinstance(x, str):
        return ml.MStr(x)
    if isinstance(x, bool):
        return M(x)
    return M(np.asarray(x, dtype=complex if np.iscomplexobj(x) else float))


def struct_to_py(st):
    out = {}
    for k, v in st.items():
        if isinstance(v, ml.MStruct):
            out[k] = struct_to_py(v)
        elif isinstance(v, ml.MStr):
            out[k] = str(v)
        else:
            out[k] = np.asarray(v)
    return out


class Gen:
    def __init__(self, ref):
        self.ref = ref
        self.path = ml.reference_search_path(ref)
        self.index = []

    def interp(self, seed):
        ut, nt = tapes(seed)
        return ml.Interp(self.path, ut, nt), ut, nt

    def save(self, name, kind, meta, arrays):
        fn = f"{name}.npz"
        np.savez_compressed(os.path.join(HERE, fn), meta=json.dumps(meta), **arrays)
        self.index.append({"name": name, "kind": kind, "file": fn})
        print(f"  {name}: " + ", ".join(f"{k}{list(np.shape(v))}" for k, v in arrays.items()))

    # -- MCfield / MCcov ------------------------------------------------------
    def mc_case(self, name, func, seed, *, sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v,
                max_itr, lam, cbs, smp_flg, sct_type, ampfunc, ampfunc0=None, lmean0=None):
        it, ut, nt = self.interp(seed)
        args = [M(float(sigt)), M(float(albedo)), M(np.reshape(box_min, (-1, 1)).astype(float)),
                M(np.reshape(box_max, (-1, 1)).astype(float)), M(np.asarray(l, float)),
                M(np.asarray(v, float)), M(bool(is_ff_l)), M(bool(is_ff_v)), M(float(max_itr)),
                M(float(lam)), M(bool(cbs)), M(float(smp_flg)), M(float(sct_type)), to_m(ampfunc)]
        if ampfunc0 is not None:
            args.append(to_m(ampfunc0))
        if lmean0 is not None:
            args.append(M(np.reshape(lmean0, (-1, 1)).astype(float)))
        nout = 1 if func == "MCfield" else 2
        outs = it.call(func, args, nout)
        arrays = {"utape": ut[:it.ui], "ntape": nt[:it.ni], "box_min": np.asarray(box_min, float),
                  "box_max": np.asarray(box_max, float), "l": np.asarray(l, float),
                  "v": np.asarray(v, float)}
        meta = {"func": func, "sigt": sigt, "albedo": albedo, "is_ff_l": bool(is_ff_l),
                "is_ff_v": bool(is_ff_v), "max_itr": max_itr, "lambda": lam, "cbs": bool(cbs),
                "smp_flg": smp_flg, "sct_type": sct_type, "has_ampfunc0": ampfunc0 is not None,
                "has_lmean0": lmean0 is not None}
        self._put_amp(arrays, meta, "ampfunc", ampfunc)
        if ampfunc0 is not None:
            self._put_amp(arrays, meta, "ampfunc0", ampfunc0)
        if lmean0 is not None:
            arrays["lmean0"] = np.asarray(lmean0, float)
        if func == "MCfield":
            arrays["u"] = np.asarray(outs[0], dtype=complex)
        else:
            arrays["Ms"] = np.asarray(outs[0], dtype=complex)
            arrays["Mm"] = np.asarray(outs[1], dtype=complex)
        self.save(name, func, meta, arrays)

    # -- MCfieldOnWave ---------------------------------------------------------
    def onwave_case(self, name, seed, *, sigt, albedo, box_min, box_max, l, v, is_ff_l, is_ff_v, max_itr, lam, cbs,
                    smp_flg, sct_type, ampfunc, ampfunc0, lmean0, Wl):
        """MCfieldOnWave takes ampfunc0, lmean0 and Wl positionally (17 arguments);
        Wl is passed as a 1 x Nl row, the shape its element-wise products need."""
        it, ut, nt = self.interp(seed)
        args = [M(float(sigt)), M(float(albedo)), M(np.reshape(box_min, (-1, 1)).astype(float)),
                M(np.reshape(box_max, (-1, 1)).astype(float)), M(np.asarray(l, float)),
                M(np.asarray(v, float)), M(bool(is_ff_l)), M(bool(is_ff_v)), M(float(max_itr)),
                M(float(lam)), M(bool(cbs)), M(float(smp_flg)), M(float(sct_type)), to_m(ampfunc), to_m(ampfunc0),
                M(np.reshape(lmean0, (-1, 1)).astype(float)), M(np.asarray(Wl, complex).reshape(1, -1))]
        u = it.call("MCfieldOnWave", args, 1)[0]
        arrays = {"utape": ut[:it.ui], "ntape": nt[:it.ni], "box_min": np.asarray(box_min, float),
                  "box_max": np.asarray(box_max, float), "l": np.asarray(l, float), "v": np.asarray(v, float),
                  "lmean0": np.asarray(lmean0, float), "Wl": np.asarray(Wl, complex).reshape(-1),
                  "u": np.asarray(u, dtype=complex)}
        meta = {"func": "MCfieldOnWave", "sigt": sigt, "albedo": albedo, "is_ff_l": bool(is_ff_l),
                "is_ff_v": bool(is_ff_v), "max_itr": max_itr, "lambda": lam, "cbs": bool(cbs), "smp_flg": smp_flg,
                "sct_type": sct_type, "has_ampfunc0": True, "has_lmean0": True}
        self._put_amp(arrays, meta, "ampfunc", ampfunc)
        self._put_amp(arrays, meta, "ampfunc0", ampfunc0)
        self.save(name, "onwave", meta, arrays)

    @staticmethod
    def _put_amp(arrays, meta, key, amp):
        if isinstance(amp, dict):
            meta[key] = "table"
            arrays[key + "_evalAmp"] = np.asarray(amp["evalAmp"]).reshape(-1).astype(complex)
            arrays[key + "_sampleIcdf"] = np.asarray(amp["sampleIcdf"], float).reshape(-1)
        else:
            meta[key] = float(amp)

    # -- tabulated tables -----------------------------------------------------
    def table(self, name, theta, f):
        it, _, _ = self.interp(0)
        st = it.call("tabulatedAmplitudeScatter", [M(np.asarray(theta, float).reshape(1, -1)),
                                                   M(np.asarray(f).reshape(1, -1))], 1)[0]
        py = struct_to_py(st)
        amp = py["ampfunc"]
        arrays = {"theta": np.asarray(theta, float).reshape(-1), "f": np.asarray(f).reshape(-1).astype(complex)}
        for k in ("cs", "samplePdf", "sampleCdf", "sampleIcdf", "evalPdf", "evalAmp"):
            arrays["out_" + k] = np.asarray(amp[k])
        meta = {"D": float(np.asarray(py["D"]).reshape(-1)[0]), "albedo": float(np.asarray(py["albedo"]).reshape(-1)[0])}
        self.save(name, "table", meta, arrays)
        return {"evalAmp": amp["evalAmp"], "sampleIcdf": amp["sampleIcdf"]}

    # -- scmc.m -----------------------------------------------------------------
    def scmc_case(self, name, seed, target, views, lights, scatter, iterations, opts):
        it, ut, nt = self.interp(seed)
        ta = it.call("boxArea", [M(float(x)) if np.isscalar(x) else M(np.asarray(x, float).reshape(1, -1))
                                 for x in target], 1)[0]
        vs = it.call(views[0], [M(np.asarray(a, float)) for a in views[1]], 1)[0]
        ls = it.call(lights[0], [M(np.asarray(a, float)) for a in lights[1]], 1)[0]
        sc = it.call(scatter[0], [M(float(a)) for a in scatter[1]], 1)[0]
        vargs = []
        for k, val in opts:
            vargs.append(ml.MStr(k))
            vargs.append(M(val) if isinstance(val, bool) else M(float(val)))
        err = None
        res = {}
        try:
            out = it.call("scmc", [ta, vs, ls, sc, M(float(iterations))] + vargs, 1)[0]
            for k in ("C", "Csingle", "field"):
                if k in out:
                    res["out_" + k] = np.asarray(out[k], dtype=complex)
        except ml.MatlabError as e:
            err = str(e)
        arrays = {"utape": ut[:it.ui], "ntape": nt[:it.ni]}
        arrays.update(res)
        meta = {"target": [np.asarray(x, float).tolist() for x in target], "views": [views[0], [np.asarray(a, float).tolist() for a in views[1]]],
                "lights": [lights[0], [np.asarray(a, float).tolist() for a in lights[1]]],
                "scatter": [scatter[0], list(scatter[1])], "iterations": iterations,
                "opts": [[k, v] for k, v in opts], "error": err}
        self.save(name, "scmc", meta, arrays)

    # -- MCfieldFourierQuad ------------------------------------------------------
    def fq_case(self, name, seed, *, sigt, albedo, box_min, box_max, l, v_max, v_stp, max_itr, lam, cbs,
                smp_flg, lmean0, vsign):
        it, ut, nt = self.interp(seed)
        args = [M(float(sigt)), M(float(albedo)), M(np.reshape(box_min, (-1, 1)).astype(float)),
                M(np.reshape(box_max, (-1, 1)).astype(float)), M(np.asarray(l, float)), M(float(v_max)),
                M(float(v_stp)), M(float(max_itr)), M(float(lam)), M(bool(cbs)), M(float(smp_flg)),
                M(np.zeros((0, 0))) if lmean0 is None else M(np.reshape(lmean0, (-1, 1)).astype(float)),
                M(float(vsign))]
        err = None
        arrays = {}
        try:
            u = it.call("MCfieldFourierQuad", args, 1)[0]
            arrays["u"] = np.asarray(u, dtype=complex)
        except ml.MatlabError as e:
            err = str(e)
        arrays.update({"utape": ut[:it.ui], "ntape": nt[:it.ni], "box_min": np.asarray(box_min, float),
                       "box_max": np.asarray(box_max, float), "l": np.asarray(l, float)})
        if lmean0 is not None:
            arrays["lmean0"] = np.asarray(lmean0, float)
        meta = {"sigt": sigt, "albedo": albedo, "v_max": v_max, "v_stp": v_stp, "max_itr": max_itr, "lambda": lam,
                "cbs": bool(cbs), "smp_flg": smp_flg, "vsign": vsign, "has_lmean0": lmean0 is not None,
                "error": err}
        self.save(name, "fourier_quad", meta, arrays)

    def fq_onwave_case(self, name, seed, *, sigt, albedo, box_min, box_max, l, v_max, v_stp, max_itr, lam, cbs,
                       smp_flg, lmean0, Wl, vsign):
        """MCfieldFourierQuadOnWave(..., lmean0, Wl, vsign): Wl as an Nl x 1 column, as its test passes it."""
        it, ut, nt = self.interp(seed)
        args = [M(float(sigt)), M(float(albedo)), M(np.reshape(box_min, (-1, 1)).astype(float)),
                M(np.reshape(box_max, (-1, 1)).astype(float)), M(np.asarray(l, float)), M(float(v_max)),
                M(float(v_stp)), M(float(max_itr)), M(float(lam)), M(bool(cbs)), M(float(smp_flg)),
                M(np.zeros((0, 0))) if lmean0 is None else M(np.reshape(lmean0, (-1, 1)).astype(float)),
                M(np.asarray(Wl, complex).reshape(-1, 1)), M(float(vsign))]
        u = it.call("MCfieldFourierQuadOnWave", args, 1)[0]
        arrays = {"u": np.asarray(u, dtype=complex), "utape": ut[:it.ui], "ntape": nt[:it.ni],
                  "box_min": np.asarray(box_min, float), "box_max": np.asarray(box_max, float),
                  "l": np.asarray(l, float), "Wl": np.asarray(Wl, complex).reshape(-1)}
        if lmean0 is not None:
            arrays["lmean0"] = np.asarray(lmean0, float)
        meta = {"sigt": sigt, "albedo": albedo, "v_max": v_max, "v_stp": v_stp, "max_itr": max_itr, "lambda": lam,
                "cbs": bool(cbs), "smp_flg": smp_flg, "vsign": vsign, "has_lmean0": lmean0 is not None}
        self.save(name, "fq_onwave", meta, arrays)

    # -- refocus ---------------------------------------------------------------
    def refocus_case(self, name, *, u, v, l, box_min, box_max, box_stp, lam):
        it, _, _ = self.interp(0)
        rU = it.call("refocus", [M(np.asarray(u, complex).reshape(-1, 1)), M(np.asarray(v, float)),
                                 M(np.asarray(l, float).reshape(-1, 1)), M(np.reshape(box_min, (-1, 1)).astype(float)),
                                 M(np.reshape(box_max, (-1, 1)).astype(float)),
                                 M(np.reshape(box_stp, (-1, 1)).astype(float)), M(float(lam))], 1)[0]
        arrays = {"u": np.asarray(u, complex).reshape(-1), "v": np.asarray(v, float), "l": np.asarray(l, float),
                  "box_min": np.asarray(box_min, float), "box_max": np.asarray(box_max, float),
                  "box_stp": np.asarray(box_stp, float), "rU": np.asarray(rU, dtype=complex)}
        self.save(name, "refocus", {"lambda": lam}, arrays)

    # -- MCCovHetro / MCsampleHetro ----------------------------------------------
    def hetero_case(self, name, func, seed, *, sigt, albedo, box_min, box_max, box_bin, l, v, is_ff_l, is_ff_v,
                    max_itr, lam, cbs, smp_flg, sct_type, ampfunc, ampfunc0=None, extra=None):
        it, ut, nt = self.interp(seed)
        sg = np.asarray(sigt, float)
        args = [M(sg), M(np.asarray(albedo, float)), M(np.reshape(box_min, (-1, 1)).astype(float)),
                M(np.reshape(box_max, (-1, 1)).astype(float)), M(np.reshape(box_bin, (-1, 1)).astype(float)),
                M(np.asarray(l, float)), M(np.asarray(v, float)), M(bool(is_ff_l)), M(bool(is_ff_v)),
                M(float(max_itr)), M(float(lam)), M(bool(cbs)), M(float(smp_flg)), M(float(sct_type)), to_m(ampfunc)]
        if ampfunc0 is not None or extra is not None:
            args.append(to_m(ampfunc0) if ampfunc0 is not None else M(np.zeros((0, 0))))
        if extra is not None:
            args.append(M(np.reshape(extra, (-1, 1)).astype(float)) if np.size(extra) > 1 else M(float(extra)))
        nout = 3 if func == "MCCovHetro" else 1
        outs = it.call(func, args, nout)
        dim = np.size(box_min)
        lm = np.asarray(l, float)
        if lm.shape[0] == 1:
            lm = np.vstack([np.sin(lm), np.cos(lm)])
        if func == "MCCovHetro":
            unmeanl = lm.mean(axis=1)
        else:
            unmeanl = np.asarray(extra, float).reshape(-1) if (extra is not None and np.size(extra) == dim) \
                else lm.mean(axis=1)
        meanl = unmeanl / np.linalg.norm(unmeanl)
        nb = it.call("null", [M(meanl.reshape(1, -1))], 1)[0]
        arrays = {"utape": ut[:it.ui], "ntape": nt[:it.ni], "sigt": sg, "albedo": np.asarray(albedo, float),
                  "box_min": np.asarray(box_min, float), "box_max": np.asarray(box_max, float),
                  "box_bin": np.asarray(box_bin, float), "l": np.asarray(l, float), "v": np.asarray(v, float),
                  "null_basis": np.asarray(nb, float)}
        meta = {"func": func, "is_ff_l": bool(is_ff_l), "is_ff_v": bool(is_ff_v), "max_itr": max_itr,
                "lambda": lam, "cbs": bool(cbs), "smp_flg": smp_flg, "sct_type": sct_type,
                "has_ampfunc0": ampfunc0 is not None, "extra": None if extra is None else np.asarray(extra, float).tolist()}
        self._put_amp(arrays, meta, "ampfunc", ampfunc)
        if ampfunc0 is not None:
            self._put_amp(arrays, meta, "ampfunc0", ampfunc0)
        if func == "MCCovHetro":
            arrays["Ms"] = np.asarray(outs[0], dtype=complex)
            arrays["Mm"] = np.asarray(outs[1], dtype=complex)
            arrays["mean1"] = np.asarray(outs[2], dtype=complex)
        else:
            arrays["u"] = np.asarray(outs[0], dtype=complex)
        self.save(name, "hetero", meta, arrays)

    def error_case(self, name, func, args_py, expect_contains=None):
        it, _, _ = self.interp(0)
        try:
            it.call(func, [to_m(a) for a in args_py], 1)
            msg = None
        except ml.MatlabError as e:
            msg = str(e)
        assert msg is not None, name
        self.save(name, "error", {"func": func, "error": msg}, {"dummy": np.zeros(1)})


def refocus_cases(g):
    print("refocus")
    r = np.random.default_rng(29)
    v3 = cap_dirs(7, 12, -1, 31)
    u3 = r.normal(size=7) + 1j * r.normal(size=7)
    g.refocus_case("refocus_3d", u=u3, v=v3, l=[0.0, 0.1, 1.0], box_min=[-3, -2, 0], box_max=[3, 2, 1.5],
                   box_stp=[0.5, 0.4, 0.3], lam=1.0)
    v2 = np.vstack([np.sin([3.0, 3.1, 3.3]), np.cos([3.0, 3.1, 3.3])])
    g.refocus_case("refocus_2d", u=r.normal(size=3) + 1j * r.normal(size=3), v=v2, l=[0.05, 1.0],
                   box_min=[-5, 0], box_max=[5, 4], box_stp=[0.25, 0.5], lam=0.8)


def fq_onwave_cases(g):
    print("MCfieldFourierQuadOnWave")
    wr = np.random.default_rng(19)
    Lq = cap_dirs(3, 6, +1, 23)
    W = wr.random(3) * np.exp(2j * np.pi * wr.random(3))
    g.fq_onwave_case("fqow_wide_box_cbs_exp", 311, sigt=0.1, albedo=0.9, box_min=[-60, -60, 0], box_max=[60, 60, 20],
                     l=Lq, v_max=0.2, v_stp=0.01, max_itr=20, lam=1.0, cbs=1, smp_flg=2, lmean0=None, Wl=W, vsign=-1)
    g.fq_onwave_case("fqow_narrow_box_nocbs_unif", 312, sigt=0.15, albedo=0.8, box_min=[-10, -10, 0],
                     box_max=[10, 10, 8], l=Lq, v_max=0.2, v_stp=0.01, max_itr=20, lam=1.0, cbs=0, smp_flg=1,
                     lmean0=[0.0, 0.1, 1.0], Wl=W, vsign=1)
    # even grid length: the parity fix (MCfieldFourierQuadOnWave.m:97-99) makes the padding integral
    g.fq_onwave_case("fqow_even_grid_cbs", 313, sigt=0.1, albedo=0.9, box_min=[-10, -10, 0], box_max=[10, 10, 8],
                     l=Lq[:, :2], v_max=0.195, v_stp=0.01, max_itr=10, lam=1.0, cbs=1, smp_flg=2, lmean0=None,
                     Wl=W[:2], vsign=-1)


def onwave_cases(g, common, box3, box2, L3, V3r, NFv, tab3d):
    print("MCfieldOnWave")
    wr = np.random.default_rng(17)
    W3 = wr.random(3) * np.exp(2j * np.pi * wr.random(3))
    g.onwave_case("onwave_3d_hg_ff_refl_cbs_exp", 120, **common, **box3, l=L3, v=V3r, is_ff_l=1, is_ff_v=1, cbs=1,
                  smp_flg=2, sct_type=3, ampfunc=0.7, ampfunc0=0.4, lmean0=[0.0, 0.1, 1.0], Wl=W3)
    g.onwave_case("onwave_3d_tab_nfv_nocbs_unif", 121, **common, **box3, l=L3, v=NFv, is_ff_l=1, is_ff_v=0, cbs=0,
                  smp_flg=1, sct_type=2, ampfunc=tab3d, ampfunc0=tab3d, lmean0=[0.0, 0.0, 1.0], Wl=W3)
    # isotropic: the reference's single-scattering line is consistent only for one light
    g.onwave_case("onwave_3d_iso_one_light_cbs", 122, **common, **box3, l=L3[:, :1], v=V3r, is_ff_l=1, is_ff_v=1,
                  cbs=1, smp_flg=2, sct_type=1, ampfunc=0, ampfunc0=0, lmean0=[0.0, 0.0, 1.0], Wl=W3[:1])
    g.onwave_case("onwave_2d_hg_cbs", 123, **common, **box2, l=np.vstack([np.sin([0.0, 0.05]), np.cos([0.0, 0.05])]),
                  v=np.vstack([np.sin([3.1, 3.2, 3.0]), np.cos([3.1, 3.2, 3.0])]), is_ff_l=1, is_ff_v=1, cbs=1,
                  smp_flg=2, sct_type=3, ampfunc=0.5, ampfunc0=0.5, lmean0=[0.0, 1.0], Wl=W3[:2])


def main(ref):
    g = Gen(ref)
    print("tables")
    import scipy.io as sio
    mat = sio.loadmat(os.path.join(ref, "examples", "buildFarFieldCovMatrix", "scatteringAmplitude.mat"))
    tab2d = g.table("table_2d_scatteringAmplitude", mat["theta"], mat["farField"])
    th3 = np.linspace(0, 1, 1001) * np.pi
    th3[-1] = np.pi
    it, _, _ = g.interp(0)
    hg3 = np.sqrt(np.asarray(it.call("evaluateHG", [M(th3.reshape(1, -1)), M(0.7), M(0.0), M(3.0)], 1)[0]))
    tab3d = g.table("table_3d_hg07", th3, hg3)

    box3 = dict(box_min=[-20, -20, 0], box_max=[20, 20, 15])
    box2 = dict(box_min=[-20, 0], box_max=[20, 15])
    L3 = cap_dirs(3, 10, +1, 11)
    V3r = cap_dirs(4, 10, -1, 12)   # reflection
    V3t = cap_dirs(4, 10, +1, 13)   # transmission
    NFv = np.array([[-5.0, 0.0, 6.0, 2.0], [1.0, -3.0, 2.0, 0.5], [-30.0, -30.0, -28.0, 40.0]])
    NFl = np.array([[0.0, 4.0, -6.0], [2.0, -1.0, 3.0], [-35.0, -40.0, -30.0]])

    print("MCfield / MCcov")
    common = dict(sigt=0.2, albedo=0.9, lam=1.0, max_itr=40)
    for func in ("MCfield", "MCcov"):
        tag = "field" if func == "MCfield" else "cov"
        g.mc_case(f"{tag}_3d_iso_ff_refl_cbs_exp", func, 101, **common, **box3, l=L3, v=V3r, is_ff_l=1, is_ff_v=1,
                  cbs=1, smp_flg=2, sct_type=1, ampfunc=0)
        g.mc_case(f"{tag}_3d_hg_ff_trans_nocbs_unif", func, 102, **common, **box3, l=L3, v=V3t, is_ff_l=1, is_ff_v=1,
                  cbs=0, smp_flg=1, sct_type=3, ampfunc=0.8)
        g.mc_case(f"{tag}_3d_hg_nfv_cbs_exp_g0", func, 103, **common, **box3, l=L3, v=NFv, is_ff_l=1, is_ff_v=0,
                  cbs=1, smp_flg=2, sct_type=3, ampfunc=0.6, ampfunc0=0.3)
        g.mc_case(f"{tag}_3d_tab_nfl_nfv_cbs_exp", func, 104, **common, **box3, l=NFl, v=NFv, is_ff_l=0, is_ff_v=0,
                  cbs=1, smp_flg=2, sct_type=2, ampfunc=tab3d)
        g.mc_case(f"{tag}_3d_tab_ff_refl_cbs_unif_t0", func, 105, **common, **box3, l=L3, v=V3r, is_ff_l=1, is_ff_v=1,
                  cbs=1, smp_flg=1, sct_type=2, ampfunc=tab3d, ampfunc0=tab3d)
        g.mc_case(f"{tag}_3d_iso_lowalbedo_roulette", func, 106, sigt=0.3, albedo=0.5, lam=0.7, max_itr=25, **box3,
                  l=L3, v=V3r, is_ff_l=1, is_ff_v=1, cbs=1, smp_flg=2, sct_type=1, ampfunc=0)
        g.mc_case(f"{tag}_2d_iso_angles_cbs_exp", func, 107, **common, **box2,
                  l=np.deg2rad([[0.0, 3.0, -4.0]]), v=np.deg2rad([[180.0, 170.0, 185.0, 200.0]]),
                  is_ff_l=1, is_ff_v=1, cbs=1, smp_flg=2, sct_type=1, ampfunc=0)
        g.mc_case(f"{tag}_2d_hg_vectors_nocbs_unif", func, 108, **common, **box2,
                  l=norm_cols([[0.1, -0.2], [1.0, 1.0]]), v=norm_cols([[0.0, 0.3, -0.1], [1.0, 1.0, 1.0]]),
                  is_ff_l=1, is_ff_v=1, cbs=0, smp_flg=1, sct_type=3, ampfunc=-0.4)
        g.mc_case(f"{tag}_2d_tab_measured_cbs_exp", func, 109, **common, **box2,
                  l=np.deg2rad([[0.0, 20.0]]), v=np.deg2rad([[0.0, 90.0, 180.0, 270.0]]),
                  is_ff_l=1, is_ff_v=1, cbs=1, smp_flg=2, sct_type=2, ampfunc=tab2d)
    g.mc_case("field_3d_hg_lmean0", "MCfield", 110, **common, **box3, l=L3, v=V3r, is_ff_l=1, is_ff_v=1,
              cbs=1, smp_flg=2, sct_type=3, ampfunc=0.5, ampfunc0=0.2, lmean0=[0.1, 0.0, 1.0])

    print("MCfieldFourierQuad")
    Lq = cap_dirs(2, 8, +1, 21)
    g.fq_case("fq_wide_box_cbs_exp", 301, sigt=0.1, albedo=0.9, box_min=[-60, -60, 0], box_max=[60, 60, 20], l=Lq,
              v_max=0.2, v_stp=0.01, max_itr=25, lam=1.0, cbs=1, smp_flg=2, lmean0=None, vsign=-1)
    g.fq_case("fq_narrow_box_nocbs_unif", 302, sigt=0.15, albedo=0.8, box_min=[-10, -10, 0], box_max=[10, 10, 8],
              l=Lq, v_max=0.2, v_stp=0.01, max_itr=25, lam=1.0, cbs=0, smp_flg=1, lmean0=[0.0, 0.1, 1.0], vsign=1)
    g.fq_case("fq_narrow_box_cbs_refl", 303, sigt=0.12, albedo=1.0, box_min=[-8, -8, 0], box_max=[8, 8, 10],
              l=cap_dirs(3, 5, +1, 22), v_max=0.3, v_stp=0.02, max_itr=20, lam=0.8, cbs=1, smp_flg=2, lmean0=None,
              vsign=-1)
    g.fq_case("fq_even_grid_errors", 304, sigt=0.1, albedo=0.9, box_min=[-10, -10, 0], box_max=[10, 10, 8], l=Lq,
              v_max=0.195, v_stp=0.01, max_itr=5, lam=1.0, cbs=1, smp_flg=2, lmean0=None, vsign=-1)

    fq_onwave_cases(g)
    refocus_cases(g)

    print("hetero")
    g2 = np.random.default_rng(7)
    sig2 = np.array([[1 / 30, 0, 1 / 60], [0, 1 / 120, 1 / 30]]).T  # testHetroCov.m's grid, 3 x 2
    L2 = np.pi - np.deg2rad([[0.0, 4.0, 12.0]])
    V2 = np.deg2rad([[-30.0, 10.0, 170.0, 200.0]])
    hb2 = dict(box_min=[-60, -60], box_max=[60, 60], box_bin=[40, 60])
    sig3 = g2.lognormal(np.log(0.15), 0.5, size=(2, 2, 3))
    hb3 = dict(box_min=[-20, -20, 0], box_max=[20, 20, 15], box_bin=[20, 20, 5])
    for func in ("MCCovHetro", "MCsampleHetro"):
        tag = "hcov" if func == "MCCovHetro" else "hfield"
        g.hetero_case(f"{tag}_2d_iso_voxelpick_cbs", func, 401, sigt=sig2, albedo=1.0, **hb2, l=L2, v=V2,
                      is_ff_l=1, is_ff_v=1, max_itr=30, lam=1.0, cbs=1, smp_flg=1, sct_type=1, ampfunc=0)
        g.hetero_case(f"{tag}_2d_hg_plane_nocbs", func, 402, sigt=sig2, albedo=0.9, **hb2, l=L2, v=V2,
                      is_ff_l=1, is_ff_v=1, max_itr=30, lam=1.0, cbs=0, smp_flg=2, sct_type=3, ampfunc=0.5)
        g.hetero_case(f"{tag}_3d_hg_plane_cbs_albgrid", func, 403, sigt=sig3,
                      albedo=g2.uniform(0.7, 1.0, size=(2, 2, 3)), **hb3, l=L3, v=V3r, is_ff_l=1, is_ff_v=1,
                      max_itr=25, lam=1.0, cbs=1, smp_flg=2, sct_type=3, ampfunc=0.7)
        # tabulated scatter only for MCsampleHetro: MCCovHetro.m:271-272 reads
        # ampfunc.pdf, a field tabulatedAmplitudeScatter does not build
        st, amp = (2, tab3d) if func == "MCsampleHetro" else (3, 0.3)
        g.hetero_case(f"{tag}_3d_voxelpick_nfv", func, 404, sigt=sig3, albedo=0.95, **hb3, l=L3, v=NFv,
                      is_ff_l=1, is_ff_v=0, max_itr=20, lam=1.0, cbs=1, smp_flg=1, sct_type=st, ampfunc=amp)
    g.hetero_case("hcov_3d_iso_plane_lrad_g0", "MCCovHetro", 405, sigt=sig3, albedo=1.0, **hb3, l=L3, v=V3t,
                  is_ff_l=1, is_ff_v=1, max_itr=25, lam=0.9, cbs=0, smp_flg=2, sct_type=3, ampfunc=0.4,
                  ampfunc0=0.2, extra=30.0)
    g.hetero_case("hfield_3d_hg_plane_lmean0", "MCsampleHetro", 406, sigt=sig3, albedo=1.0, **hb3, l=L3, v=V3r,
                  is_ff_l=1, is_ff_v=1, max_itr=25, lam=1.0, cbs=1, smp_flg=2, sct_type=3, ampfunc=0.6,
                  ampfunc0=0.3, extra=[0.1, 0.0, 1.0])

    print("scmc.m")
    tgt3 = [1.0, 5.0, [0, 15], [-20, 20], [-20, 20]]
    g.scmc_case("scmc_cov_default_hg", 201, tgt3, ("farFieldSource", [V3r]), ("farFieldSource", [L3]),
                ("HGScatter", [0.7]), 8, [])
    g.scmc_case("scmc_cov_single_field_nocbs", 202, tgt3, ("farFieldSource", [V3t]), ("farFieldSource", [L3]),
                ("isotropicScatter", [0.9]), 8,
                [("CBS", False), ("singleScattering", True), ("renderField", True), ("uniformFirstScatter", True)])
    g.scmc_case("scmc_field_only_g0", 203, tgt3, ("farFieldSource", [V3r]), ("farFieldSource", [L3]),
                ("HGScatter", [0.6, 0.3, 0.95]), 10, [("renderCov", False), ("renderField", True)])
    g.scmc_case("scmc_parfor_cov_field", 204, tgt3, ("farFieldSource", [V3r]), ("farFieldSource", [L3]),
                ("HGScatter", [0.5]), 5, [("parforIters", 3), ("renderField", True)])
    g.scmc_case("scmc_angles_2d", 205, [1.0, 5.0, [0, 15], [-20, 20]],
                ("farFieldSource", [np.deg2rad([180.0, 175.0]), [0.0]]), ("farFieldSource", [np.deg2rad([0.0, 2.0]), [0.0]]),
                ("isotropicScatter", []), 6, [])
    g.scmc_case("scmc_nearfield_views", 206, tgt3, ("nearFieldSource", [NFv]), ("farFieldSource", [L3]),
                ("HGScatter", [0.4]), 6, [("renderField", True)])
    g.scmc_case("scmc_err_option", 207, tgt3, ("farFieldSource", [V3r]), ("farFieldSource", [L3]),
                ("HGScatter", [0.4]), 6, [("mean", False)])
    g.scmc_case("scmc_err_rng_parfor", 208, tgt3, ("farFieldSource", [V3r]), ("farFieldSource", [L3]),
                ("HGScatter", [0.4]), 6, [("rng", 5), ("parforIters", 2)])
    g.scmc_case("scmc_err_cbs_type", 209, tgt3, ("farFieldSource", [V3r]), ("farFieldSource", [L3]),
                ("HGScatter", [0.4]), 6, [("CBS", 1)])

    print("errors")
    g.error_case("err_field_box", "MCfield", [0.1, 1.0, np.zeros((3, 2)), np.ones((3, 2)), L3, V3r, True, True,
                                             2.0, 1.0, True, 2.0, 1.0, 0.0])
    g.error_case("err_field_light", "MCfield", [0.1, 1.0, np.zeros((3, 1)), np.ones((3, 1)), L3[:2], V3r, True, True,
                                               2.0, 1.0, True, 2.0, 1.0, 0.0])
    onwave_cases(g, common, box3, box2, L3, V3r, NFv, tab3d)

    g.error_case("err_cov_view", "MCcov", [0.1, 1.0, np.zeros((3, 1)), np.ones((3, 1)), L3, V3r[:1], True, True,
                                          2.0, 1.0, True, 2.0, 1.0, 0.0])
    g.error_case("err_field_nargs", "MCfield", [0.1, 1.0, np.zeros((3, 1)), np.ones((3, 1)), L3, V3r, True, True,
                                               2.0, 1.0, True, 2.0, 1.0])

    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(g.index, f, indent=1)
    print(f"{len(g.index)} fixtures")


def only_onwave(ref):
    """Add the MCfieldOnWave fixtures to an existing index (the other fixtures
    are left as they are)."""
    g = Gen(ref)
    with open(os.path.join(HERE, "index.json")) as f:
        g.index = [e for e in json.load(f) if e["kind"] != "onwave"]
    z = np.load(os.path.join(HERE, "table_3d_hg07.npz"))
    tab3d = {"evalAmp": z["out_evalAmp"], "sampleIcdf": z["out_sampleIcdf"]}
    onwave_cases(g, dict(sigt=0.2, albedo=0.9, lam=1.0, max_itr=40), dict(box_min=[-20, -20, 0], box_max=[20, 20, 15]),
                 dict(box_min=[-20, 0], box_max=[20, 15]), cap_dirs(3, 10, +1, 11), cap_dirs(4, 10, -1, 12),
                 np.array([[-5.0, 0.0, 6.0, 2.0], [1.0, -3.0, 2.0, 0.5], [-30.0, -30.0, -28.0, 40.0]]), tab3d)
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(g.index, f, indent=1)
    print(f"{len(g.index)} fixtures")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref = args[0] if args else os.environ.get("SCMC_REFERENCE_TREE")
    if not ref:
        sys.exit("usage: make_golden.py <path of the mcspeckle tree> [--only-...] "
                 "(or set SCMC_REFERENCE_TREE)")
    if "--only-onwave" in sys.argv:
        only_onwave(ref)
    elif "--only-refocus" in sys.argv:
        g = Gen(ref)
        with open(os.path.join(HERE, "index.json")) as f:
            g.index = [e for e in json.load(f) if e["kind"] != "refocus"]
        refocus_cases(g)
        with open(os.path.join(HERE, "index.json"), "w") as f:
            json.dump(g.index, f, indent=1)
        print(f"{len(g.index)} fixtures")
    elif "--only-fq-onwave" in sys.argv:
        g = Gen(ref)
        with open(os.path.join(HERE, "index.json")) as f:
            g.index = [e for e in json.load(f) if e["kind"] != "fq_onwave"]
        fq_onwave_cases(g)
        with open(os.path.join(HERE, "index.json"), "w") as f:
            json.dump(g.index, f, indent=1)
        print(f"{len(g.index)} fixtures")
    else:
        main(ref)
