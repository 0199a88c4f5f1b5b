"""The CPU oracle and the host mirror against the reference itself.

Fixtures in tests/golden/ hold outputs of the reference's own .m files
(MCfield.m, MCcov.m, scmc.m, tabulatedAmplitudeScatter.m, ...) executed by
tests/golden/mlite.py with recorded random tapes (tests/golden/make_golden.py).
Fed the same tapes, the oracle must reproduce them to rounding, and must
consume exactly as many draws as the reference did.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mcspeckle_b200 import interface as I
from mcspeckle_b200 import mc as MC
from mcspeckle_b200 import scmc_api as S

RTOL = 1e-9

with open(os.path.join(GOLDEN, "index.json")) as f:
    INDEX = json.load(f)


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in z.files if k != "meta"}


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def amp(meta, arr, key):
    if meta[key] == "table":
        return {"evalAmp": arr[key + "_evalAmp"], "sampleIcdf": arr[key + "_sampleIcdf"]}
    return meta[key]


def mc_case_args(meta, arr):
    args = [meta["sigt"], meta["albedo"], arr["box_min"], arr["box_max"], arr["l"], arr["v"], meta["is_ff_l"],
            meta["is_ff_v"], meta["max_itr"], meta["lambda"], meta["cbs"], meta["smp_flg"], meta["sct_type"],
            amp(meta, arr, "ampfunc")]
    if meta["has_ampfunc0"]:
        args.append(amp(meta, arr, "ampfunc0"))
    if meta["has_lmean0"]:
        if not meta["has_ampfunc0"]:
            args.append(MC._MISSING)
        args.append(arr["lmean0"])
    return args


MC_CASES = [e["name"] for e in INDEX if e["kind"] in ("MCfield", "MCcov")]
TABLE_CASES = [e["name"] for e in INDEX if e["kind"] == "table"]
SCMC_CASES = [e["name"] for e in INDEX if e["kind"] == "scmc"]


def test_fixture_inventory():
    kinds = {e["kind"] for e in INDEX}
    assert {"MCfield", "MCcov", "table", "scmc", "error"} <= kinds
    assert len(MC_CASES) >= 18


@pytest.mark.parametrize("name", MC_CASES)
def test_oracle_matches_reference(oracle_lib, name):
    O = oracle_lib
    meta, arr = load(name)
    h = MC.mc_args(*mc_case_args(meta, arr), seed=0, precision="fp64")
    rng = O.Rng.tape(arr["utape"], arr["ntape"])
    if meta["func"] == "MCfield":
        u = O.field(h, rng)
        assert u.shape == arr["u"].shape
        assert relerr(u, arr["u"]) < RTOL
    else:
        Ms, Mm = O.cov(h, rng)
        assert Ms.shape == arr["Ms"].shape
        assert relerr(Ms, arr["Ms"]) < RTOL
        assert relerr(Mm, arr["Mm"]) < RTOL
    # the same number of rand / randn draws as the reference consumed
    assert rng.spec.used_u == arr["utape"].size
    assert rng.spec.used_n == arr["ntape"].size


@pytest.mark.parametrize("name", TABLE_CASES)
def test_tabulated_table_matches_reference(name):
    meta, arr = load(name)
    s = I.tabulatedAmplitudeScatter(arr["theta"], arr["f"])
    assert s["D"] == meta["D"]
    a = s["ampfunc"]
    for k in ("cs", "samplePdf", "sampleCdf", "sampleIcdf", "evalPdf", "evalAmp"):
        ref = np.asarray(arr["out_" + k]).reshape(-1)
        got = np.asarray(a[k]).reshape(-1)
        assert got.shape == ref.shape, k
        assert relerr(got, ref) < 1e-12, k


class TapeKernels:
    """MCcov / MCfield on the oracle with a continuing pair of tapes, the way
    successive calls share MATLAB's global stream."""

    def __init__(self, O, ut, nt):
        self.O, self.ut, self.nt = O, ut, nt
        self.pu = self.pn = 0

    def _run(self, fn, args, n_total):
        h = MC.mc_args(*args, seed=0, norm_itr=n_total, precision="fp64")
        r = self.O.Rng.tape(self.ut[self.pu:], self.nt[self.pn:])
        out = fn(h, r)
        self.pu += r.spec.used_u
        self.pn += r.spec.used_n
        return out

    def MCcov(self, *args, seed, n_total):
        return self._run(self.O.cov, args, n_total)

    def MCfield(self, *args, seed, n_total):
        return self._run(self.O.field, args, n_total)


def make_struct(kind, args):
    return getattr(I, kind)(*[np.asarray(a) if isinstance(a, list) else a for a in args])


@pytest.mark.parametrize("name", SCMC_CASES)
def test_scmc_dispatch_matches_reference(oracle_lib, name):
    meta, arr = load(name)
    t = meta["target"]
    ta = I.boxArea(*[x[0] if isinstance(x, list) and len(x) == 1 else np.asarray(x) for x in t])
    views = make_struct(*meta["views"])
    lights = make_struct(*meta["lights"])
    sc = make_struct(*meta["scatter"])
    opts = []
    for k, v in meta["opts"]:
        opts += [k, v]
    if meta["error"] is not None:
        with pytest.raises(S.ScmcInputError) as ei:
            S.build_config(ta, views, lights, sc, meta["iterations"], *opts)
        assert str(ei.value) == meta["error"]
        return
    cfg = S.build_config(ta, views, lights, sc, meta["iterations"], *opts)
    ker = TapeKernels(oracle_lib, arr["utape"], arr["ntape"])
    res = S.run_config(cfg, ker)
    for k in ("C", "Csingle", "field"):
        if "out_" + k in arr:
            assert k in res, k
            assert relerr(res[k], arr["out_" + k]) < RTOL, k
        else:
            assert k not in res, k
    assert ker.pu == arr["utape"].size and ker.pn == arr["ntape"].size


def test_argument_errors_match_reference():
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden as G
    L3 = G.cap_dirs(3, 10, +1, 11)
    V3r = G.cap_dirs(4, 10, -1, 12)
    cases = {
        "err_field_box": (MC.MCfield, [0.1, 1.0, np.zeros((3, 2)), np.ones((3, 2)), L3, V3r, True, True,
                                       2.0, 1.0, True, 2.0, 1.0, 0.0]),
        "err_field_light": (MC.MCfield, [0.1, 1.0, np.zeros((3, 1)), np.ones((3, 1)), L3[:2], V3r, True, True,
                                         2.0, 1.0, True, 2.0, 1.0, 0.0]),
        "err_cov_view": (MC.MCcov, [0.1, 1.0, np.zeros((3, 1)), np.ones((3, 1)), L3, V3r[:1], True, True,
                                    2.0, 1.0, True, 2.0, 1.0, 0.0]),
    }
    for name, (fn, args) in cases.items():
        meta, _ = load(name)
        with pytest.raises(MC.MatlabStyleError) as ei:
            fn(*args)
        assert str(ei.value) == meta["error"], name
    meta, _ = load("err_field_nargs")
    assert meta["error"] == "Not enough input arguments."
    with pytest.raises(TypeError):
        MC.MCfield(0.1, 1.0, np.zeros((3, 1)), np.ones((3, 1)), L3, V3r, True, True, 2.0, 1.0, True, 2.0, 1.0)


FQ_CASES = [e["name"] for e in INDEX if e["kind"] == "fourier_quad"]


@pytest.mark.parametrize("name", FQ_CASES)
def test_fourier_quad_oracle_matches_reference(oracle_lib, name):
    from mcspeckle_b200 import fourier_quad as FQ
    meta, arr = load(name)
    h = FQ.fq_args(meta["sigt"], meta["albedo"], arr["box_min"], arr["box_max"], arr["l"], meta["v_max"],
                   meta["v_stp"], meta["max_itr"], meta["lambda"], meta["cbs"], meta["smp_flg"],
                   arr["lmean0"] if meta["has_lmean0"] else None, meta["vsign"], seed=0, precision="fp64")
    rng = oracle_lib.Rng.tape(arr["utape"], arr["ntape"])
    u = oracle_lib.field_fourier_quad(h.args, rng, h.nv0)
    if meta["error"] is not None:
        # the reference stops on its half-integer padding (even grid length);
        # the oracle evaluates the extension and must still walk identically
        assert h.nv0 % 2 == 0
        assert np.isfinite(u).all()
    else:
        assert u.shape == arr["u"].shape
        assert relerr(u, arr["u"]) < RTOL
    assert rng.spec.used_u == arr["utape"].size
    assert rng.spec.used_n == arr["ntape"].size


HETERO_CASES = [e["name"] for e in INDEX if e["kind"] == "hetero"]


def hetero_case_args(meta, arr):
    args = [arr["sigt"], arr["albedo"], arr["box_min"], arr["box_max"], arr["box_bin"], arr["l"], arr["v"],
            meta["is_ff_l"], meta["is_ff_v"], meta["max_itr"], meta["lambda"], meta["cbs"], meta["smp_flg"],
            meta["sct_type"], amp(meta, arr, "ampfunc")]
    args.append(amp(meta, arr, "ampfunc0") if meta["has_ampfunc0"] else MC._MISSING)
    args.append(np.asarray(meta["extra"]) if meta["extra"] is not None else MC._MISSING)
    return args


@pytest.mark.parametrize("name", HETERO_CASES)
def test_hetero_oracle_matches_reference(oracle_lib, name):
    from mcspeckle_b200 import hetero as H
    meta, arr = load(name)
    cov = meta["func"] == "MCCovHetro"
    h = H.hetero_args(cov, *hetero_case_args(meta, arr), seed=0, precision="fp64", basis=arr["null_basis"])
    # the null-space axes the reference used (MATLAB's null() run by the
    # interpreter) are the ones this host mirror computes itself
    L = arr["l"] if arr["l"].shape[0] > 1 else np.vstack([np.sin(arr["l"]), np.cos(arr["l"])])
    um = np.asarray(meta["extra"], float).reshape(-1) if (not cov and meta["extra"] is not None) else L.mean(axis=1)
    assert np.allclose(H.null_basis(um / np.linalg.norm(um)), arr["null_basis"])
    rng = oracle_lib.Rng.tape(arr["utape"], arr["ntape"])
    if cov:
        Ms, Mm, m1 = oracle_lib.cov_hetero(h, rng)
        assert relerr(Ms, arr["Ms"]) < RTOL
        assert relerr(Mm, arr["Mm"]) < RTOL
        assert relerr(m1, np.asarray(arr["mean1"]).reshape(m1.shape, order="F")) < RTOL
    else:
        u = oracle_lib.field_hetero(h, rng)
        assert relerr(u, np.asarray(arr["u"]).reshape(u.shape, order="F")) < RTOL
    assert rng.spec.used_u == arr["utape"].size
    assert rng.spec.used_n == arr["ntape"].size


ONWAVE_CASES = [e["name"] for e in INDEX if e["kind"] == "onwave"]


def test_onwave_fixture_inventory():
    assert len(ONWAVE_CASES) >= 4


@pytest.mark.parametrize("name", ONWAVE_CASES)
def test_onwave_oracle_matches_reference(oracle_lib, name):
    """MCfieldOnWave.m (lights combined with complex weights Wl) run by the
    reference interpreter vs the oracle on the same tapes."""
    O = oracle_lib
    meta, arr = load(name)
    h = MC.mc_args(*mc_case_args(meta, arr), seed=0, precision="fp64")
    rng = O.Rng.tape(arr["utape"], arr["ntape"])
    u = O.field_onwave(h, arr["Wl"], rng)
    assert u.shape == arr["u"].shape
    assert relerr(u, arr["u"]) < RTOL
    assert rng.spec.used_u == arr["utape"].size
    assert rng.spec.used_n == arr["ntape"].size


def test_onwave_oracle_equals_field_times_weights(oracle_lib):
    """On the same (Philox) paths the weighted-light field is the full field
    times Wl (HG: the single-scattering amplitude is a full matrix)."""
    O = oracle_lib
    meta, arr = load("onwave_3d_hg_ff_refl_cbs_exp")
    args = mc_case_args(meta, arr)
    args[8] = 60
    h = MC.mc_args(*args, seed=5, precision="fp64")
    u = O.field_onwave(h, arr["Wl"], O.Rng.philox())
    U = O.field(h, O.Rng.philox())
    assert relerr(u, U @ arr["Wl"].reshape(-1, 1)) < 1e-12


FQOW_CASES = [e["name"] for e in INDEX if e["kind"] == "fq_onwave"]


def test_fq_onwave_fixture_inventory():
    assert len(FQOW_CASES) >= 3


@pytest.mark.parametrize("name", FQOW_CASES)
def test_fourier_quad_onwave_oracle_matches_reference(oracle_lib, name):
    """MCfieldFourierQuadOnWave.m (weighted lights, its own phase conventions
    and the pixel-count parity fix) vs the oracle on the same tapes."""
    from mcspeckle_b200 import fourier_quad as FQ
    meta, arr = load(name)
    h = FQ.fq_args(meta["sigt"], meta["albedo"], arr["box_min"], arr["box_max"], arr["l"], meta["v_max"],
                   meta["v_stp"], meta["max_itr"], meta["lambda"], meta["cbs"], meta["smp_flg"],
                   arr["lmean0"] if meta["has_lmean0"] else None, meta["vsign"], seed=0, precision="fp64")
    rng = oracle_lib.Rng.tape(arr["utape"], arr["ntape"])
    u = oracle_lib.field_fourier_quad_onwave(h.args, arr["Wl"], rng, h.nv0, as_written=True)
    assert u.shape == arr["u"].shape
    assert relerr(u, arr["u"]) < RTOL
    assert rng.spec.used_u == arr["utape"].size
    assert rng.spec.used_n == arr["ntape"].size


def test_fourier_quad_onwave_linear_in_weights(oracle_lib):
    """On the same paths the OnWave field is linear in Wl: the sum over lights
    of each light alone (weight 1) times its weight.  Holds for the formula the
    GPU uses (each vertex's own light weight)."""
    from mcspeckle_b200 import fourier_quad as FQ
    meta, arr = load("fqow_wide_box_cbs_exp")
    h = FQ.fq_args(meta["sigt"], meta["albedo"], arr["box_min"], arr["box_max"], arr["l"], meta["v_max"],
                   meta["v_stp"], 15, meta["lambda"], meta["cbs"], meta["smp_flg"], None, -1.0, seed=3,
                   precision="fp64")
    W = arr["Wl"]
    u = oracle_lib.field_fourier_quad_onwave(h.args, W, oracle_lib.Rng.philox(), h.nv0)
    parts = 0
    for j in range(W.size):
        e = np.zeros(W.size, complex)
        e[j] = 1.0
        parts = parts + W[j] * oracle_lib.field_fourier_quad_onwave(h.args, e, oracle_lib.Rng.philox(), h.nv0)
    assert relerr(u, parts) < 1e-10


REFOCUS_CASES = [e["name"] for e in INDEX if e["kind"] == "refocus"]


@pytest.mark.parametrize("name", REFOCUS_CASES)
def test_refocus_oracle_matches_reference(oracle_lib, name):
    """refocus.m run by the reference interpreter (first grid point left at 0
    by its chunk indices) vs the oracle."""
    meta, arr = load(name)
    rU = oracle_lib.refocus(arr["u"], arr["v"], arr["l"], arr["box_min"], arr["box_max"], arr["box_stp"],
                            meta["lambda"], as_written=True)
    assert rU.shape == arr["rU"].shape
    assert relerr(rU, arr["rU"]) < RTOL
    assert arr["rU"].reshape(-1, order="F")[0] == 0


def test_sample_cov_oracle_against_numpy(oracle_lib):
    """samplingFromCovMatrix.m:47-64 with an independent Cholesky."""
    g = np.random.default_rng(1)
    N = 12
    A = g.normal(size=(N, 3 * N)) + 1j * g.normal(size=(N, 3 * N))
    C = A @ A.conj().T / (3 * N)
    Sig = 0.5 * np.block([[C.real, -C.imag], [C.imag, C.real]])
    R = np.linalg.cholesky(Sig).T
    nm = g.normal(size=(4, 2 * N))
    s = nm @ R
    Z = oracle_lib.sample_cov(C, nm)
    assert relerr(Z, (s[:, :N] + 1j * s[:, N:]).T) < 1e-12
