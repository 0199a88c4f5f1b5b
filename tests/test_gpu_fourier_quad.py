"""MCfieldFourierQuad on the GPU against the FP64 oracle (same Philox paths).

The oracle restates MCfieldFourierQuad.m and is pinned to the reference by
the golden fixtures (tests/test_oracle_golden.py); the GPU evaluates the
same centred DFT per vertex instead of gridding + FFT.
"""
import numpy as np
import pytest

from cases import cap_dirs
from mcspeckle_b200 import fourier_quad as FQ

pytestmark = pytest.mark.gpu
SEED = 4242


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


FQ_CASES = {
    # wide box: pixel grid longer than the angular grid (crop of the FFT)
    "wide_cbs_exp": dict(sigt=0.1, albedo=0.9, box_min=[-60, -60, 0], box_max=[60, 60, 20], v_max=0.2, v_stp=0.01,
                         lam=1.0, cbs=1, smp=2, lmean0=None, vsign=-1, n=400),
    # narrow box: angular grid longer than the pixel grid (zero padding)
    "narrow_nocbs_unif": dict(sigt=0.15, albedo=0.8, box_min=[-10, -10, 0], box_max=[10, 10, 8], v_max=0.2,
                              v_stp=0.01, lam=1.0, cbs=0, smp=1, lmean0=[0.0, 0.1, 1.0], vsign=1, n=400),
    # an even grid length (half-integer padding: the extension)
    "even_grid": dict(sigt=0.1, albedo=0.9, box_min=[-10, -10, 0], box_max=[10, 10, 8], v_max=0.195, v_stp=0.01,
                      lam=1.0, cbs=1, smp=2, lmean0=None, vsign=-1, n=300),
    # evanescent corners of the grid (|v| > 1) and reflection
    "wide_angles": dict(sigt=0.12, albedo=1.0, box_min=[-8, -8, 0], box_max=[8, 8, 10], v_max=0.9, v_stp=0.05,
                        lam=0.8, cbs=1, smp=2, lmean0=None, vsign=-1, n=300),
}


def args_for(c, precision, seed=SEED):
    L = cap_dirs(2, 8, +1, 21)
    return FQ.fq_args(c["sigt"], c["albedo"], c["box_min"], c["box_max"], L, c["v_max"], c["v_stp"], c["n"],
                      c["lam"], c["cbs"], c["smp"], c["lmean0"], c["vsign"], seed=seed, precision=precision)


@pytest.mark.parametrize("name", list(FQ_CASES))
def test_fourier_quad_fp64_matches_oracle(gpu, oracle_lib, name):
    h = args_for(FQ_CASES[name], "fp64")
    u = FQ.field_fourier_quad_from_args(h)
    uo = oracle_lib.field_fourier_quad(h.args, oracle_lib.Rng.philox(), h.nv0)
    assert u.shape == uo.shape
    assert rel(u, uo) < 1e-10


@pytest.mark.parametrize("name", list(FQ_CASES))
def test_fourier_quad_mixed_close_to_fp64(gpu, name):
    u64 = FQ.field_fourier_quad_from_args(args_for(FQ_CASES[name], "fp64"))
    umx = FQ.field_fourier_quad_from_args(args_for(FQ_CASES[name], "mixed"))
    assert rel(umx, u64) < 1e-3


def test_fourier_quad_grid_size(gpu):
    import ctypes
    from mcspeckle_b200 import _lib
    n = ctypes.c_int64()
    _lib.check(_lib.lib().scmc_fq_grid_size(255 / 256, 1 / 128, ctypes.byref(n)))
    assert n.value == 256 == FQ.grid_length(255 / 256, 1 / 128)


# Grids of at least 64 angles per axis: MIXED / FP16 run the per-plane sums on
# tcgen05 (one GEMM slice per z plane, plane factor applied on reduction).
TC_CASES = {
    "tc_wide_cbs": dict(sigt=0.1, albedo=0.9, box_min=[-60, -60, 0], box_max=[60, 60, 20], v_max=0.32, v_stp=0.01,
                        lam=1.0, cbs=1, smp=2, lmean0=None, vsign=-1, n=300),
    "tc_narrow_nocbs": dict(sigt=0.15, albedo=0.8, box_min=[-10, -10, 0], box_max=[10, 10, 8], v_max=0.32,
                            v_stp=0.01, lam=1.0, cbs=0, smp=1, lmean0=[0.0, 0.1, 1.0], vsign=1, n=300),
    "tc_even_grid": dict(sigt=0.1, albedo=0.9, box_min=[-30, -30, 0], box_max=[30, 30, 12], v_max=0.635,
                         v_stp=0.01, lam=1.0, cbs=1, smp=2, lmean0=None, vsign=-1, n=200),
    "tc_wide_angles": dict(sigt=0.12, albedo=1.0, box_min=[-8, -8, 0], box_max=[8, 8, 10], v_max=0.9, v_stp=0.025,
                           lam=0.8, cbs=1, smp=2, lmean0=None, vsign=-1, n=200),
    # 128 angles and more: the CTA-pair form.  161: one 256 x 256 tile, rows
    # and columns past the grid zero-filled; 301: 2 x 2 tiles per plane range
    "tc_pair_161": dict(sigt=0.1, albedo=0.9, box_min=[-30, -30, 0], box_max=[30, 30, 12], v_max=0.8, v_stp=0.01,
                        lam=1.0, cbs=1, smp=2, lmean0=None, vsign=-1, n=200),
    "tc_pair_301": dict(sigt=0.12, albedo=0.95, box_min=[-20, -20, 0], box_max=[20, 20, 10], v_max=0.9,
                        v_stp=0.006, lam=1.0, cbs=0, smp=2, lmean0=[0.0, 0.05, 1.0], vsign=-1, n=120),
}


@pytest.mark.parametrize("precision", ["mixed", "fp16"])
@pytest.mark.parametrize("name", list(TC_CASES))
def test_fourier_quad_tensor_cores_close_to_fp64(gpu, name, precision):
    from mcspeckle_b200 import _lib
    c = TC_CASES[name]
    h64 = args_for(c, "fp64")
    assert h64.nv0 >= 64
    u64 = FQ.field_fourier_quad_from_args(h64)
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    try:
        u = FQ.field_fourier_quad_from_args(args_for(c, precision))
    finally:
        _lib.profile_enable(False)
    prof = _lib.profile_read(reset=True)
    assert prof["contract_flops"] > 0  # the tensor-core form ran
    assert u.shape == u64.shape and np.isfinite(u).all()
    assert rel(u, u64) < 1e-3


@pytest.mark.parametrize("name", ["tc_wide_cbs", "tc_pair_161"])
def test_fourier_quad_tensor_cores_several_plane_groups(gpu, name):
    """More entries than one group of the tensor-core form holds (2^20), so a
    batch's plane groups run back to back from one metadata upload (both the
    single-CTA and the CTA-pair forms)."""
    from mcspeckle_b200 import _lib
    c = dict(TC_CASES[name], n=400000)
    u64 = FQ.field_fourier_quad_from_args(args_for(c, "fp64"))
    h = args_for(c, "fp16")
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    try:
        u = FQ.field_fourier_quad_from_args(h)
    finally:
        _lib.profile_enable(False)
    prof = _lib.profile_read(reset=True)
    entries = prof["contract_flops"] / (8.0 * h.nv0 * h.nv0)
    assert entries > 2 ** 20
    assert rel(u, u64) < 1e-3


def test_fourier_quad_tensor_cores_fp64_anchor(gpu, oracle_lib):
    """The FP64 reference of the tensor-core tests is the oracle's estimator."""
    h = args_for(TC_CASES["tc_wide_cbs"], "fp64")
    u = FQ.field_fourier_quad_from_args(h)
    uo = oracle_lib.field_fourier_quad(h.args, oracle_lib.Rng.philox(), h.nv0)
    assert rel(u, uo) < 1e-10


# MCfieldFourierQuadOnWave: the lights combined with complex weights Wl.
def weights(n, seed=9):
    g = np.random.default_rng(seed)
    return g.random(n) * np.exp(2j * np.pi * g.random(n))


OW_CASES = {k: FQ_CASES[k] for k in ("wide_cbs_exp", "narrow_nocbs_unif", "even_grid")}
OW_CASES.update({k: TC_CASES[k] for k in ("tc_wide_cbs", "tc_even_grid", "tc_pair_161")})


@pytest.mark.parametrize("name", list(OW_CASES))
def test_fourier_quad_onwave_fp64_matches_oracle(gpu, oracle_lib, name):
    h = args_for(OW_CASES[name], "fp64")
    W = weights(h.args.nl)
    u = FQ.field_fourier_quad_onwave_from_args(h, W)
    uo = oracle_lib.field_fourier_quad_onwave(h.args, W, oracle_lib.Rng.philox(), h.nv0)
    assert u.shape == uo.shape == (h.nv0, h.nv0)
    assert rel(u, uo) < 1e-10


@pytest.mark.parametrize("precision", ["mixed", "fp16"])
@pytest.mark.parametrize("name", list(OW_CASES))
def test_fourier_quad_onwave_close_to_fp64(gpu, name, precision):
    W = weights(2)
    u64 = FQ.field_fourier_quad_onwave_from_args(args_for(OW_CASES[name], "fp64"), W)
    u = FQ.field_fourier_quad_onwave_from_args(args_for(OW_CASES[name], precision), W)
    assert np.isfinite(u).all()
    assert rel(u, u64) < 1e-3


# Extensions (not in the reference): point sources inside the medium (the
# near-field light factor of evalphaseatt.m:10-16) and HG scattering in the
# walk.  The oracle implements the same modes in FP64.
EXT_CASES = {
    "point_source_hg_cbs": (dict(FQ_CASES["wide_cbs_exp"], n=300), dict(light_point=True, hg_g=0.9)),
    "point_source_iso_nocbs": (dict(FQ_CASES["narrow_nocbs_unif"], n=300), dict(light_point=True)),
    "hg_plane_wave": (dict(FQ_CASES["wide_angles"], n=300), dict(hg_g=0.6)),
    "tc_point_source_hg": (dict(TC_CASES["tc_wide_cbs"], n=250), dict(light_point=True, hg_g=0.9)),
    "tc_hg_plane_wave": (dict(TC_CASES["tc_narrow_nocbs"], n=250), dict(hg_g=-0.4)),
    "tc_pair_point_source_hg": (dict(TC_CASES["tc_pair_161"], n=200), dict(light_point=True, hg_g=0.9)),
}


def ext_args(name, precision):
    c, ext = EXT_CASES[name]
    if ext.get("light_point"):
        # two sources inside the box, 2 and 5 wavelengths below its top face
        bmin, bmax = np.array(c["box_min"], float), np.array(c["box_max"], float)
        L = np.array([[0.0, 0.3 * bmax[0]], [0.0, -0.2 * bmax[1]], [bmin[2] + 2.0, bmin[2] + 5.0]])
    else:
        L = cap_dirs(2, 8, +1, 21)
    return FQ.fq_args(c["sigt"], c["albedo"], c["box_min"], c["box_max"], L, c["v_max"], c["v_stp"], c["n"],
                      c["lam"], c["cbs"], c["smp"], c["lmean0"], c["vsign"], seed=SEED + 1, precision=precision,
                      **ext)


@pytest.mark.parametrize("name", list(EXT_CASES))
def test_fourier_quad_extensions_match_oracle(gpu, oracle_lib, name):
    h = ext_args(name, "fp64")
    u = FQ.field_fourier_quad_from_args(h)
    uo = oracle_lib.field_fourier_quad(h.args, oracle_lib.Rng.philox(), h.nv0)
    assert np.isfinite(uo).all() and np.linalg.norm(uo) > 0
    assert rel(u, uo) < 1e-10
    for precision in ("mixed", "fp16"):
        um = FQ.field_fourier_quad_from_args(ext_args(name, precision))
        assert rel(um, uo) < 1e-3, precision


def test_fourier_quad_extensions_change_the_estimate(gpu):
    """HG sampling and a point source give a different field than the
    reference's isotropic plane-wave form on the same seed."""
    h = ext_args("hg_plane_wave", "fp64")
    u_hg = FQ.field_fourier_quad_from_args(h)
    h.args.sct_type = 0
    u_iso = FQ.field_fourier_quad_from_args(h)
    assert rel(u_hg, u_iso) > 0.05


def test_fourier_quad_point_source_with_weights_refused(gpu):
    from mcspeckle_b200 import _lib
    h = ext_args("point_source_iso_nocbs", "fp64")
    with pytest.raises(_lib.ScmcError):
        FQ.field_fourier_quad_onwave_from_args(h, weights(h.args.nl))
