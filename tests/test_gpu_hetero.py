"""MCCovHetro / MCsampleHetro on the GPU against the FP64 oracle.

The oracle restates the reference (pinned by tests/test_oracle_golden.py);
the GPU and the oracle walk the same Philox paths through the voxel medium
(Woodcock flights, voxel albedo, voxel-marched NEE attenuation).
"""
import numpy as np
import pytest

from cases import NF_V, cap_dirs, hg_table_3d
from mcspeckle_b200 import hetero as H

pytestmark = pytest.mark.gpu
SEED = 777


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def grid3(seed=7):
    g = np.random.default_rng(seed)
    return g.lognormal(np.log(0.15), 0.5, size=(2, 2, 3)), g.uniform(0.7, 1.0, size=(2, 2, 3))


SIG3, ALB3 = grid3()
SIG2 = np.array([[1 / 30, 0, 1 / 60], [0, 1 / 120, 1 / 30]]).T
L3 = cap_dirs(3, 10, +1, 11)
V3 = cap_dirs(4, 10, -1, 12)
B3 = dict(box_min=[-20, -20, 0], box_max=[20, 20, 15], box_bin=[20, 20, 5])
B2 = dict(box_min=[-60, -60], box_max=[60, 60], box_bin=[40, 60])

CASES = {
    "3d_hg_plane_cbs_albgrid": dict(sigt=SIG3, albedo=ALB3, **B3, l=L3, v=V3, ffl=1, ffv=1, cbs=1, smp=2, st=3, amp=0.7),
    "3d_iso_voxelpick_nocbs": dict(sigt=SIG3, albedo=0.95, **B3, l=L3, v=V3, ffl=1, ffv=1, cbs=0, smp=1, st=1, amp=0),
    "3d_tab_voxelpick_nfv": dict(sigt=SIG3, albedo=0.95, **B3, l=L3, v=NF_V, ffl=1, ffv=0, cbs=1, smp=1, st=2,
                                 amp=hg_table_3d()),
    "2d_hg_plane_cbs": dict(sigt=SIG2, albedo=1.0, **B2, l=np.pi - np.deg2rad([[0.0, 4.0, 12.0]]),
                            v=np.deg2rad([[-30.0, 10.0, 170.0, 200.0]]), ffl=1, ffv=1, cbs=1, smp=2, st=3, amp=0.5),
}


def args(cov, c, n, precision):
    return H.hetero_args(cov, c["sigt"], c["albedo"], c["box_min"], c["box_max"], c["box_bin"], c["l"], c["v"],
                         c["ffl"], c["ffv"], n, 1.0, c["cbs"], c["smp"], c["st"], c["amp"], seed=SEED,
                         precision=precision)


@pytest.mark.parametrize("name", list(CASES))
def test_cov_hetero_fp64_matches_oracle(gpu, oracle_lib, name):
    h = args(True, CASES[name], 200, "fp64")
    Ms, Mm, m1 = H.cov_hetero_from_args(h)
    Mso, Mmo, m1o = oracle_lib.cov_hetero(h, oracle_lib.Rng.philox())
    assert rel(Ms, Mso) < 1e-10
    assert rel(Mm, Mmo) < 1e-10
    assert rel(m1, m1o) < 1e-10


@pytest.mark.parametrize("name", list(CASES))
def test_field_hetero_fp64_matches_oracle(gpu, oracle_lib, name):
    h = args(False, CASES[name], 300, "fp64")
    u = H.field_hetero_from_args(h)
    uo = oracle_lib.field_hetero(h, oracle_lib.Rng.philox())
    assert rel(u, uo) < 1e-10


@pytest.mark.parametrize("name", list(CASES))
def test_hetero_mixed_close_to_fp64(gpu, name):
    c = CASES[name]
    Ms64, Mm64, m64 = H.cov_hetero_from_args(args(True, c, 300, "fp64"))
    for prec in ("mixed", "fp16"):
        Ms, Mm, m1 = H.cov_hetero_from_args(args(True, c, 300, prec))
        assert rel(Ms, Ms64) < 1e-3 and rel(Mm, Mm64) < 1e-3 and rel(m1, m64) < 1e-3
    u64 = H.field_hetero_from_args(args(False, c, 300, "fp64"))
    assert rel(H.field_hetero_from_args(args(False, c, 300, "mixed")), u64) < 1e-3


# Extensions (not in the reference): trilinear sigma between voxel centres and
# tables on cos(theta) bins; the oracle implements both modes in FP64.
def cos_table(g=0.7, n=513):
    from mcspeckle_b200 import interface as I
    c = 1.0 - 2.0 * np.arange(n) / (n - 1)
    f = np.sqrt((1 - g * g) / (4 * np.pi * (1 + g * g - 2 * g * c) ** 1.5))
    t = I.tabulatedAmplitudeScatterCos(c, f)["ampfunc"]
    return {"evalAmp": t["evalAmp"], "sampleIcdf": t["sampleIcdf"], "cosBins": True}


SIG_BIG = np.random.default_rng(8).lognormal(np.log(0.15), 0.6, size=(7, 6, 5))
BBIG = dict(box_min=[-21, -18, 0], box_max=[21, 18, 15], box_bin=[6, 6, 3])
EXT = {
    "tri_hg_plane_cbs": dict(sigt=SIG_BIG, albedo=0.97, **BBIG, l=L3, v=V3, ffl=1, ffv=1, cbs=1, smp=2, st=3, amp=0.7),
    "tri_costab_voxelpick_nfv": dict(sigt=SIG_BIG, albedo=0.95, **BBIG, l=L3, v=NF_V, ffl=1, ffv=0, cbs=1, smp=1,
                                     st=2, amp=cos_table()),
    "nearest_costab_plane": dict(sigt=SIG_BIG, albedo=1.0, **BBIG, l=L3, v=V3, ffl=1, ffv=1, cbs=1, smp=2, st=2,
                                 amp=cos_table(0.9), tri=False),
}


def ext_args(cov, name, n, precision):
    c = EXT[name]
    return H.hetero_args(cov, c["sigt"], c["albedo"], c["box_min"], c["box_max"], c["box_bin"], c["l"], c["v"],
                         c["ffl"], c["ffv"], n, 1.0, c["cbs"], c["smp"], c["st"], c["amp"], seed=SEED + 1,
                         precision=precision, trilinear=c.get("tri", True))


@pytest.mark.parametrize("name", list(EXT))
def test_hetero_extensions_match_oracle(gpu, oracle_lib, name):
    h = ext_args(True, name, 250, "fp64")
    Ms, Mm, m1 = H.cov_hetero_from_args(h)
    Mso, Mmo, m1o = oracle_lib.cov_hetero(h, oracle_lib.Rng.philox())
    assert rel(Ms, Mso) < 1e-10 and rel(Mm, Mmo) < 1e-10 and rel(m1, m1o) < 1e-10
    hf = ext_args(False, name, 300, "fp64")
    assert rel(H.field_hetero_from_args(hf), oracle_lib.field_hetero(hf, oracle_lib.Rng.philox())) < 1e-10
    for prec in ("mixed", "fp16"):
        Msp, Mmp, _ = H.cov_hetero_from_args(ext_args(True, name, 250, prec))
        assert rel(Msp, Mso) < 1e-3 and rel(Mmp, Mmo) < 1e-3, prec


def test_cos_bin_table_in_the_homogeneous_path(gpu, oracle_lib):
    """The cos(theta)-bin table drives MCfield / MCcov too (sampling and
    amplitudes), in FP64 against the oracle and mixed against FP64."""
    from mcspeckle_b200 import mc as MC
    base = [0.2, 0.9, np.array([-20.0, -20.0, 0.0]), np.array([20.0, 20.0, 15.0]), L3, NF_V, 1, 0, 300, 1.0,
            True, 2, 2, cos_table(0.8)]
    h = MC.mc_args(*base, seed=SEED, precision="fp64")
    assert rel(MC.field_from_args(h), oracle_lib.field(h, oracle_lib.Rng.philox())) < 1e-10
    Ms, Mm = MC.cov_from_args(h)
    Mso, Mmo = oracle_lib.cov(h, oracle_lib.Rng.philox())
    assert rel(Ms, Mso) < 1e-10 and rel(Mm, Mmo) < 1e-10
    Msm, Mmm = MC.cov_from_args(MC.mc_args(*base, seed=SEED, precision="mixed"))
    assert rel(Msm, Mso) < 1e-3 and rel(Mmm, Mmo) < 1e-3


def test_trilinear_on_a_constant_grid_matches_nearest(gpu):
    """On a constant sigma the two lookups describe the same medium: the
    estimates agree to the 1e-4 nudges of the reference's voxel march."""
    c = dict(EXT["tri_hg_plane_cbs"], sigt=np.full((7, 6, 5), 0.2))
    EXT["_const"] = c
    try:
        a = H.cov_hetero_from_args(ext_args(True, "_const", 300, "fp64"))
        EXT["_const"] = dict(c, tri=False)
        b = H.cov_hetero_from_args(ext_args(True, "_const", 300, "fp64"))
    finally:
        EXT.pop("_const")
    assert rel(a[0], b[0]) < 1e-3 and rel(a[1], b[1]) < 1e-3
