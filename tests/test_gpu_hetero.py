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
