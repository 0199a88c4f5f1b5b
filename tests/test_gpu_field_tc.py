"""The field on tensor cores (mixed / fp16 at nv >= 64 and nl >= 32).

The field sum u = sum_e alpha_e (a_e b_e^T [+ a0_e b2_e^T]) runs as a
real-expanded FP16 GEMM on tcgen05 with split-K slices; the result must stay
within 1e-3 (relative Frobenius) of the FP64 field on the same Philox paths,
and FP64 itself matches the CPU oracle.  Cases cover several row and column
tiles, partial tiles, far-field singles (af at finalisation), near-field
singles (CUDA-core) with tensor-core multis, CBS off (one term per event),
2-D, and a tabulated phase function.
"""
import numpy as np
import pytest

from cases import cap_dirs, hg_table_3d
from mcspeckle_b200 import _lib
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu

TOL = 1e-3
SEED = 424242


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


BOX = (np.array([-30.0, -30.0, 0.0]), np.array([30.0, 30.0, 12.0]))


def base(nv, nl, n=600, ffv=1, cbs=True, sct=3, amp=0.7):
    l = cap_dirs(nl, 10, +1, 5)
    v = cap_dirs(nv, 10, -1, 6) if ffv else np.stack([np.linspace(-8, 8, nv), np.zeros(nv), -np.full(nv, 25.0)])
    return [0.25, 0.95, BOX[0], BOX[1], l, v, 1, ffv, n, 1.0, cbs, 2, sct, amp]


def run(args, precision, extra=()):
    return MC.field_from_args(MC.mc_args(*(list(args) + list(extra)), seed=SEED, precision=precision))


def contract_launches(args, precision):
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    try:
        run(args, precision)
    finally:
        _lib.profile_enable(False)
    return _lib.profile_read(reset=True)["contract_launches"]


CASES = {
    "ff_64x32_cbs": base(64, 32),
    "ff_100x40_partial": base(100, 40),
    "ff_130x300_two_col_tiles": base(130, 300, n=200),
    "nfv_64x32_cbs": base(64, 32, ffv=0),
    "ff_96x48_nocbs": base(96, 48, cbs=False),
    "ff_64x32_tab": base(64, 32, sct=2, amp=hg_table_3d()),
}


@pytest.mark.parametrize("precision", ["mixed", "fp16"])
@pytest.mark.parametrize("name", list(CASES))
def test_field_tc_close_to_fp64(gpu, name, precision):
    args = CASES[name]
    u64 = run(args, "fp64")
    u = run(args, precision)
    assert u.shape == u64.shape
    assert np.isfinite(u).all()
    assert rel(u, u64) < TOL


def test_field_tc_path_is_taken(gpu):
    assert contract_launches(CASES["ff_64x32_cbs"], "mixed") > 0
    # below the size threshold the field stays on CUDA cores
    assert contract_launches(base(16, 16), "mixed") == 0


def test_field_tc_2d(gpu):
    nv, nl = 80, 40
    l = np.deg2rad(np.linspace(-8, 8, nl))[None, :]
    v = np.deg2rad(180 + np.linspace(-10, 10, nv))[None, :]
    args = [0.25, 0.95, np.array([-30.0, 0.0]), np.array([30.0, 12.0]), l, v, 1, 1, 800, 1.0, True, 2, 3, 0.5]
    u64 = run(args, "fp64")
    assert rel(run(args, "mixed"), u64) < TOL


def test_field_tc_fp64_oracle_anchor(gpu, oracle_lib):
    """The FP64 reference of these tests is itself the oracle's estimator."""
    args = base(64, 32, n=150)
    h = MC.mc_args(*args, seed=SEED, precision="fp64")
    assert rel(MC.field_from_args(h), oracle_lib.field(h, oracle_lib.Rng.philox())) < 1e-10


def test_field_tc_path_ranges_add_up(gpu):
    """Shards by path range (multi-GPU semantics) sum to one run."""
    args = base(64, 32, n=1000)
    full = run(args, "mixed")
    a = list(args)
    a[8] = 500
    h1 = MC.mc_args(*a, seed=SEED, precision="mixed", path_offset=0, norm_itr=1000)
    h2 = MC.mc_args(*a, seed=SEED, precision="mixed", path_offset=500, norm_itr=1000)
    assert rel(MC.field_from_args(h1) + MC.field_from_args(h2), full) < 1e-5
