"""MCfieldOnWave on the GPU: the lights combined with complex weights Wl.

FP64 against the oracle (itself pinned to MCfieldOnWave.m by the golden
fixtures) on the same Philox paths; equal to the full field times Wl on the
same paths (the identity the reference's OnWave test checks for
FourierQuad); MIXED / plain FP32 close to FP64.
"""
import numpy as np
import pytest

from cases import BOX2, BOX3, NF_V, cap_dirs, hg_table_3d
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu
SEED = 777


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def weights(n, seed=3):
    g = np.random.default_rng(seed)
    return g.random(n) * np.exp(2j * np.pi * g.random(n))


def base(box, l, v, ffl, ffv, cbs, smp, sct, amp, n=300):
    return [0.2, 0.9, np.asarray(box[0]), np.asarray(box[1]), l, v, ffl, ffv, n, 1.0, cbs, smp, sct, amp]


L3 = cap_dirs(5, 10, +1, 11)
V3 = cap_dirs(6, 10, -1, 12)
CASES = {
    "3d_hg_ff_cbs": (base(BOX3, L3, V3, 1, 1, True, 2, 3, 0.7), [0.4, [0.0, 0.1, 1.0]]),
    "3d_tab_nfv_nocbs": (base(BOX3, L3, NF_V, 1, 0, False, 1, 2, hg_table_3d()), [hg_table_3d(), [0.0, 0.0, 1.0]]),
    "3d_hg_nocbs_defaults": (base(BOX3, L3, V3, 1, 1, False, 2, 3, -0.3), []),
    "3d_iso_one_light": (base(BOX3, L3[:, :1], V3, 1, 1, True, 2, 1, 0), [0, [0.0, 0.0, 1.0]]),
    "2d_hg_cbs": (base(BOX2, np.array([[0.0, 0.05]]), np.array([[3.1, 3.2, 3.0]]), 1, 1, True, 2, 3, 0.5),
                  [0.5, [0.0, 1.0]]),
}


def holder(name, precision):
    args, extra = CASES[name]
    return MC.mc_args(*(args + extra), seed=SEED, precision=precision)


@pytest.mark.parametrize("name", list(CASES))
def test_onwave_fp64_matches_oracle(gpu, oracle_lib, name):
    h = holder(name, "fp64")
    W = weights(h.args.nl)
    u = MC.field_onwave_from_args(h, W)
    uo = oracle_lib.field_onwave(h, W, oracle_lib.Rng.philox())
    assert u.shape == uo.shape == (h.args.nv, 1)
    assert rel(u, uo) < 1e-10


@pytest.mark.parametrize("name", ["3d_hg_ff_cbs", "3d_tab_nfv_nocbs", "2d_hg_cbs"])
def test_onwave_equals_field_times_weights(gpu, name):
    h = holder(name, "fp64")
    W = weights(h.args.nl)
    u = MC.field_onwave_from_args(h, W)
    U = MC.field_from_args(holder(name, "fp64"))
    assert rel(u, U @ W.reshape(-1, 1)) < 1e-10


@pytest.mark.parametrize("name", list(CASES))
def test_onwave_mixed_and_fp32_close_to_fp64(gpu, name):
    W = weights(holder(name, "fp64").args.nl)
    u64 = MC.field_onwave_from_args(holder(name, "fp64"), W)
    assert rel(MC.field_onwave_from_args(holder(name, "mixed"), W), u64) < 1e-3
    assert rel(MC.field_onwave_from_args(holder(name, "fp32"), W), u64) < 1e-2


def test_onwave_large_view_chunks(gpu):
    """More views than one CTA chunk (2048) and many lights."""
    l = cap_dirs(150, 10, +1, 5)
    v = cap_dirs(2500, 10, -1, 6)
    args = [0.2, 0.95, np.array([-30.0, -30.0, 0.0]), np.array([30.0, 30.0, 12.0]), l, v, 1, 1, 200, 1.0, True, 2,
            3, 0.6]
    W = weights(150)
    u64 = MC.field_onwave_from_args(MC.mc_args(*args, seed=SEED, precision="fp64"), W)
    U = MC.field_from_args(MC.mc_args(*args, seed=SEED, precision="fp64"))
    assert rel(u64, U @ W.reshape(-1, 1)) < 1e-10
    assert rel(MC.field_onwave_from_args(MC.mc_args(*args, seed=SEED, precision="mixed"), W), u64) < 1e-3
