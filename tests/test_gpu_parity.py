"""Parity of the CUDA path (through the C ABI) with the CPU FP64 oracle.

The GPU walk and the oracle draw from the same per-path Philox-4x32-10
streams, so in FP64 mode they compute the same estimator on the same paths:
tolerance 1e-10 relative (Frobenius).  Mixed precision (FP16 hi+lo tensor
cores, FP32 phases after FP64 range reduction) must stay within 1e-3 of
FP64 on the same paths.
"""
import numpy as np
import pytest

from cases import grid_dirs, small_cases
from mcspeckle_b200 import _abi
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 1e-3
SEED = 1234567


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def args_for(case, **kw):
    name, args, extra = case
    return MC.mc_args(*(args + extra), seed=SEED, **kw)


CASES = small_cases(300)
IDS = [c[0] for c in CASES]


def test_philox_streams_bit_exact(gpu, oracle_lib):
    for seed, path in [(0, 0), (SEED, 7), (2**63 + 5, 2**40 + 3)]:
        gu = MC.philox_stream(seed, path, 0, 257)
        ou = oracle_lib.philox_stream(seed, path, 0, 257)
        assert np.array_equal(gu, ou)
        gn = MC.philox_stream(seed, path, 1, 257)
        on = oracle_lib.philox_stream(seed, path, 1, 257)
        assert np.max(np.abs(gn - on)) < 1e-13


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_records_match_oracle_walk(gpu, oracle_lib, case):
    h = args_for(case, precision="fp64")
    r = MC.export_records(h, True, 20000)
    o = oracle_lib.records(h, oracle_lib.Rng.philox(), True, 20000)
    assert r.n == o.n
    assert np.array_equal(r.plen, o.plen)
    assert np.array_equal(r.path, o.path)
    for k in ("x", "ow", "x1", "w1", "wpx", "xi"):
        a, b = getattr(r, k), getattr(o, k)
        assert np.max(np.abs(a - b)) <= 1e-9 * max(1.0, np.max(np.abs(b))), k


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_field_fp64_matches_oracle(gpu, oracle_lib, case):
    h = args_for(case, precision="fp64")
    u = MC.field_from_args(h)
    uo = oracle_lib.field(h, oracle_lib.Rng.philox())
    assert u.shape == uo.shape
    assert rel(u, uo) < FP64_TOL


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_cov_fp64_matches_oracle(gpu, oracle_lib, case):
    h = args_for(case, precision="fp64")
    Ms, Mm = MC.cov_from_args(h)
    Mso, Mmo = oracle_lib.cov(h, oracle_lib.Rng.philox())
    assert rel(Ms, Mso) < FP64_TOL
    assert rel(Mm, Mmo) < FP64_TOL


@pytest.mark.parametrize("case", CASES[:4], ids=IDS[:4])
def test_replay_of_gpu_records(gpu, oracle_lib, case):
    """Oracle accumulation of the GPU's own records equals the GPU result."""
    hf = args_for(case, precision="fp64")
    rf = MC.export_records(hf, True, 20000)
    recs = oracle_lib.Records(rf.n)
    for k in ("x", "ow", "x1", "w1", "wpx", "xi", "plen", "path"):
        setattr(recs, k, getattr(rf, k))
    recs.n = rf.n
    assert rel(MC.field_from_args(hf), oracle_lib.field_from_records(hf, recs)) < FP64_TOL
    rc = MC.export_records(hf, False, 20000)
    recs = oracle_lib.Records(rc.n)
    for k in ("x", "ow", "x1", "w1", "wpx", "xi", "plen", "path"):
        setattr(recs, k, getattr(rc, k))
    recs.n = rc.n
    Ms, Mm = MC.cov_from_args(hf)
    Mso, Mmo = oracle_lib.cov_from_records(hf, recs)
    assert rel(Ms, Mso) < FP64_TOL and rel(Mm, Mmo) < FP64_TOL


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_mixed_and_fp32_close_to_fp64(gpu, case):
    h64 = args_for(case, precision="fp64")
    hmx = args_for(case, precision="mixed")
    h32 = args_for(case, precision="fp32")
    u64 = MC.field_from_args(h64)
    assert rel(MC.field_from_args(hmx), u64) < MIXED_TOL
    assert rel(MC.field_from_args(h32), u64) < 1e-2
    Ms64, Mm64 = MC.cov_from_args(h64)
    Msm, Mmm = MC.cov_from_args(hmx)
    assert rel(Msm, Ms64) < MIXED_TOL
    assert rel(Mmm, Mm64) < MIXED_TOL
    Ms16, Mm16 = MC.cov_from_args(args_for(case, precision="fp16"))
    assert rel(Ms16, Ms64) < MIXED_TOL and rel(Mm16, Mm64) < MIXED_TOL
    Ms32, Mm32 = MC.cov_from_args(h32)
    assert rel(Ms32, Ms64) < 1e-2 and rel(Mm32, Mm64) < 1e-2


@pytest.mark.parametrize("precision", ["mixed", "fp16"])
@pytest.mark.parametrize("nside_v,nside_l", [(4, 4), (8, 4), (5, 3), (6, 5), (8, 8)])
def test_tensor_core_cov_tiles(gpu, nside_v, nside_l, precision):
    """Mixed (tcgen05) vs FP64 covariance at sizes that exercise several
    tiles, partial tiles and the diagonal tiles of the Hermitian update."""
    l = grid_dirs(nside_l, 5, +1)
    v = grid_dirs(nside_v, 5, -1)
    base = [1.01 / 10, 1 / 1.01, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]), l, v, 1, 1,
            2000, 1.0, True, 2, 3, 0.8]
    Ms64, Mm64 = MC.cov_from_args(MC.mc_args(*base, seed=SEED, precision="fp64"))
    Msm, Mmm = MC.cov_from_args(MC.mc_args(*base, seed=SEED, precision=precision))
    assert rel(Msm, Ms64) < MIXED_TOL
    assert rel(Mmm, Mm64) < MIXED_TOL
    # Hermitian structure C(v1,v2,l1,l2) = conj(C(v2,v1,l2,l1))
    assert np.max(np.abs(Mmm - np.conj(Mmm.transpose(1, 0, 3, 2)))) <= 1e-12 * np.max(np.abs(Mmm))
    # the diagonal of a sum of t t^H is real and non-negative
    d = np.einsum("iijj->ij", Mmm)
    assert np.all(d.imag == 0) and np.all(d.real >= 0)


def test_path_ranges_add_up(gpu):
    """Sharding by path ranges: two halves with the total normalisation sum
    to one run (the multi-GPU and parforIters semantics)."""
    name, args, extra = CASES[0]
    n = 4000
    a = list(args)
    a[8] = n
    full = MC.field_from_args(MC.mc_args(*(a + extra), seed=SEED, precision="fp64"))
    a[8] = n // 2
    h1 = MC.mc_args(*(a + extra), seed=SEED, precision="fp64", path_offset=0, norm_itr=n)
    h2 = MC.mc_args(*(a + extra), seed=SEED, precision="fp64", path_offset=n // 2, norm_itr=n)
    assert rel(MC.field_from_args(h1) + MC.field_from_args(h2), full) < 1e-12
    Ms, Mm = MC.cov_from_args(MC.mc_args(*(args[:8] + [n] + args[9:] + extra), seed=SEED, precision="fp64"))
    a1 = MC.cov_from_args(h1)
    a2 = MC.cov_from_args(h2)
    assert rel(a1[0] + a2[0], Ms) < 1e-12 and rel(a1[1] + a2[1], Mm) < 1e-12


def test_edge_cases(gpu):
    name, args, extra = CASES[0]
    a = list(args)
    a[8] = 0
    u = MC.field_from_args(MC.mc_args(*a, seed=1, precision="fp64"))
    assert np.all(u == 0)
    Ms, Mm = MC.cov_from_args(MC.mc_args(*a, seed=1, precision="mixed"))
    assert np.all(Ms == 0) and np.all(Mm == 0)
    # a single light and view
    a = list(args)
    a[4] = args[4][:, :1]
    a[5] = args[5][:, :1]
    a[8] = 500
    h = MC.mc_args(*a, seed=3, precision="fp64")
    u = MC.field_from_args(h)
    assert u.shape == (1, 1) and np.isfinite(u).all()
    # event cap
    a = list(args)
    with pytest.raises(MC._lib.ScmcError) as ei:
        MC.field_from_args(MC.mc_args(*a, seed=3, precision="fp64", max_events_per_path=1))
    assert ei.value.status == _abi.SCMC_ERR_LIMIT
    # invalid precision reaches the C ABI validation
    h = MC.mc_args(*a, seed=3, precision="fp64")
    h.args.precision = 9
    with pytest.raises(MC._lib.ScmcError) as ei:
        MC.field_from_args(h)
    assert ei.value.status == _abi.SCMC_ERR_INVALID
