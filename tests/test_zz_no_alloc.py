"""scmc_field_noalloc - the field entry point for callers that cannot
allocate device memory (under a pre-sized memory budget, in a real-time loop
that must not take the allocator's locks, or on threads where cudaMalloc is
not allowed).

Every test calls it through the C ABI and compares it with scmc_field, the
existing entry point, on two calls in a row: different path counts, cases
and seeds, so a second call that kept anything from the first (the fixed
scratch keeps its contents between calls) would show.  Collected last so
that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

from cases import cap_dirs, grid_dirs, small_cases
from mcspeckle_b200 import _abi, _lib
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu
# Same CUDA-core kernels on both sides.  In the reduced precisions scmc_field
# walks once and takes its records in any order, so which events one CTA sums
# in FP32 before its FP64 atomic add differs from the no-alloc entry point's
# path-ordered records: agreement to FP32 rounding, not bit for bit.
TOL = {"fp64": 1e-10, "mixed": 1e-6, "fp16": 1e-6, "fp32": 1e-5}
MIXED_TOL = 1e-3  # against FP64, as the other mixed-precision parity tests


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def noalloc(h, shape):
    import torch

    L = _lib.lib()
    L.scmc_field_noalloc.argtypes = [ctypes.POINTER(_abi.McArgs), ctypes.c_void_p, ctypes.c_void_p]
    L.scmc_field_noalloc.restype = ctypes.c_int
    d_u = torch.full((2 * int(np.prod(shape)),), float("nan"), dtype=torch.float64, device="cuda")
    _lib.check(L.scmc_field_noalloc(ctypes.byref(h.args), d_u.data_ptr(), None))
    return d_u.cpu().numpy().view(np.complex128).reshape(shape, order="F")


def case_args(case, n, seed, precision):
    name, args, extra = case
    a = list(args)
    a[8] = n
    return MC.mc_args(*(a + extra), seed=seed, precision=precision)


def test_field_noalloc_matches_scmc_field_on_two_calls(gpu):
    cases = small_cases(20000)
    # first call: 20000 paths (several internal batches); second: another case, 5000 paths
    for case, n, seed in ((cases[0], 20000, 11), (cases[2], 5000, 12)):
        h = case_args(case, n, seed, "fp64")
        ref = MC.field_from_args(h)
        got = noalloc(h, ref.shape)
        assert np.isfinite(got).all()
        assert rel(got, ref) < TOL["fp64"], case[0]


@pytest.mark.parametrize("precision", ["fp32", "mixed", "fp16"])
def test_field_noalloc_other_precisions_2d_and_tables(gpu, precision):
    """2-D, tabulated 3-D (near-field lights and views) and tabulated 2-D,
    with ampfunc0, in the reduced precisions: the tables go into the fixed
    scratch and both entry points run the same CUDA-core accumulation."""
    cases = small_cases(3000)
    for case, n, seed in ((cases[6], 3000, 21), (cases[3], 2500, 22), (cases[8], 3000, 23), (cases[4], 2000, 24)):
        h = case_args(case, n, seed, precision)
        ref = MC.field_from_args(h)
        got = noalloc(h, ref.shape)
        assert np.isfinite(got).all()
        assert rel(got, ref) < TOL[precision], (case[0], precision)


def test_field_noalloc_mixed_at_tensor_core_sizes(gpu):
    """At nv >= 64 and nl >= 32 scmc_field_device takes the tensor-core form in
    MIXED mode while scmc_field_noalloc stays on CUDA cores: both within the
    mixed tolerance of FP64 on the same paths, twice in a row."""
    l = grid_dirs(6, 5, +1)[:, :32]
    v = grid_dirs(8, 5, -1)
    base = [0.1, 1 / 1.01, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]), l, v, 1, 1, 3000, 1.0,
            True, 2, 3, 0.8]
    for n, seed in ((3000, 31), (1500, 32)):
        b = list(base)
        b[8] = n
        u64 = MC.field_from_args(MC.mc_args(*b, seed=seed, precision="fp64"))
        hmx = MC.mc_args(*b, seed=seed, precision="mixed")
        got = noalloc(hmx, u64.shape)
        assert rel(got, u64) < MIXED_TOL
        assert rel(MC.field_from_args(hmx), u64) < MIXED_TOL


def test_field_noalloc_halves_batches_when_records_overflow(gpu):
    """An optically thick, non-absorbing slab (60 mean free paths, albedo 1):
    about 150 events per path, so a batch of 8192 paths has more events than
    the fixed scratch holds; the call re-walks smaller batches and must still
    equal scmc_field.  A second, ordinary call follows."""
    l = cap_dirs(3, 10, +1, 11)
    v = cap_dirs(4, 10, -1, 12)
    thick = [1.0, 1.0, np.array([-300.0, -300.0, 0.0]), np.array([300.0, 300.0, 60.0]), l, v, 1, 1, 6000, 1.0,
             True, 2, 1, 0]
    h = MC.mc_args(*thick, seed=41, precision="fp64")
    ref = MC.field_from_args(h)
    assert rel(noalloc(h, ref.shape), ref) < TOL["fp64"]
    h2 = case_args(small_cases(2000)[1], 2000, 42, "fp64")
    ref2 = MC.field_from_args(h2)
    assert rel(noalloc(h2, ref2.shape), ref2) < TOL["fp64"]


def test_field_noalloc_limits(gpu):
    """Sizes beyond the fixed scratch are refused with SCMC_ERR_INVALID and a
    message; the next call works."""
    name, args, extra = small_cases(100)[0]
    a = list(args)
    a[4] = cap_dirs(256, 10, +1, 5)
    a[5] = cap_dirs(257, 10, -1, 6)  # nv * nl = 65792 > 65536
    with pytest.raises(_lib.ScmcError) as ei:
        noalloc(MC.mc_args(*a, seed=1, precision="fp64"), (257, 256))
    assert ei.value.status == _abi.SCMC_ERR_INVALID and "65536" in str(ei.value)
    # a tabulated table longer than 16384 entries
    big = {"evalAmp": np.full(16385, 0.1 + 0.0j), "sampleIcdf": np.linspace(0, np.pi, 16385)}
    a = list(args)
    a[12], a[13] = 2, big
    with pytest.raises(_lib.ScmcError) as ei:
        noalloc(MC.mc_args(*a, seed=1, precision="fp64"), (4, 3))
    assert ei.value.status == _abi.SCMC_ERR_INVALID and "16384" in str(ei.value)
    h = case_args(small_cases(500)[0], 500, 3, "fp64")
    ref = MC.field_from_args(h)
    assert rel(noalloc(h, ref.shape), ref) < TOL["fp64"]
