"""scmc_field_noalloc - the field entry point for callers that cannot
allocate device memory (under a pre-sized memory budget, in a real-time loop
that must not take the allocator's locks, or on threads where cudaMalloc is
not allowed).

It is called through the C ABI and compared with scmc_field, the existing
entry point, on two calls in a row: different path counts and seeds, so a
second call that kept anything from the first (the fixed scratch keeps its
contents between calls) would show.  Collected last so that a run stopping
at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

from cases import small_cases
from mcspeckle_b200 import _abi, _lib
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu
TOL = 1e-10  # FP64 mode, the same tolerance as the other FP64 parity tests


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_field_noalloc_matches_scmc_field_on_two_calls(gpu):
    import torch

    L = _lib.lib()
    L.scmc_field_noalloc.argtypes = [ctypes.POINTER(_abi.McArgs), ctypes.c_void_p, ctypes.c_void_p]
    L.scmc_field_noalloc.restype = ctypes.c_int
    cases = small_cases(20000)
    # first call: 20000 paths (several internal batches); second: another case, 5000 paths
    for (name, args, extra), n, seed in ((cases[0], 20000, 11), (cases[2], 5000, 12)):
        a = list(args)
        a[8] = n
        h = MC.mc_args(*(a + extra), seed=seed, precision="fp64")
        ref = MC.field_from_args(h)
        d_u = torch.full((2 * ref.size,), float("nan"), dtype=torch.float64, device="cuda")
        _lib.check(L.scmc_field_noalloc(ctypes.byref(h.args), d_u.data_ptr(), None))
        got = d_u.cpu().numpy().view(np.complex128).reshape(ref.shape, order="F")
        assert np.isfinite(got).all()
        assert rel(got, ref) < TOL, name
