"""GPU against the FP64 oracle at the exact geometry of each measured
configuration, with only the path count reduced so the oracle finishes in
seconds.

  cov64      64 x 64 covariance (N = 4096): the multi-tile FP64 CUDA-core
             product and the CTA-pair tensor-core product (FP16, hi+lo), each
             against the oracle rather than against the GPU's own FP64 mode.
  fq256      256 x 256 FourierQuad, about 10^4 z planes on a 5000-wavelength
             box: the CUDA-core FP64 form and the plane-loop tensor-core form.
  hetero128  128^3 voxel grid, 128 x 128 covariance (N = 16384), 1024-bin
             three-lobe table: the division-free voxel march on rays that
             cross the whole grid, and the tensor-core product.

FP64 must agree with the oracle to 1e-10 (same Philox paths), the reduced
precisions to 1e-3 (Frobenius, relative).
"""
import os

import numpy as np
import pytest

from mcspeckle_b200 import _lib
from mcspeckle_b200 import fourier_quad as FQ
from mcspeckle_b200 import mc as MC
from mcspeckle_b200 import workloads as WL

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 1e-3
# FourierQuad in FP16 rounds both operands, A = s_e T (the event's amplitude
# times its twiddle) and B = T, to 2^-11 relative; on the near field of a
# point source the terms cancel into a sum several times smaller than their
# RMS, so the FP16 form lands near 1.3e-3 there (hi+lo "mixed" rounds only B
# and stays under 1e-3).
FQ_FP16_TOL = 2e-3
THREADS = os.cpu_count() or 1


def rel(a, b, mask=None):
    if mask is not None:
        m = np.broadcast_to(mask, b.shape)
        a, b = a[m], b[m]
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_cov64_geometry_against_oracle(gpu, oracle_lib):
    args = WL.cov64_args(100)
    ho = MC.mc_args(*args, seed=77, precision="fp64")
    Mso, Mmo = oracle_lib.cov(ho, oracle_lib.Rng.philox(), threads=THREADS)
    Ms, Mm = MC.cov_from_args(ho)
    assert rel(Ms, Mso) < FP64_TOL and rel(Mm, Mmo) < FP64_TOL
    for prec in ("fp16", "mixed"):
        Ms, Mm = MC.cov_from_args(MC.mc_args(*args, seed=77, precision=prec))
        assert rel(Ms, Mso) < MIXED_TOL, prec
        assert rel(Mm, Mmo) < MIXED_TOL, prec
        assert rel(Ms + Mm, Mso + Mmo) < MIXED_TOL, prec


def test_cov64_hi_lo_compensates_both_operands(gpu):
    """MIXED (hi+lo) compensates both operands' FP16 rounding and keeps short
    FP32 chunks, so on the 64 x 64 geometry it is several times closer to
    FP64 than FP16 (measured 4.1e-5 against 4.1e-4 at 1e5 paths)."""
    args = WL.cov64_args(20000)
    ref = MC.cov_from_args(MC.mc_args(*args, seed=79, precision="fp64"))
    e16 = rel(np.concatenate([x.ravel() for x in MC.cov_from_args(MC.mc_args(*args, seed=79, precision="fp16"))]),
              np.concatenate([x.ravel() for x in ref]))
    emx = rel(np.concatenate([x.ravel() for x in MC.cov_from_args(MC.mc_args(*args, seed=79, precision="mixed"))]),
              np.concatenate([x.ravel() for x in ref]))
    assert e16 < MIXED_TOL
    assert emx < 1e-4 and emx < e16 / 4, (emx, e16)


@pytest.mark.parametrize("extended", [False, True], ids=["reference_form", "hg09_point_source"])
def test_fq256_geometry_against_oracle(gpu, oracle_lib, extended):
    h = WL.fq256_args(40, extended=extended, seed=78, precision="fp64")
    assert h.nv0 == 256
    uo = oracle_lib.field_fourier_quad(h.args, oracle_lib.Rng.philox(), h.nv0)
    mask = WL.fq256_propagating()
    u = FQ.field_fourier_quad_from_args(h)
    assert rel(u, uo, mask) < FP64_TOL
    for prec, tol in (("fp16", FQ_FP16_TOL), ("mixed", MIXED_TOL)):
        hp = WL.fq256_args(40, extended=extended, seed=78, precision=prec)
        assert rel(FQ.field_fourier_quad_from_args(hp), uo, mask) < tol, prec


def _device_cov_hetero(h):
    import torch

    n = h.nv * h.nv * h.nl * h.nl
    Ms = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    Mm = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    m1 = torch.empty(2 * h.nv * h.nl, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().scmc_cov_hetero_device(h.ref, Ms.data_ptr(), Mm.data_ptr(), m1.data_ptr(), None))
    torch.cuda.synchronize()
    return Ms, Mm, m1


def _rel_dev(x, ref):
    """Relative Frobenius error of a device array against a device reference, in chunks."""
    num = den = 0.0
    step = 1 << 27
    for k in range(0, ref.numel(), step):
        r = ref[k:k + step]
        num += float(((x[k:k + step] - r) ** 2).sum())
        den += float((r ** 2).sum())
    return (num / den) ** 0.5


@pytest.mark.parametrize("extended", [False, True], ids=["reference_form", "trilinear_cos_bins"])
def test_hetero128_geometry_against_oracle(gpu, oracle_lib, extended):
    """The covariance outputs are 2 x 4.3 GB: the oracle's are moved to the
    device once and compared there, chunk by chunk."""
    import torch

    h = WL.hetero128_args(8, seed=79, precision="fp64", extended=extended)
    Mso, Mmo, m1o = oracle_lib.cov_hetero(h, oracle_lib.Rng.philox(), threads=THREADS)
    ref = [torch.from_numpy(x.reshape(-1, order="F").view(np.float64)).cuda() for x in (Mso, Mmo, m1o)]
    del Mso, Mmo
    got = _device_cov_hetero(h)
    for g, r in zip(got, ref):
        assert _rel_dev(g, r) < FP64_TOL
    del got
    for prec in ("fp16", "mixed"):
        got = _device_cov_hetero(WL.hetero128_args(8, seed=79, precision=prec, extended=extended))
        for g, r in zip(got[:2], ref[:2]):
            assert _rel_dev(g, r) < MIXED_TOL, prec
        del got
        torch.cuda.empty_cache()
