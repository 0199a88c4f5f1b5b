"""The bounded device waits of the tensor-core kernels, made to run out.

scmc_test_wait_fault(1) makes every tensor-core launch issue no copy and wait
only 1 ms: the MMA issuer's first wait gives up, the kernel flags its error,
waits for nothing in flight, frees its tensor memory and returns.  Each call
must then report SCMC_ERR_TIMEOUT, and once the fault is off the next call on
the same context must be correct again.  Covers the CTA-pair covariance
kernel (N >= 256), the single-CTA kernel (covariance N < 256 and the
tensor-core field) and the FourierQuad plane loop.
"""
import numpy as np
import pytest

from cases import grid_dirs
from mcspeckle_b200 import _abi, _lib
from mcspeckle_b200 import fourier_quad as FQ
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def cov_args(nside_v, nside_l, n=1500):
    return [0.101, 1 / 1.01, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]),
            grid_dirs(nside_l, 5, +1), grid_dirs(nside_v, 5, -1), 1, 1, n, 1.0, True, 2, 3, 0.8]


def field_tc_args():
    return [0.1, 1 / 1.01, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]), grid_dirs(6, 5, +1),
            grid_dirs(8, 5, -1), 1, 1, 2000, 1.0, True, 2, 3, 0.8]


def fq_args(precision):
    L = np.array([[0.0], [0.05], [1.0]])
    return FQ.fq_args(0.1, 0.9, [-60, -60, 0], [60, 60, 20], L / np.linalg.norm(L), 0.32, 0.01, 300, 1.0, 1, 2,
                      None, -1, seed=5, precision=precision)


SOLVES = {
    "cov_cta_pair": lambda p: MC.cov_from_args(MC.mc_args(*cov_args(8, 4), seed=3, precision=p)),
    "cov_single_cta": lambda p: MC.cov_from_args(MC.mc_args(*cov_args(4, 3), seed=3, precision=p)),
    "field_tensor_cores": lambda p: MC.field_from_args(MC.mc_args(*field_tc_args(), seed=3, precision=p)),
    "fourier_quad_planes": lambda p: FQ.field_fourier_quad_from_args(fq_args(p)),
}


def fault(on):
    _lib.check(_lib.lib().scmc_test_wait_fault(int(on)))


@pytest.mark.parametrize("precision", ["fp16", "mixed"])
@pytest.mark.parametrize("name", list(SOLVES))
def test_bounded_wait_runs_out_and_context_recovers(gpu, name, precision):
    solve = SOLVES[name]
    ref = solve("fp64")
    fault(True)
    try:
        with pytest.raises(_lib.ScmcError) as ei:
            solve(precision)
        assert ei.value.status == _abi.SCMC_ERR_TIMEOUT
        assert "bounded wait" in str(ei.value)
    finally:
        fault(False)
    got = solve(precision)
    ref, got = (ref, got) if isinstance(ref, tuple) else ((ref,), (got,))
    for r, g in zip(ref, got):
        assert np.isfinite(g).all()
        assert rel(g, r) < 1e-3
