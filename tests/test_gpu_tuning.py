"""Tuned launch parameters change speed, not results: solves with the
autotuner's alternatives (3-stage CTA pair, small covariance chunks, small
path batches, field split-K, small FourierQuad plane groups) stay within the
mixed tolerance of FP64 on the same paths, and FP64 is unchanged by the path
batch size up to the order of its sums."""
import ctypes as C

import numpy as np
import pytest

from cases import grid_dirs
from mcspeckle_b200 import _abi, _lib
from mcspeckle_b200 import fourier_quad as FQ
from mcspeckle_b200 import mc as MC

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture()
def tuning():
    L = _lib.lib()
    _lib.check(L.scmc_tuning_clear())

    def put(kind, prec, **vals):
        t = _abi.Tuning(kind=kind, precision=_abi.PRECISIONS[prec], n_lo=0, n_hi=1 << 40, **vals)
        _lib.check(L.scmc_tuning_set(C.byref(t)))
    yield put
    _lib.check(L.scmc_tuning_clear())


def cov_args(n=3000):
    return [0.101, 1 / 1.01, np.array([-100.0, -100.0, 0.0]), np.array([100.0, 100.0, 50.0]), grid_dirs(4, 5, +1),
            grid_dirs(8, 5, -1), 1, 1, n, 1.0, True, 2, 3, 0.8]


def test_tuned_covariance(gpu, tuning):
    ref = MC.cov_from_args(MC.mc_args(*cov_args(), seed=5, precision="fp64"))
    tuning(_abi.SCMC_TUNE_COV, "fp16", stages=3, chunk_events=4096, path_batch=1000)
    tuning(_abi.SCMC_TUNE_COV, "mixed", chunk_events=2048, path_batch=700)
    tuning(_abi.SCMC_TUNE_COV, "fp64", path_batch=900)
    for prec in ("fp16", "mixed"):
        got = MC.cov_from_args(MC.mc_args(*cov_args(), seed=5, precision=prec))
        assert rel(got[0], ref[0]) < 1e-3 and rel(got[1], ref[1]) < 1e-3, prec
    got = MC.cov_from_args(MC.mc_args(*cov_args(), seed=5, precision="fp64"))
    assert rel(got[0], ref[0]) < 1e-12 and rel(got[1], ref[1]) < 1e-12


def test_tuned_field_and_fourier_quad(gpu, tuning):
    base = cov_args(4000)
    base[4], base[5] = grid_dirs(6, 5, +1), grid_dirs(9, 5, -1)  # 81 views x 36 lights: tensor-core field
    ref = MC.field_from_args(MC.mc_args(*base, seed=6, precision="fp64"))
    tuning(_abi.SCMC_TUNE_FIELD, "fp16", ksplit=3, path_batch=1500)
    assert rel(MC.field_from_args(MC.mc_args(*base, seed=6, precision="fp16")), ref) < 1e-3
    L = np.array([[0.0], [0.05], [1.0]])
    fq = lambda p: FQ.fq_args(0.1, 0.9, [-60, -60, 0], [60, 60, 20], L / np.linalg.norm(L), 0.32, 0.01, 600, 1.0, 1,
                              2, None, -1, seed=7, precision=p)  # noqa: E731
    uref = FQ.field_fourier_quad_from_args(fq("fp64"))
    tuning(_abi.SCMC_TUNE_FQ, "fp16", group_entries=4096, path_batch=200)
    assert rel(FQ.field_fourier_quad_from_args(fq("fp16")), uref) < 1e-3
