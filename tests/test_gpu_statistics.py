"""Statistical parity on the GPU (the north-star check): covariance
estimates from independent Philox keys on the GPU, in FP64 and in the mixed
precision, against the oracle reading MATLAB-order tapes of independent
random numbers (the reference's estimator and draw order), batch by batch,
within 3 standard errors per entry; and the identity E[u u^H] = Ms + Mm of
examples/testHetro/testHetroCov.m:70-84 with both sides from the GPU (field
samples of 100 paths each against covariance batches)."""
import numpy as np
import pytest

from cases import small_cases
from mcspeckle_b200 import mc as MC
from stats_util import agree, batch_stats, tape_rng, z_scores

pytestmark = pytest.mark.gpu
K, N_PATHS = 30, 2000


def case_args(ci, n):
    name, args, extra = small_cases(n)[ci]
    a = list(args)
    a[8] = n
    return name, a + extra


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("ci", [0, 1, 3])
def test_gpu_estimates_agree_with_tape_oracle(gpu, oracle_lib, ci, precision):
    O = oracle_lib
    name, a = case_args(ci, N_PATHS)
    gpu_b = np.array([sum(MC.cov_from_args(MC.mc_args(*a, seed=9000 + k, precision=precision))) for k in range(K)])
    tape_b = np.array([sum(O.cov(MC.mc_args(*a, seed=0, precision="fp64"), tape_rng(O, 700 + k))) for k in range(K)])
    m1, s1 = batch_stats(gpu_b)
    m2, s2 = batch_stats(tape_b)
    ok, frac, zmax = agree(z_scores(m1, s1, m2, s2))
    assert ok, (name, precision, frac, zmax)


def test_gpu_field_outer_products_estimate_gpu_covariance(gpu):
    name, a = case_args(3, N_PATHS)  # near-field lights and views, tabulated, CBS
    m_c, s_c = batch_stats(np.array([sum(MC.cov_from_args(MC.mc_args(*a, seed=9100 + k, precision="fp64")))
                                     for k in range(K)]))
    S, m = 3000, 100
    b = a[:8] + [m] + a[9:]
    us = np.array([MC.field_from_args(MC.mc_args(*b, seed=9200, precision="fp64", path_offset=m * s))
                   for s in range(S)])
    mu, s_u = batch_stats(np.einsum("sij,skl->sikjl", us, us.conj()))
    ok, frac, zmax = agree(z_scores(mu, s_u, m_c, s_c))
    assert ok, (frac, zmax)
