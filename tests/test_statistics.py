"""Statistical parity on CPU: the estimator on the per-path Philox streams
(the GPU's random numbers; the GPU's FP64 mode equals the oracle on them to
1e-10) against the same estimator reading MATLAB-order tapes of independent
uniforms and normals (the reference's draw order), over independent batches,
within 3 standard errors; the field-vs-covariance identity E[u u^H] = Ms + Mm
that examples/testHetro/testHetroCov.m:70-84 checks; and that the test has
the power to see a planted change of the medium."""
import numpy as np
import pytest

from cases import small_cases
from mcspeckle_b200 import mc as MC
from stats_util import agree, batch_stats, tape_rng, z_scores

K, N_PATHS = 30, 2000


def case_args(ci, n):
    name, args, extra = small_cases(n)[ci]
    a = list(args)
    a[8] = n
    return name, a + extra


def cov_batches(O, a, rng_of):
    return np.array([sum(O.cov(MC.mc_args(*a, seed=1000 + k, precision="fp64"), rng_of(k))) for k in range(K)])


@pytest.mark.parametrize("ci", [0, 1, 3])
def test_philox_and_tape_estimators_agree(oracle_lib, ci):
    O = oracle_lib
    name, a = case_args(ci, N_PATHS)
    m1, s1 = batch_stats(cov_batches(O, a, lambda k: O.Rng.philox()))
    m2, s2 = batch_stats(cov_batches(O, a, lambda k: tape_rng(O, 500 + k)))
    ok, frac, zmax = agree(z_scores(m1, s1, m2, s2))
    assert ok, (name, frac, zmax)


def test_field_outer_products_estimate_the_covariance(oracle_lib):
    O = oracle_lib
    name, a = case_args(0, N_PATHS)
    m_c, s_c = batch_stats(cov_batches(O, a, lambda k: O.Rng.philox()))
    S, m = 3000, 100
    b = a[:8] + [m] + a[9:]
    us = np.array([O.field(MC.mc_args(*b, seed=77, precision="fp64", path_offset=m * s), O.Rng.philox())
                   for s in range(S)])
    mu, s_u = batch_stats(np.einsum("sij,skl->sikjl", us, us.conj()))  # (v1, v2, l1, l2)
    ok, frac, zmax = agree(z_scores(mu, s_u, m_c, s_c))
    assert ok, (frac, zmax)


def test_planted_change_is_detected(oracle_lib):
    """The same comparison against a medium with albedo 0.85 instead of 0.9
    fails: the test can tell estimators apart."""
    O = oracle_lib
    name, a = case_args(0, N_PATHS)
    m1, s1 = batch_stats(cov_batches(O, a, lambda k: O.Rng.philox()))
    b = list(a)
    b[1] = 0.85
    m2, s2 = batch_stats(cov_batches(O, b, lambda k: tape_rng(O, 500 + k)))
    ok, frac, zmax = agree(z_scores(m1, s1, m2, s2))
    assert not ok and zmax > 5.5, (frac, zmax)
