"""Batch means and standard errors for the statistical parity tests.

Two estimators of the same expectation agree when, entry by entry, their
batch means differ by at most a few combined standard errors
z = (m1 - m2) / sqrt(se1^2 + se2^2).  Entries are taken real and imaginary
parts separately; entries whose combined standard error is zero (the exactly
real diagonal's imaginary part) are skipped.
"""
import numpy as np


def batch_stats(samples):
    """Mean and standard error (real parts in .real, imaginary in .imag)
    over the first axis."""
    s = np.asarray(samples)
    return s.mean(axis=0), complex_se(s)


def z_scores(m1, se1, m2, se2):
    """z of the real and imaginary parts; se1, se2 carry the standard errors
    of the real parts in .real and of the imaginary parts in .imag."""
    m1, m2 = np.asarray(m1).ravel(), np.asarray(m2).ravel()
    se1, se2 = np.asarray(se1).ravel(), np.asarray(se2).ravel()
    scale = max(float(np.max(np.abs(m2))), 1e-300)
    parts = []
    for f in (np.real, np.imag):
        den = np.sqrt(f(se1) ** 2 + f(se2) ** 2)
        ok = den > 1e-12 * scale
        parts.append((f(m1) - f(m2))[ok] / den[ok])
    return np.concatenate(parts)


def complex_se(samples):
    """Standard errors of the real and imaginary parts, as one complex array."""
    s = np.asarray(samples)
    k = s.shape[0]
    return (s.real.std(axis=0, ddof=1) + 1j * s.imag.std(axis=0, ddof=1)) / np.sqrt(k)


def agree(z, max_frac_over_3=0.03, max_abs=5.5):
    """Under agreement about 0.3-0.5 % of the z exceed 3 and none 5.5."""
    z = np.abs(z)
    frac, zmax = float(np.mean(z > 3.0)), float(z.max())
    return frac <= max_frac_over_3 and zmax < max_abs, frac, zmax


def tape_rng(O, seed, nu=200_000, nn=200_000):
    """An oracle random source reading MATLAB-order tapes of independent
    uniforms and normals (numpy, seeded): the reference's draw order with
    random numbers unrelated to the Philox streams."""
    g = np.random.default_rng(seed)
    return O.Rng.tape(g.random(nu), g.standard_normal(nn))
