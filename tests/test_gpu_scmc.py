"""scmc() on the GPU: the argument sets of the golden scmc runs (the
reference's scmc.m executed on its own .m files) sent through
mcspeckle_b200.scmc, i.e. scmc_api._GpuKernels and the C ABI, against
scmc_api.run_config driving the FP64 oracle with the same Philox keys.

The dispatch itself (option parsing, Config, the parforIters fold, the
Csingle / C split, the field normalisation, seeding through rng) is pinned to
the reference on CPU (tests/test_oracle_golden.py, draw for draw); here the
same dispatch runs the GPU kernels and must give the oracle's result to
1e-10 in FP64 and 1e-3 in the mixed precision.
"""
import numpy as np
import pytest

from mcspeckle_b200 import interface as I
from mcspeckle_b200 import mc as MC
from mcspeckle_b200 import scmc_api as S
from test_oracle_golden import SCMC_CASES, load, make_struct

pytestmark = pytest.mark.gpu

RUN_CASES = [n for n in SCMC_CASES if not n.startswith("scmc_err")]


class PhiloxOracleKernels:
    """MCcov / MCfield of the oracle on the per-path Philox streams of a key."""

    def __init__(self, O):
        self.O = O

    def MCcov(self, *args, seed, n_total):
        return self.O.cov(MC.mc_args(*args, seed=seed, norm_itr=n_total, precision="fp64"), self.O.Rng.philox())

    def MCfield(self, *args, seed, n_total):
        return self.O.field(MC.mc_args(*args, seed=seed, norm_itr=n_total, precision="fp64"), self.O.Rng.philox())


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def scmc_inputs(name):
    meta, _ = load(name)
    t = meta["target"]
    ta = I.boxArea(*[x[0] if isinstance(x, list) and len(x) == 1 else np.asarray(x) for x in t])
    opts = []
    for k, v in meta["opts"]:
        opts += [k, v]
    return (ta, make_struct(*meta["views"]), make_struct(*meta["lights"]), make_struct(*meta["scatter"]),
            meta["iterations"], opts)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-3)])
@pytest.mark.parametrize("name", RUN_CASES)
def test_scmc_on_gpu_matches_oracle_dispatch(gpu, oracle_lib, name, precision, tol):
    ta, views, lights, sc, iters, opts = scmc_inputs(name)
    MC.rng(2024)  # both runs draw their keys from the same stream state
    got = S.scmc(ta, views, lights, sc, iters, *opts, precision=precision)
    MC.rng(2024)
    cfg = S.build_config(ta, views, lights, sc, iters, *opts)
    want = S.run_config(cfg, PhiloxOracleKernels(oracle_lib))
    keys = [k for k in ("C", "Csingle", "field") if k in want]
    assert keys and sorted(k for k in got if k != "Config") == sorted(keys)
    for k in keys:
        assert np.shape(got[k]) == np.shape(want[k]), k
        assert rel(got[k], want[k]) < tol, (k, rel(got[k], want[k]))


def test_scmc_config_reuse_on_gpu(gpu):
    """scmc(Config) reruns a stored Config (scmc.m:236-239): with a fixed rng
    option the second run repeats the first exactly."""
    ta, views, lights, sc, iters, opts = scmc_inputs("scmc_cov_default_hg")
    first = S.scmc(ta, views, lights, sc, iters, *(opts + ["rng", 5]), precision="fp64")
    again = S.scmc(first["Config"], precision="fp64")
    for k in ("C", "Csingle", "field"):
        if k in first:
            assert np.array_equal(first[k], again[k]), k
