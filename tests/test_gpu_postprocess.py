"""Post-processing on the GPU: refocus.m and field samples from a covariance
(the samplingFromCovMatrix example).

refocus in FP64 equals the oracle (itself pinned to refocus.m by golden
fixtures) to 1e-10, with and without the reference's unwritten first grid
point; MIXED within 1e-3.  Sampling equals the oracle given the same Philox
normals (1e-10), and the sample covariance of many samples approaches C.
"""
import json
import os

import numpy as np
import pytest

from cases import cap_dirs
from conftest import GOLDEN
from mcspeckle_b200 import mc as MC
from mcspeckle_b200 import postprocess as PP

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return json.loads(str(z["meta"])), {k: z[k] for k in z.files if k != "meta"}


@pytest.mark.parametrize("name", ["refocus_3d", "refocus_2d"])
def test_refocus_matches_reference_fixture(gpu, name):
    meta, a = golden(name)
    rU = PP.refocus(a["u"], a["v"], a["l"], a["box_min"], a["box_max"], a["box_stp"], meta["lambda"])
    assert rU.shape == a["rU"].shape
    assert rel(rU, a["rU"]) < 1e-10


@pytest.mark.parametrize("as_written", [True, False])
def test_refocus_fp64_and_mixed_vs_oracle(gpu, oracle_lib, as_written):
    g = np.random.default_rng(4)
    v = cap_dirs(300, 15, -1, 8)
    u = g.normal(size=300) + 1j * g.normal(size=300)
    args = (u, v, [0.0, 0.05, 1.0], [-20, -20, 0], [20, 20, 6], [0.5, 0.5, 0.75], 1.0)
    ro = oracle_lib.refocus(*args, as_written=as_written)
    r64 = PP.refocus(*args, as_written=as_written)
    assert rel(r64, ro) < 1e-10
    assert (r64.reshape(-1, order="F")[0] == 0) == as_written
    assert rel(PP.refocus(*args, as_written=as_written, precision="mixed"), ro) < 1e-3


def test_sample_cov_matches_oracle(gpu, oracle_lib):
    g = np.random.default_rng(2)
    N = 150  # Sigma 300 x 300: several 64-column blocks and a partial one
    A = g.normal(size=(N, 2 * N)) + 1j * g.normal(size=(N, 2 * N))
    C = A @ A.conj().T / (2 * N)
    T, seed = 3, 12345
    Z = PP.sample_from_cov(C, T, seed)
    normals = np.stack([MC.philox_stream(seed, t, 1, 2 * N) for t in range(T)])
    Zo = oracle_lib.sample_cov(C, normals)
    assert Z.shape == (N, T)
    assert rel(Z, Zo) < 1e-10


def test_sample_cov_statistics(gpu):
    """E[z z^H] = C for the samples (1000 samples, loose tolerance)."""
    g = np.random.default_rng(3)
    N = 8
    A = g.normal(size=(N, 3 * N)) + 1j * g.normal(size=(N, 3 * N))
    C = A @ A.conj().T / (3 * N)
    Z = PP.sample_from_cov(C, 4000, 99)
    Ce = Z @ Z.conj().T / Z.shape[1]
    assert rel(Ce, C) < 0.08


def test_sample_from_rendered_covariance(gpu):
    """The example's flow: a covariance from MCcov (2 lights, near-field
    views), joined into the N x N matrix, samples shaped views x lights."""
    l = np.array([[0.0, np.sin(np.deg2rad(4))], [0.0, 0.0], [1.0, np.cos(np.deg2rad(4))]])
    v = np.stack([np.linspace(-5, 5, 11), np.zeros(11), -10 * np.ones(11)])
    args = [2.0, 1.0, np.array([-10.0, -10.0, 0.0]), np.array([10.0, 10.0, 1.0]), l, v, 1, 0, 4000, 1.0, True, 2, 1,
            0]
    Ms, Mm = MC.cov_from_args(MC.mc_args(*args, seed=5, precision="fp64"))
    Cmat = Ms + Mm
    z = PP.sample_from_cov(Cmat, 2, 7)
    assert z.shape == (11, 2, 2) and np.isfinite(z).all()
    U = PP.united_cov(Cmat)
    assert np.allclose(U[:11, 11:], Cmat[:, :, 0, 1])


def test_sample_cov_singular_is_an_error(gpu):
    from mcspeckle_b200 import _lib
    C = np.zeros((4, 4), complex)
    C[0, 0] = 1.0
    with pytest.raises(_lib.ScmcError):
        PP.sample_from_cov(C, 1, 0)


def test_memory_effect_offsets_match_numpy(gpu):
    """The offset-mean reduction (memoryEffectMeasurements.m:72-86) on the GPU
    against NumPy: a random covariance on uneven grids, and Ms + Mm of the
    64 x 64 covariance configuration (8 x 8 view and light grids)."""
    from mcspeckle_b200 import mc as MC
    from mcspeckle_b200 import postprocess as PP
    from mcspeckle_b200 import workloads as WL
    g = np.random.default_rng(3)
    nvx, nvy, nlx, nly = 3, 5, 4, 2
    nv, nl = nvx * nvy, nlx * nly
    A = g.normal(size=(nv, nv, nl, nl)) + 1j * g.normal(size=(nv, nv, nl, nl))
    B = g.normal(size=A.shape) + 1j * g.normal(size=A.shape)
    R = PP.memory_effect_offsets(A, B, views_grid=(nvx, nvy), lights_grid=(nlx, nly))
    Rn = PP.memory_effect_offsets_numpy(A + B, (nvx, nvy), (nlx, nly))
    assert R.dtype == np.complex64 and R.shape == Rn.shape
    assert np.linalg.norm(R - Rn) / np.linalg.norm(Rn) < 1e-6
    # the configuration's own geometry (grid_rect flattens x-major: ix * 8 + iy, so
    # the grid's fast axis is its y axis)
    Ms, Mm = MC.cov_from_args(MC.mc_args(*WL.cov64_args(2000), seed=5, precision="fp16"))
    R = PP.memory_effect_offsets(Ms, Mm, views_grid=(8, 8), lights_grid=(8, 8))
    Rn = PP.memory_effect_offsets_numpy(Ms + Mm, (8, 8), (8, 8))
    assert R.shape == (15, 15, 15, 15)
    assert np.linalg.norm(R - Rn) / np.linalg.norm(Rn) < 1e-6
    # zero offset: the mean of the diagonal intensities is real and positive
    assert abs(Rn[7, 7, 7, 7].imag) < 1e-9 * abs(Rn[7, 7, 7, 7]) and Rn[7, 7, 7, 7].real > 0


def test_memory_effect_offsets_device_entry(gpu):
    import torch

    from mcspeckle_b200 import _lib
    from mcspeckle_b200 import postprocess as PP
    g = np.random.default_rng(4)
    nvx, nvy, nlx, nly = 4, 4, 2, 2
    nv, nl = 16, 4
    A = g.normal(size=(nv, nv, nl, nl)) + 1j * g.normal(size=(nv, nv, nl, nl))
    dA = torch.from_numpy(np.ascontiguousarray(A.reshape(-1, order="F")).view(np.float64)).cuda()
    nout = 7 * 7 * 3 * 3
    dR = torch.zeros(2 * nout, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().scmc_cov_offsets_device(dA.data_ptr(), None, nvx, nvy, nlx, nly, dR.data_ptr(), 0, None))
    torch.cuda.synchronize()
    R = dR.cpu().numpy().view(np.complex64).reshape(7, 7, 3, 3, order="F")
    Rn = PP.memory_effect_offsets_numpy(A, (nvx, nvy), (nlx, nly))
    assert np.linalg.norm(R - Rn) / np.linalg.norm(Rn) < 1e-6
