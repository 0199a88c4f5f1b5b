"""The MEX shims under mex/ (MCfield, MCcov, MCfieldFourierQuad), compiled
with gcc against a stub mex.h and a fake libscmc_gpu that records the argument
structs it receives: MATLAB's positional arguments must arrive in the C ABI
as the reference's .m files interpret them (MCfield.m:41-110, MCcov.m:45-70,
MCfieldFourierQuad.m:59-66), with the reference's error messages."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from mcspeckle_b200 import _abi

STUB = os.path.join(ROOT, "tests", "mexstub")


@pytest.fixture(scope="module")
def shims(tmp_path_factory):
    out = tmp_path_factory.mktemp("mex")
    libs = {}
    for name in ("MCfield", "MCcov", "MCfieldFourierQuad"):
        so = str(out / f"{name}.so")
        subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-Wno-unused-function", "-shared", "-fPIC",
                        "-I", STUB, "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "mex"),
                        os.path.join(ROOT, "mex", f"{name}_mex.c"), os.path.join(STUB, "mexstub.c"),
                        os.path.join(STUB, "fake_scmc.c"), "-o", so, "-lm"], check=True)
        L = C.CDLL(so)
        L.stub_double.restype = C.c_void_p
        L.stub_double.argtypes = [C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p]
        L.stub_struct2.restype = C.c_void_p
        L.stub_struct2.argtypes = [C.c_char_p, C.c_void_p, C.c_char_p, C.c_void_p]
        L.stub_run.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
        L.stub_err_id.restype = C.c_char_p
        L.stub_err_msg.restype = C.c_char_p
        L.stub_ndim.argtypes = [C.c_void_p]
        L.stub_dim.restype = C.c_size_t
        L.stub_dim.argtypes = [C.c_void_p, C.c_int]
        L.stub_is_complex.argtypes = [C.c_void_p]
        L.stub_data.restype = C.POINTER(C.c_double)
        L.stub_data.argtypes = [C.c_void_p]
        libs[name] = L
    return libs


class Mex:
    def __init__(self, L):
        self.L = L
        self._keep = []

    def arr(self, x):
        if isinstance(x, dict):
            return self.L.stub_struct2(b"evalAmp", self.arr(x["evalAmp"]), b"sampleIcdf", self.arr(x["sampleIcdf"]))
        a = np.asarray(x)
        if a.ndim == 0:
            a = a.reshape(1, 1)
        elif a.ndim == 1:
            a = a.reshape(1, -1)
        re = np.ascontiguousarray(a.real.astype(float).reshape(-1, order="F"))
        im = np.ascontiguousarray(a.imag.astype(float).reshape(-1, order="F")) if np.iscomplexobj(a) else None
        self._keep += [re, im]
        return self.L.stub_double(a.shape[0], a.shape[1], re.ctypes.data, None if im is None else im.ctypes.data)

    def call(self, nlhs, *args):
        prhs = (C.c_void_p * len(args))(*[self.arr(a) for a in args])
        plhs = (C.c_void_p * max(nlhs, 1))()
        rc = self.L.stub_run(nlhs, plhs, len(args), prhs)
        if rc:
            raise RuntimeError(self.L.stub_err_id().decode(), self.L.stub_err_msg().decode())
        return [self.out(plhs[i]) for i in range(nlhs)]

    def out(self, p):
        shape = tuple(self.L.stub_dim(p, k) for k in range(self.L.stub_ndim(p)))
        n = int(np.prod(shape))
        assert self.L.stub_is_complex(p)
        d = np.ctypeslib.as_array(self.L.stub_data(p), shape=(2 * n,)).copy()
        return d.view(np.complex128).reshape(shape, order="F")

    def mc(self):
        return _abi.McArgs.in_dll(self.L, "fake_mc")

    def fq(self):
        return _abi.FqArgs.in_dll(self.L, "fake_fq")

    def doubles(self, name, n):
        return np.ctypeslib.as_array((C.c_double * n).in_dll(self.L, name)).copy()


BOX3 = (np.array([[-20.0], [-20.0], [0.0]]), np.array([[20.0], [20.0], [15.0]]))
BOX2 = (np.array([[-20.0], [0.0]]), np.array([[20.0], [15.0]]))


def base3(nl=3, nv=4):
    g = np.random.default_rng(1)
    l = g.normal(size=(3, nl))
    v = g.normal(size=(3, nv))
    return [0.2, 0.9, BOX3[0], BOX3[1], l, v, 1, 1, 500, 1.0, True, 2, 3, 0.8]


def test_mcfield_arguments_reach_the_abi(shims):
    m = Mex(shims["MCfield"])
    args = base3()
    (u,) = m.call(1, *args)
    a = m.mc()
    assert (a.dim, a.nl, a.nv, a.max_itr, a.smp_flg, a.do_cbs) == (3, 3, 4, 500, 2, 1)
    assert a.sigt == 0.2 and a.albedo == 0.9 and a.lambda_ == 1.0
    assert list(a.box_min) == [-20.0, -20.0, 0.0] and list(a.box_max) == [20.0, 20.0, 15.0]
    assert a.ampfunc.sct_type == 3 and a.ampfunc.g == 0.8 and not a.has_ampfunc0 and not a.has_lmean0
    assert np.array_equal(m.doubles("fake_l", 9), args[4].reshape(-1, order="F"))
    assert np.array_equal(m.doubles("fake_v", 12), args[5].reshape(-1, order="F"))
    # the key comes from two draws of MATLAB's randi, the precision from the environment
    assert a.seed == ((123456789 << 31) ^ 987654321) and a.precision == _abi.PRECISIONS["mixed"]
    assert u.shape == (4, 3) and np.array_equal(u.reshape(-1, order="F"), np.arange(12) - 1j * np.arange(12))


def test_mcfield_2d_angle_rows_become_sin_cos(shims):
    """MCfield.m:52-66: in 2-D a 1 x N row of angles is [sin(l); cos(l)]."""
    m = Mex(shims["MCfield"])
    la = np.deg2rad([[0.0, 3.0, -4.0]])
    va = np.deg2rad([[180.0, 170.0, 185.0, 200.0]])
    m.call(1, 0.2, 0.9, BOX2[0], BOX2[1], la, va, 1, 1, 100, 1.0, True, 2, 1, 0)
    a = m.mc()
    assert (a.dim, a.nl, a.nv) == (2, 3, 4)
    assert np.allclose(m.doubles("fake_l", 6), np.stack([np.sin(la[0]), np.cos(la[0])]).reshape(-1, order="F"))
    assert np.allclose(m.doubles("fake_v", 8), np.stack([np.sin(va[0]), np.cos(va[0])]).reshape(-1, order="F"))


def test_mcfield_tables_ampfunc0_and_lmean0(shims):
    m = Mex(shims["MCfield"])
    n = 5
    amp = {"evalAmp": np.linspace(0.1, 0.5, n) + 0.01j * np.arange(n), "sampleIcdf": np.linspace(0, np.pi, n)}
    amp_real = {"evalAmp": np.linspace(0.2, 0.6, n), "sampleIcdf": np.linspace(0, np.pi, n)}
    args = base3()
    args[12], args[13] = 2, amp
    m.call(1, *args, amp_real, np.array([[0.0], [0.1], [1.0]]))
    a = m.mc()
    assert a.ampfunc.sct_type == 2 and a.ampfunc.table_n == n
    assert np.allclose(m.doubles("fake_amp", 2 * n).view(np.complex128), amp["evalAmp"])
    assert np.allclose(m.doubles("fake_icdf", n), amp["sampleIcdf"])
    assert a.has_ampfunc0 and a.ampfunc0.table_n == n
    # a real evalAmp (MATLAB stores all-real complex arrays as real) is promoted
    assert np.allclose(m.doubles("fake_amp0", 2 * n).view(np.complex128), amp_real["evalAmp"])
    assert a.has_lmean0 and list(a.lmean0) == [0.0, 0.1, 1.0]


def test_mcfield_reference_error_messages(shims):
    m = Mex(shims["MCfield"])
    args = base3()
    with pytest.raises(RuntimeError) as e:
        m.call(1, *args[:13])
    assert e.value.args[1] == "Not enough input arguments."
    with pytest.raises(RuntimeError) as e:
        m.call(1, *(args + [0.8, np.zeros((3, 1)), 7]))
    assert e.value.args[1] == "Too many input arguments."
    bad = list(args)
    bad[3] = np.array([[20.0], [20.0]])
    with pytest.raises(RuntimeError) as e:
        m.call(1, *bad)
    assert e.value.args[1] == "Invalid box size"
    bad = list(args)
    bad[4] = np.zeros((2, 3))
    with pytest.raises(RuntimeError) as e:
        m.call(1, *bad)
    assert e.value.args[1] == "Invalid light source input"
    bad = list(args)
    bad[5] = np.zeros((1, 3))
    with pytest.raises(RuntimeError) as e:
        m.call(1, *bad)
    assert e.value.args[1] == "Invalid view source input"
    # a failure inside the library becomes a MATLAB error with its message
    C.c_int.in_dll(shims["MCfield"], "fake_fail").value = 1
    try:
        with pytest.raises(RuntimeError) as e:
            m.call(1, *args)
        assert e.value.args == ("scmc:gpu:failed", "fake failure")
    finally:
        C.c_int.in_dll(shims["MCfield"], "fake_fail").value = 0


def test_mccov_outputs_and_argument_count(shims):
    m = Mex(shims["MCcov"])
    args = base3(nl=2, nv=3)
    Ms, Mm = m.call(2, *args)
    assert Ms.shape == Mm.shape == (3, 3, 2, 2)
    assert np.array_equal(Ms.reshape(-1, order="F"), np.arange(36) - 1j * np.arange(36))
    assert not C.c_int.in_dll(shims["MCcov"], "fake_cov_mm_null").value
    (Ms,) = m.call(1, *args)  # [Ms] = MCcov(...) skips copying Mm back
    assert C.c_int.in_dll(shims["MCcov"], "fake_cov_mm_null").value
    with pytest.raises(RuntimeError) as e:  # narginchk(14, 15): MCcov takes no lmean0
        m.call(2, *(args + [0.8, np.zeros((3, 1))]))
    assert e.value.args[1] == "Too many input arguments."


def test_mcfield_fourier_quad_defaults(shims):
    m = Mex(shims["MCfieldFourierQuad"])
    L = np.array([[0.0, 0.1], [0.0, 0.0], [1.0, 0.99]])
    args = [0.1, 0.9, BOX3[0], BOX3[1], L, 0.2, 0.01, 300, 1.0, 1, 2]
    (u,) = m.call(1, *args)
    a = m.fq()
    assert a.nl == 2 and a.vsign == -1.0 and not a.has_lmean0 and a.v_max == 0.2 and a.v_stp == 0.01
    assert np.array_equal(m.doubles("fake_l", 6), L.reshape(-1, order="F"))
    assert u.shape == (41, 41, 2)
    (u,) = m.call(1, *args, np.zeros((0, 0)), 1)  # lmean0 = [] keeps the default (lines 59-64)
    a = m.fq()
    assert not a.has_lmean0 and a.vsign == 1.0
    m.call(1, *args, np.array([[0.0], [0.1], [1.0]]), -1)
    assert m.fq().has_lmean0 and list(m.fq().lmean0) == [0.0, 0.1, 1.0]
    bad = list(args)
    bad[2], bad[3] = BOX2
    with pytest.raises(RuntimeError) as e:
        m.call(1, *bad)
    assert e.value.args[1] == "Invalid box size"
