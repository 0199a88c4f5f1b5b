"""Loader for the in-tree CUDA library libscmc_gpu.so.

There is no CPU fallback: if the library is missing or no sm_100 device is
visible, calls fail loudly with ScmcError.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libscmc_gpu.so")
_lock = threading.Lock()
_lib = None

_STATUS = {
    _abi.SCMC_ERR_INVALID: "invalid argument",
    _abi.SCMC_ERR_CUDA: "CUDA error",
    _abi.SCMC_ERR_NOMEM: "out of memory",
    _abi.SCMC_ERR_NODEVICE: "no sm_100 device",
    _abi.SCMC_ERR_TIMEOUT: "device wait timed out",
    _abi.SCMC_ERR_CANCELLED: "cancelled",
    _abi.SCMC_ERR_LIMIT: "limit exceeded",
}


class ScmcError(RuntimeError):
    """A non-zero scmc_status from the C ABI (message from scmc_last_error)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def lib():
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ScmcError(_abi.SCMC_ERR_NODEVICE,
                            f"libscmc_gpu.so is not built ({LIB_PATH}); run mcspeckle_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        lp = C.POINTER(C.c_int64)
        mp = C.POINTER(_abi.McArgs)
        L.scmc_abi_version.restype = C.c_int
        L.scmc_last_error.restype = C.c_char_p
        L.scmc_launch_count.restype = C.c_int64
        L.scmc_field.argtypes = [mp, dp]
        L.scmc_field_device.argtypes = [mp, C.c_void_p, C.c_void_p]
        L.scmc_cov.argtypes = [mp, dp, dp]
        L.scmc_field_onwave.argtypes = [mp, dp, dp]
        L.scmc_field_onwave_device.argtypes = [mp, dp, C.c_void_p, C.c_void_p]
        L.scmc_cov_device.argtypes = [mp, C.c_void_p, C.c_void_p, C.c_void_p]
        L.scmc_export_records.argtypes = [mp, C.c_int32, C.c_int64, dp, dp, dp, dp, dp, dp, ip, lp, lp]
        L.scmc_philox_stream.argtypes = [C.c_uint64, C.c_uint64, C.c_int32, C.c_int64, dp]
        L.scmc_field_from_records.argtypes = [mp, C.c_int64, dp, dp, dp, dp, dp, dp, ip, lp, dp]
        fq = C.POINTER(_abi.FqArgs)
        L.scmc_fq_grid_size.argtypes = [C.c_double, C.c_double, C.POINTER(C.c_int64)]
        L.scmc_field_fourier_quad.argtypes = [fq, dp]
        L.scmc_field_fourier_quad_device.argtypes = [fq, C.c_void_p, C.c_void_p]
        L.scmc_field_fourier_quad_onwave.argtypes = [fq, dp, dp]
        L.scmc_field_fourier_quad_onwave_device.argtypes = [fq, dp, C.c_void_p, C.c_void_p]
        L.scmc_field_noalloc.argtypes = [mp, C.c_void_p, C.c_void_p]
        hp = C.POINTER(_abi.HeteroArgs)
        L.scmc_cov_hetero.argtypes = [hp, dp, dp, dp]
        L.scmc_field_hetero.argtypes = [hp, dp]
        L.scmc_cov_hetero_device.argtypes = [hp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.scmc_field_hetero_device.argtypes = [hp, C.c_void_p, C.c_void_p]
        vp = C.c_void_p
        L.scmc_server_create.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.POINTER(vp)]
        L.scmc_server_submit.argtypes = [vp, C.c_int32, mp, dp, dp, C.POINTER(C.c_int64)]
        L.scmc_server_wait.argtypes = [vp, C.c_int64, C.c_int64, C.POINTER(_abi.RequestInfo)]
        L.scmc_server_stats_read.argtypes = [vp, C.POINTER(_abi.ServerStats)]
        L.scmc_server_destroy.argtypes = [vp]
        L.scmc_refocus_grid.argtypes = [C.c_int32, dp, dp, dp, lp, lp]
        L.scmc_refocus.argtypes = [dp, dp, C.c_int64, C.c_int32, dp, dp, dp, dp, C.c_double, C.c_int32, C.c_int32,
                                   C.c_int32, dp]
        L.scmc_sample_cov.argtypes = [dp, C.c_int64, C.c_int64, C.c_uint64, C.c_int32, dp]
        L.scmc_profile_enable.argtypes = [C.c_int32]
        fp = C.POINTER(C.c_float)
        L.scmc_cov_offsets.argtypes = [dp, dp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, fp, C.c_int32]
        L.scmc_cov_offsets_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                              C.c_void_p, C.c_int32, C.c_void_p]
        L.scmc_cov_offsets.restype = C.c_int
        L.scmc_cov_offsets_device.restype = C.c_int
        L.scmc_test_wait_fault.argtypes = [C.c_int32]
        L.scmc_tuning_set.argtypes = [C.POINTER(_abi.Tuning)]
        L.scmc_tuning_load.argtypes = [C.c_char_p]
        L.scmc_tuning_get.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.POINTER(_abi.Tuning)]
        for name in ("scmc_tuning_set", "scmc_tuning_clear", "scmc_tuning_load", "scmc_tuning_get"):
            getattr(L, name).restype = C.c_int
        L.scmc_test_wait_fault.restype = C.c_int
        L.scmc_profile_read.argtypes = [C.POINTER(_abi.StageTimes), C.c_int32]
        for name in ("scmc_field", "scmc_field_device", "scmc_cov", "scmc_cov_device",
                     "scmc_export_records", "scmc_philox_stream", "scmc_profile_enable", "scmc_profile_read",
                     "scmc_fq_grid_size", "scmc_field_fourier_quad", "scmc_field_fourier_quad_device",
                     "scmc_field_noalloc", "scmc_cov_hetero", "scmc_field_hetero", "scmc_cov_hetero_device",
                     "scmc_field_hetero_device", "scmc_field_onwave", "scmc_field_onwave_device", "scmc_field_fourier_quad_onwave",
                     "scmc_field_fourier_quad_onwave_device", "scmc_refocus_grid", "scmc_refocus", "scmc_sample_cov", "scmc_field_from_records", "scmc_server_create",
                     "scmc_server_submit", "scmc_server_wait", "scmc_server_stats_read", "scmc_server_destroy"):
            getattr(L, name).restype = C.c_int
        _lib = L
        return _lib


def check(status: int) -> None:
    if status != 0:
        msg = lib().scmc_last_error().decode(errors="replace")
        raise ScmcError(status, msg or _STATUS.get(status, f"status {status}"))


def launch_count() -> int:
    return int(lib().scmc_launch_count())


def profile_enable(on: bool = True) -> None:
    check(lib().scmc_profile_enable(int(on)))


def profile_read(reset: bool = True) -> dict:
    t = _abi.StageTimes()
    check(lib().scmc_profile_read(C.byref(t), int(reset)))
    return t.as_dict()
