"""Request server: continuous batching of MCfield / MCcov solves.

A thin host wrapper over scmc_server_* in libscmc_gpu.so.  The server owns
worker slots, each with its own CUDA stream and scratch memory; submitted
requests are admitted FIFO when a slot is idle and their device-memory
estimate fits the HBM budget, and requests on different slots overlap on the
GPU.  A request is exactly one MCfield / MCcov call (MCfield.m:1, MCcov.m:1):
same arguments, same result as mc.field_from_args / mc.cov_from_args, alone
or in the mix.

    with Server(slots=8) as srv:
        t = srv.submit_field(mc.mc_args(...))
        u, info = srv.wait(t)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi, _lib
from ._abi import ArgsHolder


@dataclass
class Ticket:
    id: int
    kind: int
    shape: tuple
    out0: np.ndarray
    out1: np.ndarray | None


class Server:
    def __init__(self, device: int = 0, slots: int = 8, hbm_budget: float = 80e9):
        self._h = C.c_void_p()
        _lib.check(_lib.lib().scmc_server_create(int(device), int(slots), int(hbm_budget), C.byref(self._h)))
        self.device = device
        self._pending: dict[int, Ticket] = {}
        self._finished: dict[int, tuple] = {}

    # -- submission ---------------------------------------------------------
    def _submit(self, kind: int, h: ArgsHolder, want_ms=True, want_mm=True) -> Ticket:
        a = h.args
        dp = C.POINTER(C.c_double)
        if kind == _abi.SCMC_REQ_FIELD:
            shape = (a.nv, a.nl)
            out0 = np.zeros(2 * a.nv * a.nl)
            out1 = None
        else:
            shape = (a.nv, a.nv, a.nl, a.nl)
            n = 2 * a.nv * a.nv * a.nl * a.nl
            out0 = np.zeros(n) if want_ms else None
            out1 = np.zeros(n) if want_mm else None
        p0 = out0.ctypes.data_as(dp) if out0 is not None else None
        p1 = out1.ctypes.data_as(dp) if out1 is not None else None
        tid = C.c_int64()
        _lib.check(_lib.lib().scmc_server_submit(self._h, kind, h.ref, p0, p1, C.byref(tid)))
        t = Ticket(int(tid.value), kind, shape, out0, out1)
        self._pending[t.id] = t  # keeps the output arrays alive while the server writes them
        return t

    def submit_field(self, h: ArgsHolder) -> Ticket:
        return self._submit(_abi.SCMC_REQ_FIELD, h)

    def submit_cov(self, h: ArgsHolder, want_ms: bool = True, want_mm: bool = True) -> Ticket:
        return self._submit(_abi.SCMC_REQ_COV, h, want_ms, want_mm)

    # -- completion ---------------------------------------------------------
    def poll(self, t: Ticket) -> bool:
        """True once the request has finished (its result is then read by wait)."""
        info = _abi.RequestInfo()
        st = _lib.lib().scmc_server_wait(self._h, t.id, 0, C.byref(info))
        if st == _abi.SCMC_ERR_TIMEOUT and not info.finished:
            return False
        self._finished[t.id] = (st, info)
        return True

    def wait(self, t: Ticket, timeout_ms: int = -1):
        """(result, info dict).  result: u (field) or (Ms, Mm) (cov), shaped
        like mc.field_from_args / mc.cov_from_args; raises ScmcError on failure."""
        done = self._finished.pop(t.id, None)
        if done is None:
            info = _abi.RequestInfo()
            st = _lib.lib().scmc_server_wait(self._h, t.id, int(timeout_ms), C.byref(info))
            if st == _abi.SCMC_ERR_TIMEOUT and not info.finished:
                raise _lib.ScmcError(st, "request has not finished")
        else:
            st, info = done
        self._pending.pop(t.id, None)
        _lib.check(st)
        if t.kind == _abi.SCMC_REQ_FIELD:
            res = t.out0.view(np.complex128).reshape(t.shape, order="F")
        else:
            res = tuple(None if o is None else o.view(np.complex128).reshape(t.shape, order="F")
                        for o in (t.out0, t.out1))
        return res, info.as_dict()

    def stats(self) -> dict:
        s = _abi.ServerStats()
        _lib.check(_lib.lib().scmc_server_stats_read(self._h, C.byref(s)))
        return s.as_dict()

    def close(self):
        if self._h:
            _lib.check(_lib.lib().scmc_server_destroy(self._h))
            self._h = C.c_void_p()
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
