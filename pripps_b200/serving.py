"""Client of the continuous-batching request loop (pd_submit / pd_wait).

Requests are copied at submission and admitted to the device as soon as the
context's memory budget allows; the tiles of every admitted request run
interleaved in each step of the device loop, so a request that arrives while
others are on the GPU starts without waiting for them to finish. Results are
independent of what ran beside them (per-request fixed-order reduction).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _lib
from .debye import DebyeRequest


class Server:
    def __init__(self, ctx: Optional[_lib.Context] = None):
        self.ctx = ctx or _lib.default_context()
        self._nq = {}

    def submit(self, req: DebyeRequest) -> int:
        r = req.c_struct()
        t = C.c_uint64()
        _lib.check(_lib.lib().pd_submit(self.ctx.handle, C.byref(r), C.byref(t)), self.ctx.handle)
        self._nq[t.value] = req.nq
        return t.value

    def poll(self, ticket: int) -> bool:
        rc = _lib.lib().pd_poll(self.ctx.handle, ticket)
        if rc < 0:
            _lib.check(rc, self.ctx.handle)
        return rc == 1

    def wait(self, ticket: int, timeout_s: Optional[float] = None) -> np.ndarray:
        out = np.empty((6, self._nq[ticket]), dtype=np.float64)
        ms = -1 if timeout_s is None else int(timeout_s * 1000)
        _lib.check(_lib.lib().pd_wait(self.ctx.handle, ticket, ms, _lib.dptr(out)),
                   self.ctx.handle)
        return out

    def cancel(self, ticket: int) -> None:
        _lib.check(_lib.lib().pd_cancel(self.ctx.handle, ticket), self.ctx.handle)

    def times(self, ticket: int) -> Tuple[float, float, float]:
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _lib.check(_lib.lib().pd_ticket_times(self.ctx.handle, ticket, C.byref(a), C.byref(b),
                                              C.byref(c)), self.ctx.handle)
        return a.value, b.value, c.value


class Router:
    """Serving replicas: one request loop per device (pd_router_*); each whole
    request goes to the replica with the least pending work."""

    def __init__(self, devices, mem_budget_bytes: int = 0):
        devs = (C.c_int * len(devices))(*devices)
        self._r = C.c_void_p()
        rc = _lib.lib().pd_router_create(devs, len(devices), int(mem_budget_bytes),
                                         C.byref(self._r))
        if rc != _lib.PD_OK:
            _lib.check(rc, None, _lib.lib().pd_router_last_error().decode())
        self._nq = {}

    def _check(self, rc):
        if rc != _lib.PD_OK:
            msg = _lib.lib().pd_router_last_error().decode()
            if rc == _lib.PD_EINVAL:
                raise _lib.ValidationError(msg)
            raise _lib.DeviceError(rc, msg)

    def submit(self, req: DebyeRequest) -> int:
        r = req.c_struct()
        t = C.c_uint64()
        self._check(_lib.lib().pd_router_submit(self._r, C.byref(r), C.byref(t)))
        self._nq[t.value] = req.nq
        return t.value

    def wait(self, ticket: int, timeout_s: Optional[float] = None) -> np.ndarray:
        out = np.empty((6, self._nq[ticket]), dtype=np.float64)
        ms = -1 if timeout_s is None else int(timeout_s * 1000)
        self._check(_lib.lib().pd_router_wait(self._r, ticket, ms, _lib.dptr(out)))
        return out

    def replica(self, ticket: int) -> int:
        k = C.c_uint32()
        self._check(_lib.lib().pd_router_replica(self._r, ticket, C.byref(k), None, None))
        return k.value

    def close(self) -> None:
        if self._r:
            _lib.lib().pd_router_destroy(self._r)
            self._r = C.c_void_p()
