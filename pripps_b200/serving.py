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
