"""One Debye solve spread over the GPUs of a process group.

The tiles of a solve are independent: rank r of W runs every W-th tile in
cost order (pd_plan_set_shard), producing partial six-term profiles whose sum
over the ranks is the full result (rank 0 also carries the i = j terms and the
exact q = 0 sums). One all-reduce of 6·nq doubles over NCCL (NVLink /
NVSwitch) then gives every rank the full profiles. Coordinates and form-factor
tables are replicated — 16 bytes per atom.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _lib
from .debye import DebyeRequest


def tiles(req: DebyeRequest, rank: int = 0, world: int = 1,
          ctx: Optional[_lib.Context] = None) -> Tuple[np.ndarray, np.ndarray]:
    """Host-only: the [n, 5] tiles (i0, j0, j1, q-block, frame) of `rank`'s
    share and the padded-index -> atom permutation. No GPU needed."""
    lib = _lib.lib()
    r = req.c_struct()
    n, npad = C.c_uint64(), C.c_uint64()
    h = ctx.handle if ctx is not None else None
    _lib.check(lib.pd_plan_tiles(h, C.byref(r), rank, world, None, 0, C.byref(n), None, 0,
                                 C.byref(npad)), h)
    out = np.empty((n.value, 5), dtype=np.int32)
    perm = np.empty(npad.value, dtype=np.int32)
    _lib.check(lib.pd_plan_tiles(h, C.byref(r), rank, world,
                                 out.ctypes.data_as(C.POINTER(C.c_int32)), n.value, C.byref(n),
                                 perm.ctypes.data_as(C.POINTER(C.c_int32)), len(perm),
                                 C.byref(npad)), h)
    return out, perm


class ShardedPlan:
    """A plan restricted to this rank's tiles; `execute` returns the full
    terms after an all-reduce over `group` (torch.distributed)."""

    def __init__(self, req: DebyeRequest, ctx: _lib.Context, rank: int, world: int):
        self.req, self.ctx, self.rank, self.world = req, ctx, rank, world
        self._plan = C.c_void_p()
        lib = _lib.lib()
        r = req.c_struct()
        _lib.check(lib.pd_plan_create(ctx.handle, C.byref(r), C.byref(self._plan)), ctx.handle)
        _lib.check(lib.pd_plan_set_shard(ctx.handle, self._plan, rank, world), ctx.handle)

    @property
    def handle(self):
        return self._plan

    def execute_partial(self, xyz_dev, out_dev, stream_ptr) -> None:
        """Enqueue this rank's partial profiles into out_dev (device [6, nq])."""
        _lib.check(_lib.lib().pd_plan_execute(self.ctx.handle, self._plan, xyz_dev, out_dev,
                                              stream_ptr), self.ctx.handle)

    def execute(self, xyz_t, group=None):
        """Full terms on every rank: partial solve, then one SUM all-reduce."""
        import torch
        import torch.distributed as dist
        out = torch.empty((6, self.req.nq), dtype=torch.float64, device=xyz_t.device)
        self.execute_partial(xyz_t.data_ptr(), out.data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
        if self.world > 1:
            dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
        return out

    def close(self):
        if self._plan:
            _lib.lib().pd_plan_destroy(self.ctx.handle, self._plan)
            self._plan = C.c_void_p()
