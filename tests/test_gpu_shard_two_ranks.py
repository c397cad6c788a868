"""The tile-sharded solve on the GPU: two ranks, one device.

Each rank is its own process with its own CUDA context on cuda:0 and runs its
share of the solve's tiles (pd_plan_set_shard); the ranks add their partial
six-term profiles with one all-reduce over gloo on the host. The kernels of
the two ranks never wait on each other: only the host collective joins them,
so sharing one device changes their timing and nothing else. The all-reduced
profiles must equal the single-rank solve to FP64 rounding (the shares are
reduced in another association order), for the FP32 and the FP64 forms.
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, term_errors

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _request(precision):
    from pripps_b200 import workloads
    return workloads.small_globule(6000, 17, nq=300, precision=precision).request


def _worker(rank, world, port, precision, result_path):
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    from pripps_b200 import _lib, shard
    torch.cuda.set_device(0)
    ctx = _lib.Context(0)
    req = _request(precision)
    plan = shard.ShardedPlan(req, ctx, rank, world)
    try:
        xyz = torch.from_numpy(req.xyz).cuda()
        out = torch.empty((6, req.nq), dtype=torch.float64, device="cuda")
        plan.execute_partial(xyz.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        part = out.cpu()
    finally:
        plan.close()
    dist.all_reduce(part, op=dist.ReduceOp.SUM)
    if rank == 0:
        np.save(result_path, part.numpy())
    dist.barrier()
    dist.destroy_process_group()
    ctx.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_two_ranks_on_one_device_sum_to_the_single_rank_solve(tmp_path, gpu_ctx, precision):
    from pripps_b200.debye import solve
    path = str(tmp_path / "terms.npy")
    mp.start_processes(_worker, args=(2, _free_port(), precision, path), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(path)
    ref = solve(_request(precision), gpu_ctx)
    assert np.all(term_errors(got, ref) < 1e-12), term_errors(got, ref)


def _plan_info(plan):
    import ctypes as C
    from pripps_b200 import _lib
    tiles, dbytes = C.c_uint64(), C.c_uint64()
    _lib.check(_lib.lib().pd_plan_info(plan, None, None, None, C.byref(tiles), C.byref(dbytes),
                                       None), None)
    return tiles.value, dbytes.value


def test_shard_plans_hold_only_their_share(gpu_ctx):
    """A sharded plan keeps only its tiles' slots and lists: each of two
    shards holds less device memory than the whole plan, their partial
    profiles add up to the whole solve, and world = 1 restores the whole
    plan bit for bit."""
    import ctypes as C

    import torch

    from pripps_b200 import _lib
    lib = _lib.lib()
    req = _request("fp32")
    r = req.c_struct()
    xyz = torch.from_numpy(req.xyz).cuda()
    sp = torch.cuda.current_stream().cuda_stream

    def run(plan):
        out = torch.empty((6, req.nq), dtype=torch.float64, device="cuda")
        _lib.check(lib.pd_plan_execute(gpu_ctx.handle, plan, xyz.data_ptr(), out.data_ptr(), sp),
                   gpu_ctx.handle)
        torch.cuda.synchronize()
        return out.cpu().numpy()

    plans = []
    try:
        for _ in range(3):
            p = C.c_void_p()
            _lib.check(lib.pd_plan_create(gpu_ctx.handle, C.byref(r), C.byref(p)), gpu_ctx.handle)
            plans.append(p)
        whole = run(plans[2])
        tiles_all, bytes_all = _plan_info(plans[2])
        parts = []
        for rank in range(2):
            _lib.check(lib.pd_plan_set_shard(gpu_ctx.handle, plans[rank], rank, 2), gpu_ctx.handle)
            tiles, nbytes = _plan_info(plans[rank])
            assert tiles < tiles_all and nbytes < bytes_all
            parts.append(run(plans[rank]))
        assert np.all(term_errors(parts[0] + parts[1], whole) < 1e-12)
        _lib.check(lib.pd_plan_set_shard(gpu_ctx.handle, plans[0], 0, 1), gpu_ctx.handle)
        assert _plan_info(plans[0]) == (tiles_all, bytes_all)
        assert np.array_equal(run(plans[0]), whole)
    finally:
        for p in plans:
            lib.pd_plan_destroy(gpu_ctx.handle, p)
