"""Serving replicas across GPUs (pd_router_*): the routing policy on the CPU,
and on one GPU two replicas (two request loops sharing the device) whose
results equal the solo solve bit for bit, with work spread over both."""
import ctypes as C

import numpy as np
import pytest

from pripps_b200 import _lib, workloads
from pripps_b200.debye import solve


def choose(loads):
    arr = (C.c_double * len(loads))(*loads)
    k = C.c_uint32()
    assert _lib.lib().pd_route_choose(arr, len(loads), C.byref(k)) == _lib.PD_OK
    return k.value


def test_route_goes_to_least_pending_work():
    assert choose([0.0]) == 0
    assert choose([5e12, 1e12, 3e12]) == 1
    assert choose([2.0, 2.0, 1.0, 1.0]) == 2  # ties: lowest index
    assert choose([0.0, 0.0]) == 0


def test_route_rejects_empty():
    k = C.c_uint32()
    assert _lib.lib().pd_route_choose(None, 0, C.byref(k)) == _lib.PD_EINVAL


def test_router_needs_devices():
    r = C.c_void_p()
    assert _lib.lib().pd_router_create(None, 0, 0, C.byref(r)) == _lib.PD_EINVAL


@pytest.mark.gpu
def test_two_replicas_on_one_device_match_solo_solves():
    from pripps_b200.serving import Router
    reqs = [workloads.small_globule(n, 50 + n, nq=nq, qmax=0.6, solvent=(n % 2 == 0),
                                    precision="fp32").request
            for n, nq in [(4000, 200), (900, 64), (2500, 300), (1200, 100), (3100, 128),
                          (600, 40)]]
    router = Router([0, 0])
    try:
        tickets = [router.submit(r) for r in reqs]
        replicas = {router.replica(t) for t in tickets}
        outs = [router.wait(t, timeout_s=120) for t in tickets]
        # a ticket whose result was taken is gone from the router
        with pytest.raises(Exception):
            router.replica(tickets[0])
    finally:
        router.close()
    assert replicas == {0, 1}
    ctx = _lib.Context(0)  # a fresh context: the replicas' tuning table
    try:
        for r, o in zip(reqs, outs):
            assert np.array_equal(o, solve(r, ctx))
    finally:
        ctx.close()
