"""Failure path of the pair kernel's bounded waits, made to happen without
faulting or hanging the GPU.

The FP32 pair kernel stages atoms into shared memory with bulk copies and
waits for each on an mbarrier, giving up after a poll limit. The request flag
PD_FLAG_TEST_EXPIRED_WAIT makes the CTA that takes a launch's first tile wait
for a copy that is never issued, with a short limit, so the wait expires with
nothing in flight. The reference turns a lost device into Error::Internal
rather than a silent result (src/gpu.rs:577-621); here every blocking entry
point must return PD_ETIMEOUT, and the context must keep working.
"""
import ctypes as C

import numpy as np
import pytest

from pripps_b200 import _lib, workloads
from pripps_b200.debye import solve


def _flagged(req):
    r = req.c_struct()
    r.flags = _lib.PD_FLAG_TEST_EXPIRED_WAIT
    return r


def test_flag_passes_validation_and_others_do_not():
    """CPU: the test flag is accepted by the host checks; other bits are not."""
    w = workloads.small_globule(300, 2, nq=16)
    out = [C.c_uint64() for _ in range(4)]
    r = _flagged(w.request)
    assert _lib.lib().pd_plan_inspect(None, C.byref(r), *[C.byref(o) for o in out]) == _lib.PD_OK
    r.flags = 1
    assert _lib.lib().pd_plan_inspect(None, C.byref(r), *[C.byref(o) for o in out]) == \
        _lib.PD_EINVAL


@pytest.mark.gpu
def test_expired_wait_is_a_timeout_and_the_context_survives(gpu_ctx):
    w = workloads.small_globule(3000, 7, nq=64, qmax=0.6, precision="fp32")
    want = solve(w.request, gpu_ctx)
    lib = _lib.lib()
    out = np.zeros((6, 64))
    r = _flagged(w.request)
    rc = lib.pd_solve(gpu_ctx.handle, C.byref(r), _lib.dptr(out))
    assert rc == _lib.PD_ETIMEOUT, (rc, _lib.last_error(gpu_ctx.handle))
    assert "expired" in _lib.last_error(gpu_ctx.handle)
    assert np.isnan(out).any()  # the dead CTA's tiles are poisoned, not silently wrong
    # the context keeps working: the same request without the flag
    assert np.array_equal(solve(w.request, gpu_ctx), want)


@pytest.mark.gpu
def test_expired_wait_through_a_plan_and_the_request_loop():
    w = workloads.small_globule(2500, 9, nq=48, qmax=0.5, precision="fp32")
    lib = _lib.lib()
    ctx = _lib.Context(0)
    try:
        want = solve(w.request, ctx)
        r = _flagged(w.request)
        # plan: its host execution reports the expired wait
        plan = C.c_void_p()
        _lib.check(lib.pd_plan_create(ctx.handle, C.byref(r), C.byref(plan)), ctx.handle)
        out = np.zeros((6, 48))
        xyz = np.ascontiguousarray(w.request.xyz)
        rc = lib.pd_plan_execute_host(ctx.handle, plan, _lib.dptr(xyz), _lib.dptr(out))
        assert rc == _lib.PD_ETIMEOUT
        lib.pd_plan_destroy(ctx.handle, plan)
        # request loop: the flagged ticket fails; the loop serves the next one.
        # (One at a time: a CTA whose wait expired poisons every tile it takes
        # afterwards, whichever request they belong to, and flags each.)
        t_bad, t_good = C.c_uint64(), C.c_uint64()
        _lib.check(lib.pd_submit(ctx.handle, C.byref(r), C.byref(t_bad)), ctx.handle)
        bad = np.zeros((6, 48))
        assert lib.pd_wait(ctx.handle, t_bad, 60_000, _lib.dptr(bad)) == _lib.PD_ETIMEOUT
        r_ok = w.request.c_struct()
        _lib.check(lib.pd_submit(ctx.handle, C.byref(r_ok), C.byref(t_good)), ctx.handle)
        good = np.zeros((6, 48))
        assert lib.pd_wait(ctx.handle, t_good, 60_000, _lib.dptr(good)) == _lib.PD_OK
        assert np.array_equal(good, want)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_flag_has_no_effect_on_the_fp64_kernel(gpu_ctx):
    """The FP64 kernel stages nothing, so it has no copy wait to expire."""
    w = workloads.small_globule(400, 3, nq=16, precision="fp64")
    out = np.zeros((6, 16))
    r = _flagged(w.request)
    assert _lib.lib().pd_solve(gpu_ctx.handle, C.byref(r), _lib.dptr(out)) == _lib.PD_OK
    assert np.array_equal(out, solve(w.request, gpu_ctx))
