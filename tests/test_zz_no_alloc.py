"""pd_solve_noalloc: the solve for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc when they call in: a framework that owns
all device memory through its own allocator or reserved pool, a serving loop
where an allocation would synchronise the device, a plug-in inside a host
whose memory policy it does not control. pd_solve_noalloc serves them from a
fixed scratch array compiled into the library. These tests call it through
the C ABI and compare it with pd_solve, the allocating entry point, on the
same requests: several calls in a row on one device, each of a different
size, so that contents left in the shared scratch by the previous call would
show up in the next result. Both entry points run the same plan, kernels and
fixed-order reduction, so their results must agree bit for bit.

This file sorts last so that a run stopping at its first failure has run
every other test before it.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import term_errors
from pripps_b200 import _lib, workloads
from pripps_b200.debye import DebyeRequest, solve

def _noalloc(w, torch):
    """One pd_solve_noalloc call: device coordinates in, device terms out."""
    req = w.request
    lib = _lib.lib()
    xyz = torch.from_numpy(np.ascontiguousarray(req.xyz)).cuda()
    out = torch.full((6, req.nq), float("nan"), dtype=torch.float64, device="cuda")
    r = req.c_struct()
    r.xyz = None  # ignored by the entry point: the coordinates are xyz_dev
    rc = lib.pd_solve_noalloc(C.byref(r), C.c_void_p(xyz.data_ptr()),
                              C.c_void_p(out.data_ptr()),
                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc, None, "pd_solve_noalloc")
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.fixture
def default_ctx():
    """A context with the default kernel shapes, as pd_solve_noalloc uses."""
    ctx = _lib.Context(0)
    yield ctx
    ctx.close()


@pytest.mark.gpu
def test_noalloc_matches_pd_solve_on_consecutive_calls(default_ctx):
    torch = pytest.importorskip("torch")
    cases = [
        workloads.small_globule(1500, 11, nq=96, qmax=0.6, solvent=True, precision="fp32"),
        workloads.small_globule(700, 12, nq=40, qmax=0.5, solvent=False, precision="fp64"),
        workloads.small_globule(2600, 13, nq=150, qmax=0.8, solvent=True, precision="fp32"),
    ]
    # Two calls of the first case around the others: the second must not see
    # what the larger and smaller requests left in the scratch.
    for w in cases + cases[:1]:
        want = solve(w.request, default_ctx)
        got = _noalloc(w, torch)
        assert np.all(np.isfinite(got)), w.name
        assert np.array_equal(got, want), (w.name, term_errors(got, want))


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream():
    """The call uploads from host memory that lives only during the call, so
    a CUDA graph could not replay it: on a capturing stream it returns
    PD_EINVAL and enqueues nothing."""
    torch = pytest.importorskip("torch")
    w = workloads.small_globule(300, 5, nq=16, precision="fp32")
    xyz = torch.from_numpy(np.ascontiguousarray(w.request.xyz)).cuda()
    out = torch.zeros((6, 16), dtype=torch.float64, device="cuda")
    other = torch.zeros(4, device="cuda")
    torch.cuda.synchronize()
    r = w.request.c_struct()
    r.xyz = None
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.graph(g, stream=s):
        rc = _lib.lib().pd_solve_noalloc(C.byref(r), C.c_void_p(xyz.data_ptr()),
                                         C.c_void_p(out.data_ptr()),
                                         C.c_void_p(s.cuda_stream))
        other.add_(1.0)  # keeps the captured graph non-empty
    assert rc == _lib.PD_EINVAL
    assert "captured" in _lib.last_error(None)
    del g
    torch.cuda.synchronize()
    assert torch.all(out == 0)


@pytest.mark.gpu
def test_noalloc_trajectory_mean_matches_pd_solve(default_ctx):
    torch = pytest.importorskip("torch")
    w = workloads.trajectory_5k_256("fp32", n_frames=3)
    # a smaller structure keeps this quick; same frame logic
    req = w.request
    req.xyz = np.ascontiguousarray(req.xyz[:, :900])
    req.species = np.ascontiguousarray(req.species[:900])
    if req.hyd_weights is not None:
        req.hyd_weights = np.ascontiguousarray(req.hyd_weights[:900])
    want = solve(req, default_ctx)
    for _ in range(2):
        got = _noalloc(w, torch)
        assert np.array_equal(got, want), term_errors(got, want)


def test_noalloc_refuses_requests_beyond_the_scratch():
    """Host-side check, before any device work: no GPU needed."""
    rng = np.random.default_rng(3)
    n, nq = 200000, 1000
    req = DebyeRequest(rng.uniform(-60, 60, (n, 3)), rng.integers(0, 4, n).astype(np.uint32),
                       rng.uniform(1, 8, (4, nq)), rng.uniform(0.5, 2, (4, nq)),
                       np.where(rng.random(n) < 0.3, 1.2, 0.0), rng.uniform(5, 10, nq),
                       0.0, 1.0, nq, None, "fp32")
    r = req.c_struct()
    rc = _lib.lib().pd_solve_noalloc(C.byref(r), C.c_void_p(256), C.c_void_p(256), None)
    assert rc == _lib.PD_EBUDGET
    msg = _lib.last_error(None)
    assert str(_lib.PD_NOALLOC_SCRATCH_BYTES) in msg and "scratch" in msg, msg


def test_noalloc_size_guide_holds():
    """Host-only: the header's guide — at nq = 1,000 an FP32 solve of 100,000
    atoms with solvent and one hydration weight per element fits the fixed
    scratch and 200,000 atoms do not; with a weight per atom 20,000 atoms fit
    and 70,000 do not — checked on the layout the entry point computes with
    the shipped tuning table."""
    if os.environ.get("PRIPPS_DEBYE_TUNING"):
        pytest.skip("a tuning file other than the shipped one is in use")
    def need(n, nq, per_atom_weights=False):
        rng = np.random.default_rng(n)
        w = np.where(rng.random(n) < 0.3, 1.2, 0.0)
        if per_atom_weights:
            w = w * rng.uniform(0.05, 1.0, n)
        req = DebyeRequest(rng.uniform(-50, 50, (n, 3)), rng.integers(0, 4, n).astype(np.uint32),
                           rng.uniform(1, 8, (4, nq)), rng.uniform(0.5, 2, (4, nq)),
                           w, rng.uniform(5, 10, nq), 0.0, 0.5, nq, None, "fp32")
        r = req.c_struct()
        out = C.c_uint64()
        _lib.check(_lib.lib().pd_request_device_bytes(None, C.byref(r), 0, C.byref(out)), None,
                   "pd_request_device_bytes")
        return out.value
    assert need(100_000, 1000) <= _lib.PD_NOALLOC_SCRATCH_BYTES
    assert need(200_000, 1000) > _lib.PD_NOALLOC_SCRATCH_BYTES
    assert need(20_000, 1000, True) <= _lib.PD_NOALLOC_SCRATCH_BYTES
    assert need(70_000, 1000, True) > _lib.PD_NOALLOC_SCRATCH_BYTES


def test_noalloc_rejects_missing_buffers():
    w = workloads.small_globule(50, 3, nq=8)
    r = w.request.c_struct()
    assert _lib.lib().pd_solve_noalloc(C.byref(r), None, C.c_void_p(256), None) == _lib.PD_EINVAL
    assert _lib.lib().pd_solve_noalloc(None, C.c_void_p(256), C.c_void_p(256), None) == \
        _lib.PD_EINVAL
