"""Kernel-shape tuning table: the file format, bucket keys and how a loaded
table reaches the plans. The file checks run on the CPU; the GPU tests load a
table into a context and check that solves, plans and pd_tuning_lookup use
its shape."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT
from pripps_b200 import _lib, workloads
from pripps_b200.debye import solve

SHIPPED = ROOT / "pripps_b200" / "data" / "tuning_b200.txt"


def check(path):
    n = C.c_uint64()
    rc = _lib.lib().pd_tuning_check(str(path).encode(), C.byref(n))
    return rc, n.value


def test_well_formed_file_parses(tmp_path):
    p = tmp_path / "t.txt"
    p.write_text("# comment\n"
                 "fp32 class single 16 9 128 16384 2 588.2\n"
                 "\n"
                 "fp32 weighted frames 12 8 64 1024 2 3.5  # trailing comment\n"
                 "fp64 class single 13 8 32 2048 1 0\n")
    assert check(p) == (_lib.PD_OK, 3)


@pytest.mark.parametrize("line", [
    "fp16 class single 16 9 128 16384 2 1",     # precision
    "fp32 klass single 16 9 128 16384 2 1",     # mode
    "fp32 class single 16 9 100 16384 2 1",     # q block not instantiated
    "fp32 class single 16 9 128 1000 2 1",      # j chunk not a multiple of 32
    "fp32 weighted single 16 9 128 4096 2 1",   # weighted mode stops at K = 64
    "fp64 class single 16 9 32 4096 2 1",       # FP64 runs one pair per pass
    "fp32 class single 16 9 128 16384 2",       # missing field
    "fp32 class single 16 9 128 16384 2 1 7",   # extra field
])
def test_malformed_line_is_rejected_with_its_number(tmp_path, line):
    p = tmp_path / "t.txt"
    p.write_text("fp32 class single 10 7 64 512 4 1.0\n" + line + "\n")
    rc, _ = check(p)
    assert rc == _lib.PD_EINVAL
    assert f"{p}:2" in _lib.last_error(None)


def test_missing_file():
    assert check("/nonexistent/tuning.txt")[0] == _lib.PD_ENOTFOUND


def test_shipped_table_parses():
    if not SHIPPED.exists():
        pytest.skip("no shipped tuning table")
    rc, n = check(SHIPPED)
    assert rc == _lib.PD_OK and n > 0


def lookup(req, ctx=None):
    r = req.c_struct()
    k, tj, np_, tab = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_int()
    _lib.check(_lib.lib().pd_tuning_lookup(ctx, C.byref(r), C.byref(k), C.byref(tj),
                                           C.byref(np_), C.byref(tab)), ctx, "pd_tuning_lookup")
    return (k.value, tj.value, np_.value), bool(tab.value)


def test_lookup_without_context_uses_the_shipped_table():
    """Without a context the lookup uses the table a new context would load:
    the shipped file's entry for a tuned bucket, the default shape for a
    bucket the file does not name."""
    if os.environ.get("PRIPPS_DEBYE_TUNING") or not SHIPPED.exists():
        pytest.skip("no shipped table in use")
    entries = {}
    for line in SHIPPED.read_text().splitlines():
        f = line.split("#")[0].split()
        if f:
            entries[tuple(f[:5])] = (int(f[5]), int(f[6]), int(f[7]))
    w = workloads.small_globule(5000, 1, nq=300)  # 2^12 <= 5,000 < 2^13, 2^8 <= 300 < 2^9
    key = ("fp32", "class", "single", "12", "8")
    shape, from_table = lookup(w.request)
    assert from_table == (key in entries)
    if from_table:
        assert shape == entries[key]
    w64 = workloads.small_globule(5000, 1, nq=300, precision="fp64")
    if ("fp64", "class", "single", "12", "8") not in entries:
        shape64, tab64 = lookup(w64.request)
        assert not tab64 and shape64[2] == 1  # the FP64 kernel runs one pair per pass


def test_weighted_default_is_a_weighted_kernel_shape():
    """A weighted-mode request (a distinct hydration weight per atom) in a
    bucket no table names gets a shape the weighted kernels have — the one
    its plan runs — not the class-mode default."""
    if os.environ.get("PRIPPS_DEBYE_TUNING"):
        pytest.skip("a tuning file other than the shipped one is in use")
    w = workloads.small_globule(300, 7, nq=300)  # 2^8 <= 300 < 2^9: no weighted entry
    req = w.request
    req.hyd_weights = np.linspace(0.1, 2.0, req.n_atoms)
    shape, from_table = lookup(req)
    assert not from_table
    assert (shape[0], shape[2]) in {(32, 2), (64, 2), (64, 4)}


@pytest.mark.gpu
def test_loaded_table_drives_solves_and_plans(tmp_path):
    """A table entry for the request's bucket is what a plan gets, and the
    solve under that shape still matches the default-shape solve."""
    w = workloads.small_globule(5000, 4, nq=300, qmax=0.6, solvent=True, precision="fp32")
    p = tmp_path / "tune.txt"
    # 5,000 atoms -> log2 12; nq 300 -> log2 8; solvent with one weight per
    # element -> class mode
    p.write_text("fp32 class single 12 8 96 512 2 1.0\n")
    ctx = _lib.Context(0)
    try:
        assert lookup(w.request, ctx.handle) == lookup(w.request)
        ref = solve(w.request, ctx)
        _lib.check(_lib.lib().pd_tuning_load(ctx.handle, str(p).encode()), ctx.handle)
        assert lookup(w.request, ctx.handle) == ((96, 512, 2), True)
        plan = C.c_void_p()
        r = w.request.c_struct()
        _lib.check(_lib.lib().pd_plan_create(ctx.handle, C.byref(r), C.byref(plan)), ctx.handle)
        k, tj, np_ = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _lib.check(_lib.lib().pd_plan_info(plan, C.byref(k), C.byref(tj), C.byref(np_), None,
                                           None, None), None)
        _lib.lib().pd_plan_destroy(ctx.handle, plan)
        assert (k.value, tj.value, np_.value) == (96, 512, 2)
        from conftest import term_errors
        assert np.all(term_errors(solve(w.request, ctx), ref) < 1e-5)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_autotune_request_saves_to_the_environment_file(tmp_path, monkeypatch):
    """With PRIPPS_DEBYE_TUNING set, a context loads that file and the
    autotuner writes its result there; a new context then uses it."""
    p = tmp_path / "tune.txt"
    monkeypatch.setenv("PRIPPS_DEBYE_TUNING", str(p))
    w = workloads.small_globule(3000, 5, nq=200, qmax=0.5, solvent=True, precision="fp32")
    ctx = _lib.Context(0)
    try:
        r = w.request.c_struct()
        k, tj, np_, ms = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_double()
        _lib.check(_lib.lib().pd_autotune_request(ctx.handle, C.byref(r), C.byref(k), C.byref(tj),
                                                  C.byref(np_), C.byref(ms)), ctx.handle)
        assert ms.value > 0
    finally:
        ctx.close()
    assert check(p) == (_lib.PD_OK, 1)
    ctx2 = _lib.Context(0)
    try:
        assert lookup(w.request, ctx2.handle) == ((k.value, tj.value, np_.value), True)
    finally:
        ctx2.close()
