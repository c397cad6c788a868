"""The C-ABI library on the CPU: it loads, exports every declared symbol, and
its host-only entry points (validation, planning, combine) behave. No call
here touches a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O
from pripps_b200 import _lib, workloads
from pripps_b200.debye import DebyeRequest


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(pd_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_functions()
    assert len(names) >= 20, names
    for n in sorted(names):
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    # and the binding's table covers the same set
    assert names == set(_lib.SIGNATURES), names ^ set(_lib.SIGNATURES)


def _req(n=300, nq=37, solvent=True, seed=0, precision="fp32", weights_mode="class"):
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(-10, 10, (n, 3))
    sp = rng.integers(0, 4, n).astype(np.uint32)
    ffA = rng.uniform(1, 8, (4, nq))
    ffC = rng.uniform(0.5, 2, (4, nq)) if solvent else None
    if solvent:
        if weights_mode == "class":
            w = np.where(rng.random(n) < 0.4, 1.5, 0.0)
        else:
            w = rng.uniform(0, 2, n)
        fw = rng.uniform(5, 10, nq)
    else:
        w = fw = None
    return DebyeRequest(xyz, sp, ffA, ffC, w, fw, 0.0, 0.5, nq, None, precision)


def inspect(req, ctx=None):
    r = req.c_struct()
    out = [C.c_uint64() for _ in range(4)]
    rc = _lib.lib().pd_plan_inspect(ctx, C.byref(r), *[C.byref(o) for o in out])
    return rc, [o.value for o in out]


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 127, 128, 129, 300, 1000])
@pytest.mark.parametrize("solvent,mode", [(False, "class"), (True, "class"), (True, "weighted")])
def test_plan_covers_every_pair_once(n, solvent, mode):
    req = _req(n=n, solvent=solvent, weights_mode=mode)
    rc, (ncls, npad, ntiles, covered) = inspect(req)
    assert rc == 0, _lib.last_error()
    assert covered == n * (n - 1) // 2
    assert npad % 128 == 0 and npad >= n
    if mode == "weighted" and n > 100:
        assert ncls <= 4  # species only: weights vary per atom
    if n == 1:
        assert ntiles == 0


def test_plan_covers_pairs_for_workload_shapes():
    w = workloads.sphere_solvent_10k()
    rc, (ncls, npad, ntiles, covered) = inspect(w.request)
    assert rc == 0
    assert covered == w.pairs
    assert ncls == 8  # 4 species × {buried, exposed}


@pytest.mark.parametrize("n_keys", [1, 47, 48, 49, 200])
def test_atom_classes_follow_the_key_count(n_keys):
    """Classes are the distinct (species, hydration weight) keys while there
    are at most 48 of them, else the species present (weighted mode); -0.0
    and 0.0 are one weight."""
    rng = np.random.default_rng(n_keys)
    n = 3000
    req = _req(n=n, solvent=True, weights_mode="class")
    sp = rng.integers(0, 4, n).astype(np.uint32)
    keys = [(int(k % 4), 0.25 * (k // 4)) for k in range(n_keys)]
    pick = rng.integers(0, n_keys, n)
    pick[:n_keys] = np.arange(n_keys)  # every key present
    sp = np.array([keys[k][0] for k in pick], dtype=np.uint32)
    w = np.array([keys[k][1] for k in pick])
    w[(w == 0.0) & (rng.random(n) < 0.5)] = -0.0
    req.species, req.hyd_weights = sp, w
    rc, (ncls, npad, ntiles, covered) = inspect(req)
    assert rc == 0, _lib.last_error()
    assert covered == n * (n - 1) // 2
    expect = len(set(keys)) if len(set(keys)) <= 48 else len(set(sp.tolist()))
    assert ncls == expect


def test_validation_errors_before_any_device_work():
    base = _req(n=10, nq=5)
    bad = []
    r = _req(n=10, nq=5); r.xyz[3, 1] = np.nan; bad.append(r)
    r = _req(n=10, nq=5); r.species[2] = 9; bad.append(r)
    r = _req(n=10, nq=5); r.ff_atoms[0, 0] = np.inf; bad.append(r)
    r = _req(n=10, nq=5); r.qmin, r.qmax = 0.5, 0.1; bad.append(r)
    r = _req(n=10, nq=5); r.hyd_weights[0] = np.nan; bad.append(r)
    for r in bad:
        rc, _ = inspect(r)
        assert rc == _lib.PD_EINVAL
    s = base.c_struct()
    s.nq = 0
    out = [C.c_uint64() for _ in range(4)]
    assert _lib.lib().pd_plan_inspect(None, C.byref(s), *[C.byref(o) for o in out]) == _lib.PD_EINVAL
    s = base.c_struct()
    s.n_atoms = 0
    assert _lib.lib().pd_plan_inspect(None, C.byref(s), *[C.byref(o) for o in out]) == _lib.PD_EINVAL
    s = base.c_struct()
    s.flags = 1
    assert _lib.lib().pd_plan_inspect(None, C.byref(s), *[C.byref(o) for o in out]) == _lib.PD_EINVAL
    # frame weights that sum to zero are rejected (src/trajectory.rs:234-238)
    r = _req(n=10, nq=5)
    r.xyz = np.stack([r.xyz, r.xyz])
    r.frame_weights = np.array([1.0, -1.0])
    rc, _ = inspect(r)
    assert rc == _lib.PD_EINVAL
    # NULL request / NULL context on the device entry points
    assert _lib.lib().pd_solve(None, None, None) == _lib.PD_EINVAL
    assert _lib.lib().pd_poll(None, 1) == _lib.PD_EINVAL


def test_combine_matches_oracle():
    rng = np.random.default_rng(7)
    t = rng.normal(size=(6, 11))
    total = np.empty(11)
    assert _lib.lib().pd_combine(_lib.dptr(np.ascontiguousarray(t)), 11, 1.1, 0.04,
                                 _lib.dptr(total)) == 0
    for k in range(11):
        assert total[k] == O.combine(t[:, k].copy(), 1.1, 0.04)


def test_context_without_gpu_fails_loudly():
    """On a host without a GPU the backend refuses instead of computing on
    the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = C.c_void_p()
    rc = _lib.lib().pd_ctx_create(0, 0, C.byref(ctx))
    assert rc == _lib.PD_ENODEV
    assert _lib.last_error(None)
