"""Test configuration: the `gpu` marker and shared helpers.

Tests marked `gpu` need an sm_100 device and call the CUDA backend through
its C ABI; everything else runs on the CPU (oracle, host logic, ABI exports).
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and the CUDA backend")


def load_golden(name):
    return json.loads((GOLDEN / name).read_text())


def request_digest(req) -> str:
    """SHA-256 of a DebyeRequest's inputs (positions, species, form-factor
    tables, hydration weights, grid): ties an oracle fixture to the exact
    inputs it was computed from."""
    h = hashlib.sha256()
    for a in (req.xyz, np.asarray(req.species).astype(np.uint32), req.ff_atoms,
              req.ff_excluded, req.hyd_weights, req.ff_water):
        if a is not None:
            h.update(np.ascontiguousarray(a, dtype=a.dtype).tobytes())
    h.update(np.array([req.qmin, req.qmax, req.nq], dtype=np.float64).tobytes())
    return h.hexdigest()


def term_errors(got, ref):
    """Per-row max error of a [6, nq] term table: relative for the self rows
    (atoms, excluded, hydration are >= 0); for the cross rows, which change
    sign, the error normalised by sqrt(self_a·self_b) (Cauchy–Schwarz bound of
    the cross term)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    err = np.zeros(6)
    pairs = {3: (0, 1), 4: (0, 2), 5: (1, 2)}
    for r in range(6):
        d = np.abs(got[r] - ref[r])
        if r < 3:
            scale = np.abs(ref[r])
        else:
            a, b = pairs[r]
            scale = np.sqrt(np.abs(ref[a] * ref[b]))
        mask = scale > 0
        if np.any(d[~mask] > 0):
            err[r] = np.inf
        if mask.any():
            err[r] = max(err[r], float(np.max(d[mask] / scale[mask])))
    return err


@pytest.fixture(scope="session")
def gpu_ctx():
    from pripps_b200 import _lib
    ctx = _lib.Context(0)
    yield ctx
    ctx.close()
