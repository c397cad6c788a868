"""ctypes front end of the FP64 CPU oracle (debye_oracle.c).

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline legs of bench.py compare the backend against it. The product
path (pripps_b200) never imports it.

Every function restates the reference's f64 Debye code on the same inputs the
CUDA backend receives (see debye_oracle.c for the file:line map).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libdebye_oracle.so"

_D = C.POINTER(C.c_double)
_U32 = C.POINTER(C.c_uint32)
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.pdo_sinc.restype = C.c_double
        L.pdo_sinc.argtypes = [C.c_double]
        L.pdo_linear_q_values.restype = None
        L.pdo_linear_q_values.argtypes = [C.c_double, C.c_double, C.c_size_t, _D]
        L.pdo_self_intensity.restype = C.c_double
        L.pdo_self_intensity.argtypes = [_D, _D, C.c_size_t, C.c_double]
        L.pdo_cross_intensity.restype = C.c_double
        L.pdo_cross_intensity.argtypes = [_D, _D, C.c_size_t, _D, _D, C.c_size_t, C.c_double]
        L.pdo_combine.restype = C.c_double
        L.pdo_combine.argtypes = [_D, C.c_double, C.c_double]
        L.pdo_build_model.restype = C.c_int
        L.pdo_build_model.argtypes = [C.c_size_t, _D, _U32, C.c_size_t, _D, _D, _D, _D,
                                      C.c_double, C.c_double, C.c_size_t, _U32, C.c_size_t,
                                      C.c_int, C.c_int, _D]
        L.pdo_build_model_sets.restype = C.c_int
        L.pdo_build_model_sets.argtypes = [C.c_size_t, _D, _U32, _D, C.c_size_t, _D, _U32, _D,
                                           C.c_size_t, _D, _D, _D, C.c_double, C.c_double,
                                           C.c_size_t, _U32, C.c_size_t, C.c_int, C.c_int, _D]
        L.pdo_direct_rows.restype = None
        L.pdo_direct_rows.argtypes = [C.c_size_t, _D, _U32, _D, _D, C.c_size_t, _D, C.c_size_t,
                                      _D]
        L.pdo_vacuum.restype = C.c_int
        L.pdo_vacuum.argtypes = [C.c_size_t, _D, _U32, _D, C.c_double, C.c_double, C.c_size_t,
                                 _U32, C.c_size_t, C.c_int, C.c_int, _D]
        L.pdo_eval_gaussian.restype = C.c_double
        L.pdo_eval_gaussian.argtypes = [C.c_double, _D, _D, C.c_size_t, C.c_double]
        L.pdo_eval_polynomial.restype = C.c_double
        L.pdo_eval_polynomial.argtypes = [C.c_double, _D, C.c_size_t]
        L.pdo_interpolate.restype = C.c_double
        L.pdo_interpolate.argtypes = [_D, _D, C.c_size_t, C.c_double]
        L.pdo_fraser.restype = C.c_double
        L.pdo_fraser.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double]
        L.pdo_sasa_full_weight.restype = C.c_double
        L.pdo_sasa_full_weight.argtypes = [C.c_double, C.c_double]
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(_D)


def _c(a, dt=np.float64):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def sinc(x: float) -> float:
    return lib().pdo_sinc(float(x))


def linear_q_values(qmin, qmax, nq) -> np.ndarray:
    out = np.empty(nq)
    lib().pdo_linear_q_values(qmin, qmax, nq, _d(out))
    return out


def self_intensity(xyz, f, q) -> float:
    xyz, f = _c(xyz), _c(f)
    return lib().pdo_self_intensity(_d(xyz), _d(f), len(f), float(q))


def cross_intensity(axyz, af, bxyz, bf, q) -> float:
    axyz, af, bxyz, bf = _c(axyz), _c(af), _c(bxyz), _c(bf)
    return lib().pdo_cross_intensity(_d(axyz), _d(af), len(af), _d(bxyz), _d(bf), len(bf), float(q))


def build_model(xyz, species, ff_atoms, ff_excluded=None, hyd_weights=None, ff_water=None,
                qmin=0.0, qmax=0.5, nq=None, q_index=None, threads=0,
                precise=False) -> np.ndarray:
    """[len(q_index) or nq, 6] terms in DebyeTerms order (src/debye.rs:78-136).
    precise=True: the same sums with long double accumulators."""
    xyz = _c(xyz).reshape(-1, 3)
    species = _c(species, np.uint32)
    ff_atoms = _c(ff_atoms)
    nq = ff_atoms.shape[1] if nq is None else nq
    qi = None if q_index is None else _c(q_index, np.uint32)
    nqi = nq if qi is None else len(qi)
    out = np.empty((nqi, 6))
    rc = lib().pdo_build_model(len(species), _d(xyz), species.ctypes.data_as(_U32),
                               ff_atoms.shape[0], _d(ff_atoms), _d(_c(ff_excluded)),
                               _d(_c(hyd_weights)), _d(_c(ff_water)), qmin, qmax, nq,
                               None if qi is None else qi.ctypes.data_as(_U32), nqi, int(threads),
                               int(bool(precise)), _d(out))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return out


def build_model_sets(xyz, species, ff_atoms, exc_xyz=None, exc_kind=None, ff_excluded=None,
                     hyd_xyz=None, hyd_weights=None, ff_water=None, qmin=0.0, qmax=0.5,
                     nq=None, q_index=None, threads=0, precise=False) -> np.ndarray:
    """[len(q_index) or nq, 6] terms of build_model with the excluded-volume
    and hydration dummies at their own positions (src/debye.rs:83-130):
    excluded dummy i at exc_xyz[i] has form factor ff_excluded[exc_kind[i]],
    hydration dummy i at hyd_xyz[i] has hyd_weights[i]·ff_water."""
    xyz = _c(xyz).reshape(-1, 3)
    species = _c(species, np.uint32)
    ff_atoms = _c(ff_atoms)
    nq = ff_atoms.shape[1] if nq is None else nq
    n_exc = 0 if exc_xyz is None else len(exc_kind)
    n_hyd = 0 if hyd_xyz is None else len(hyd_weights)
    exc_xyz = None if n_exc == 0 else _c(exc_xyz).reshape(-1, 3)
    exc_kind = None if n_exc == 0 else _c(exc_kind, np.uint32)
    hyd_xyz = None if n_hyd == 0 else _c(hyd_xyz).reshape(-1, 3)
    hyd_w = None if n_hyd == 0 else _c(hyd_weights)
    qi = None if q_index is None else _c(q_index, np.uint32)
    nqi = nq if qi is None else len(qi)
    out = np.empty((nqi, 6))
    rc = lib().pdo_build_model_sets(
        len(species), _d(xyz), species.ctypes.data_as(_U32), _d(ff_atoms), n_exc, _d(exc_xyz),
        None if exc_kind is None else exc_kind.ctypes.data_as(_U32),
        _d(None if n_exc == 0 else _c(ff_excluded)), n_hyd, _d(hyd_xyz), _d(hyd_w),
        _d(None if n_hyd == 0 else _c(ff_water)), qmin, qmax, nq,
        None if qi is None else qi.ctypes.data_as(_U32), nqi, int(threads), int(bool(precise)),
        _d(out))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return out


def direct_rows(xyz, kind, ff, qvec, n_molecules=1, weight=None) -> np.ndarray:
    """[n_vec, 4] = (Re A, Im A, |A|², Σ_m |F_m|²) per q-vector
    (src/explicit.rs:208-230)."""
    xyz = _c(xyz).reshape(-1, 3)
    kind = _c(kind, np.uint32)
    ff = _c(ff)
    qvec = _c(qvec).reshape(-1, 3)
    out = np.empty((len(qvec), 4))
    lib().pdo_direct_rows(len(kind), _d(xyz), kind.ctypes.data_as(_U32),
                          _d(None if weight is None else _c(weight)), _d(ff), len(qvec),
                          _d(qvec), int(n_molecules), _d(out))
    return out


def vacuum(xyz, species, ff_atoms, qmin=0.0, qmax=0.5, nq=None, q_index=None,
           threads=0, precise=False) -> np.ndarray:
    xyz = _c(xyz).reshape(-1, 3)
    species = _c(species, np.uint32)
    ff_atoms = _c(ff_atoms)
    nq = ff_atoms.shape[1] if nq is None else nq
    qi = None if q_index is None else _c(q_index, np.uint32)
    nqi = nq if qi is None else len(qi)
    out = np.empty(nqi)
    rc = lib().pdo_vacuum(len(species), _d(xyz), species.ctypes.data_as(_U32), _d(ff_atoms),
                          qmin, qmax, nq, None if qi is None else qi.ctypes.data_as(_U32), nqi,
                          int(threads), int(bool(precise)), _d(out))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return out


def combine(t6, volume_scale, contrast_density) -> float:
    t6 = _c(t6)
    return lib().pdo_combine(_d(t6), float(volume_scale), float(contrast_density))


def eval_gaussian(q, ab, c) -> float:
    a = _c([x[0] for x in ab])
    b = _c([x[1] for x in ab])
    return lib().pdo_eval_gaussian(float(q), _d(a), _d(b), len(a), float(c))


def eval_polynomial(q, coeff) -> float:
    cf = _c(coeff)
    return lib().pdo_eval_polynomial(float(q), _d(cf), len(cf))


def interpolate(xs, ys, x) -> float:
    xs, ys = _c(xs), _c(ys)
    return lib().pdo_interpolate(_d(xs), _d(ys), len(xs), float(x))


def fraser(q, volume, rho, denominator) -> float:
    return lib().pdo_fraser(float(q), float(volume), float(rho), float(denominator))


def sasa_full_weight(radius, probe) -> float:
    return lib().pdo_sasa_full_weight(float(radius), float(probe))


def terms_for_request(req, q_index=None, threads=0, precise=False) -> np.ndarray:
    """Oracle terms [6, nq_sel] for a pripps_b200 DebyeRequest (one frame).
    Rows follow the C ABI order (DebyeTerms field order)."""
    if req.hyd_weights is None and req.ff_excluded is None:
        v = vacuum(req.xyz, req.species, req.ff_atoms, req.qmin, req.qmax, req.nq, q_index,
                   threads, precise)
        out = np.zeros((6, len(v)))
        out[0] = v
        return out
    t = build_model(req.xyz, req.species, req.ff_atoms, req.ff_excluded, req.hyd_weights,
                    req.ff_water, req.qmin, req.qmax, req.nq, q_index, threads, precise)
    return t.T.copy()
