"""ctypes binding of libpripps_debye.so (declarations in include/pripps_debye.h).

The library is loaded from this package directory. There is no fallback: if
the shared object is missing the import of :func:`lib` raises, and every
device entry point fails with ``DeviceError`` when no sm_100 GPU is present.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from .errors import DeviceError, ValidationError

LIB_PATH = Path(__file__).resolve().parent / "libpripps_debye.so"

PD_OK = 0
PD_EINVAL = -1
PD_ENOMEM = -2
PD_EBUDGET = -3
PD_ETIMEOUT = -4
PD_EDEVICE = -5
PD_ENOTFOUND = -6
PD_ECANCELED = -7
PD_ENODEV = -8

PD_FLAG_TEST_EXPIRED_WAIT = 0x80000000

PD_FP32_FP64RED = 0
PD_FP64 = 1
PRECISIONS = {"fp32": PD_FP32_FP64RED, "fp64": PD_FP64}


class PdLattice(C.Structure):
    _fields_ = [
        ("species", C.c_uint32),
        ("reserved", C.c_uint32),
        ("origin", C.c_double * 3),
        ("spacing", C.c_double),
        ("extent", C.c_uint32 * 3),
        ("reserved2", C.c_uint32),
    ]


class PdFormFactor(C.Structure):
    _fields_ = [
        ("type", C.c_uint32),
        ("n", C.c_uint32),
        ("qlo", C.c_double),
        ("qhi", C.c_double),
        ("params", C.POINTER(C.c_double)),
    ]


class PdDirectRequest(C.Structure):
    _fields_ = [
        ("n_points", C.c_uint64),
        ("xyz", C.POINTER(C.c_double)),
        ("kind", C.POINTER(C.c_uint32)),
        ("n_kinds", C.c_uint32),
        ("reserved", C.c_uint32),
        ("ff", C.POINTER(C.c_double)),
        ("n_vectors", C.c_uint64),
        ("qvec", C.POINTER(C.c_double)),
        ("n_molecules", C.c_uint64),
        ("weight", C.POINTER(C.c_double)),
    ]


class PdRequest(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_uint64),
        ("xyz", C.POINTER(C.c_double)),
        ("species", C.POINTER(C.c_uint32)),
        ("n_species", C.c_uint32),
        ("precision", C.c_uint32),
        ("ff_atoms", C.POINTER(C.c_double)),
        ("ff_excluded", C.POINTER(C.c_double)),
        ("hyd_weights", C.POINTER(C.c_double)),
        ("ff_water", C.POINTER(C.c_double)),
        ("qmin", C.c_double),
        ("qmax", C.c_double),
        ("nq", C.c_uint64),
        ("n_frames", C.c_uint64),
        ("frame_weights", C.POINTER(C.c_double)),
        ("flags", C.c_uint32),
        ("n_lattices", C.c_uint32),
        ("lattices", C.POINTER(PdLattice)),
    ]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_U64P = C.POINTER(C.c_uint64)
_U32P = C.POINTER(C.c_uint32)

# name -> (restype, argtypes); the exact set include/pripps_debye.h declares.
SIGNATURES = {
    "pd_ctx_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_P)]),
    "pd_ctx_destroy": (None, [_P]),
    "pd_solve": (C.c_int, [_P, C.POINTER(PdRequest), _D]),
    "pd_plan_create": (C.c_int, [_P, C.POINTER(PdRequest), C.POINTER(_P)]),
    "pd_plan_execute": (C.c_int, [_P, _P, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pd_plan_execute_host": (C.c_int, [_P, _P, _D, _D]),
    "pd_plan_info": (C.c_int, [_P, _U32P, _U32P, _U32P, _U64P, _U64P, _U64P]),
    "pd_plan_set_profiling": (C.c_int, [_P, _P, C.c_int]),
    "pd_plan_pair_kernel_ms": (C.c_int, [_P, _P, _D, _U64P]),
    "pd_plan_destroy": (None, [_P, _P]),
    "pd_plan_set_shard": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32]),
    "pd_plan_tiles": (C.c_int, [_P, C.POINTER(PdRequest), C.c_uint32, C.c_uint32,
                                C.POINTER(C.c_int32), C.c_uint64, _U64P, C.POINTER(C.c_int32),
                                C.c_uint64, _U64P]),
    "pd_submit": (C.c_int, [_P, C.POINTER(PdRequest), _U64P]),
    "pd_wait": (C.c_int, [_P, C.c_uint64, C.c_int, _D]),
    "pd_poll": (C.c_int, [_P, C.c_uint64]),
    "pd_cancel": (C.c_int, [_P, C.c_uint64]),
    "pd_ticket_times": (C.c_int, [_P, C.c_uint64, _D, _D, _D]),
    "pd_combine": (C.c_int, [_D, C.c_uint64, C.c_double, C.c_double, _D]),
    "pd_last_error": (C.c_char_p, [_P]),
    "pd_get_tuning": (C.c_int, [_P, C.c_uint64, C.c_uint64, C.c_uint32, _U32P, _U32P, _U32P]),
    "pd_set_tuning": (C.c_int, [_P, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_uint32]),
    "pd_autotune": (C.c_int, [_P, C.c_uint64, C.c_uint64, C.c_uint32]),
    "pd_autotune_request": (C.c_int, [_P, C.POINTER(PdRequest), _U32P, _U32P, _U32P, _D]),
    "pd_tuning_lookup": (C.c_int, [_P, C.POINTER(PdRequest), _U32P, _U32P, _U32P,
                                   C.POINTER(C.c_int)]),
    "pd_tuning_load": (C.c_int, [_P, C.c_char_p]),
    "pd_tuning_save": (C.c_int, [_P, C.c_char_p]),
    "pd_tuning_check": (C.c_int, [C.c_char_p, _U64P]),
    "pd_plan_inspect": (C.c_int, [_P, C.POINTER(PdRequest), _U64P, _U64P, _U64P, _U64P]),
    "pd_request_device_bytes": (C.c_int, [_P, C.POINTER(PdRequest), C.c_int, _U64P]),
    "pd_measure_fp32_peak": (C.c_int, [_P, _D, _D]),
    "pd_launch_count": (C.c_uint64, [_P]),
    "pd_router_create": (C.c_int, [C.POINTER(C.c_int), C.c_uint32, C.c_uint64, C.POINTER(_P)]),
    "pd_router_destroy": (None, [_P]),
    "pd_router_submit": (C.c_int, [_P, C.POINTER(PdRequest), _U64P]),
    "pd_router_wait": (C.c_int, [_P, C.c_uint64, C.c_int, _D]),
    "pd_router_poll": (C.c_int, [_P, C.c_uint64]),
    "pd_router_cancel": (C.c_int, [_P, C.c_uint64]),
    "pd_router_replica": (C.c_int, [_P, C.c_uint64, _U32P, C.POINTER(_P), _U64P]),
    "pd_route_choose": (C.c_int, [_D, C.c_uint32, _U32P]),
    "pd_router_last_error": (C.c_char_p, []),
    "pd_solve_noalloc": (C.c_int, [C.POINTER(PdRequest), C.c_void_p, C.c_void_p, C.c_void_p]),
    "pd_direct": (C.c_int, [_P, C.POINTER(PdDirectRequest), _D]),
    "pd_direct_lattice": (C.c_int, [_P, C.POINTER(PdDirectRequest), C.POINTER(C.c_int32), _D,
                                    _D]),
    "pd_formfactor_tables": (C.c_int, [_P, C.POINTER(PdFormFactor), C.c_uint32, C.c_double,
                                       C.c_double, C.c_uint64, _D]),
    "pd_stream_open": (C.c_int, [_P, C.POINTER(PdRequest), C.c_uint32, C.POINTER(_P)]),
    "pd_stream_push": (C.c_int, [_P, _P, _D, _D, C.c_uint64]),
    "pd_stream_finish": (C.c_int, [_P, _P, _D]),
}

# Size of the fixed device scratch behind pd_solve_noalloc.
PD_NOALLOC_SCRATCH_BYTES = 64 << 20

_lib = None


def lib() -> C.CDLL:
    """Load the library once. Raises if the shared object is missing: the
    package has no other implementation of the Debye sum."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing; build it with `python -m pripps_b200.build` "
                "(the CUDA backend is the only implementation)")
        handle = C.CDLL(str(LIB_PATH), mode=C.RTLD_GLOBAL)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def last_error(ctx=None) -> str:
    msg = lib().pd_last_error(ctx)
    return msg.decode() if msg else ""


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc == PD_OK:
        return
    msg = last_error(ctx) or what
    if rc == PD_EINVAL:
        raise ValidationError(msg)
    raise DeviceError(rc, msg)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_D) if a is not None else None


def u32ptr(a: np.ndarray):
    return a.ctypes.data_as(_U32P)


class Context:
    """Owns a pd_ctx on one CUDA device."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0):
        self._ctx = _P()
        check(lib().pd_ctx_create(int(device), int(mem_budget_bytes), C.byref(self._ctx)), None,
              "pd_ctx_create failed")
        self.device = device

    @property
    def handle(self):
        return self._ctx

    def close(self):
        if self._ctx:
            lib().pd_ctx_destroy(self._ctx)
            self._ctx = _P()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def launch_count(self) -> int:
        return int(lib().pd_launch_count(self._ctx))


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        dev = int(os.environ.get("PRIPPS_DEBYE_DEVICE", "0"))
        _default_ctx = Context(dev)
    return _default_ctx
