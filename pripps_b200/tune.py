"""Build the kernel-shape tuning table on this machine's GPU.

    python -m pripps_b200.tune [--out pripps_b200/data/tuning_b200.txt] [--quick]

Runs the library's autotuner (pd_autotune_request: every instantiated shape,
timed after an L2 flush) on
  * the named workloads in their FP32 form: the 100,000-atom ellipsoid with
    solvent (nq 1,000), the 10,000-atom sphere with solvent (nq 500), the
    256-frame 5,000-atom trajectory (nq 300), the 1,000-atom vacuum sphere;
  * one synthetic solvent globule per bucket of a serving stream of 500 to
    50,000 atoms and 100 to 1,000 q points (floor(log2 N) 8..15 × floor(log2
    nq) 6..9), at the bucket's geometric middle, once with one hydration
    weight per element (class mode) and, from 2,048 atoms up, once with a
    continuous weight per atom as SASA areas give (weighted mode);
  * the 20,000-atom ellipsoid with per-atom weights (ellipsoid_sasa_20k);
and writes the table that pd_ctx_create loads (data/tuning_b200.txt beside
the library, or the file named by PRIPPS_DEBYE_TUNING).
"""
from __future__ import annotations

import argparse
import ctypes as C
import time
from pathlib import Path

import numpy as np

from . import _lib, workloads

DEFAULT_OUT = Path(__file__).resolve().parent / "data" / "tuning_b200.txt"


def tune(ctx: _lib.Context, req) -> tuple:
    r = req.c_struct()
    k, tj, np_, ms = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_double()
    _lib.check(_lib.lib().pd_autotune_request(ctx.handle, C.byref(r), C.byref(k), C.byref(tj),
                                              C.byref(np_), C.byref(ms)), ctx.handle,
               "pd_autotune_request")
    return (k.value, tj.value, np_.value), ms.value


def stream_buckets(quick: bool):
    for nb in range(8, 16):
        for qb in range(6, 10):
            n = int(round(2 ** (nb + 0.5)))
            nq = min(max(int(round(2 ** (qb + 0.5))), 100), 1000)
            if quick and (nb % 2 or qb % 2):
                continue
            yield n, nq


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=str(DEFAULT_OUT))
    ap.add_argument("--quick", action="store_true", help="every other stream bucket only")
    args = ap.parse_args(argv)
    ctx = _lib.Context(0)
    t0 = time.time()
    try:
        named = [workloads.sphere_vacuum_1k("fp32"), workloads.sphere_solvent_10k("fp32"),
                 workloads.trajectory_5k_256("fp32"), workloads.ellipsoid_sasa_20k("fp32"),
                 workloads.ellipsoid_solvent_100k("fp32")]
        rows = []
        for n, nq in stream_buckets(args.quick):
            w = workloads.small_globule(n, 1000 + n, nq=nq, qmax=0.6, solvent=True,
                                        precision="fp32")
            variants = [("class", w.request)]
            if n >= 2048:
                req = w.request
                rng = np.random.default_rng(n)
                req_w = workloads.DebyeRequest(
                    req.xyz, req.species, req.ff_atoms, req.ff_excluded,
                    req.hyd_weights * rng.uniform(0.05, 1.0, req.n_atoms), req.ff_water,
                    req.qmin, req.qmax, req.nq, None, req.precision)
                variants.append(("weighted", req_w))
            for label, req in variants:
                shape, ms = tune(ctx, req)
                rows.append((f"stream N={n} nq={nq} {label}", shape, ms))
                print(f"{rows[-1][0]:36s} K={shape[0]:3d} TJ={shape[1]:5d} NP={shape[2]} "
                      f"{ms:9.3f} ms", flush=True)
        # the named workloads last: their entries win where a bucket repeats
        for w in named:
            shape, ms = tune(ctx, w.request)
            rows.append((w.name, shape, ms))
            print(f"{w.name:36s} K={shape[0]:3d} TJ={shape[1]:5d} NP={shape[2]} {ms:9.3f} ms",
                  flush=True)
        _lib.check(_lib.lib().pd_tuning_save(ctx.handle, args.out.encode()), ctx.handle,
                   "pd_tuning_save")
    finally:
        ctx.close()
    print(f"wrote {args.out} ({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
