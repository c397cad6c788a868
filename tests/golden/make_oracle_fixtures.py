"""Oracle fixtures of the solvent workloads, for the -m gpu parity tests.

    python tests/golden/make_oracle_fixtures.py sphere10k [--threads T]
    python tests/golden/make_oracle_fixtures.py ellipsoid100k [--threads T] [--q-index i,j,...]
    python tests/golden/make_oracle_fixtures.py sasa20k [--threads T]

Runs the FP64 CPU oracle in its compensated form (long double accumulators,
the reference's loop structure of src/debye.rs:214-250 otherwise) on the
seeded synthetic workloads of pripps_b200.workloads and writes, next to this
script:

  oracle_sphere_solvent_10k.json
      10,000 atoms in a 35 Å sphere, FoXS Fraser excluded volume and
      Bernoulli(0.35) surface hydration, q ∈ [0, 0.5], nq = 500: all six
      profiles on the whole grid (about 25 CPU-minutes per 8 cores);
  oracle_ellipsoid_solvent_100k.json
      100,000 atoms in an 80 × 40 × 40 Å prolate ellipsoid with the same
      solvent model, q ∈ [0, 1], nq = 1,000: all six profiles on a q subset
      (about 37 CPU-minutes per point on one core);
  oracle_ellipsoid_sasa_20k.json
      20,000 atoms at the same density with a continuous hydration weight per
      atom (the kernels' weighted mode), q ∈ [0, 1], nq = 512: all six
      profiles at q = 0, the small-q residual form, both sides of the first
      64-point q-block seam, every minimum of the atoms profile (95 … 503;
      located as for the 100k subset) and qmax.

Each fixture carries a SHA-256 digest of the request's inputs (positions,
species, form-factor tables, hydration weights), so a test can tell a
changed generator from a kernel error. The default 100k subset is
    0, 1, 2, 3          q = 0 and the small-q residual form
    72, 108             the first minima of the hydration and atoms profiles
    127, 128            the last point of the first 128-point q-block and the
                        first point of the next (the recurrence's longest run
                        and a fresh seed)
    186, 264, 500, 655  further minima of the atoms profile
    812, 894, 965       the deepest minima (965: I_atoms(q) = 4.9e-6·I_atoms(0))
    999                 qmax
(the minima were located with a pair-distance histogram of the same
structure, 0.002 Å bins).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

sys.path.insert(0, str(HERE.parent))

from conftest import request_digest  # noqa: E402
from oracle import oracle as O  # noqa: E402
from pripps_b200 import workloads  # noqa: E402

DEFAULT_100K = [0, 1, 2, 3, 72, 108, 127, 128, 186, 264, 500, 655, 812, 894, 965, 999]
DEFAULT_SASA20K = [0, 1, 2, 3, 63, 64, 95, 164, 231, 300, 372, 436, 503, 511]


def write(name: str, w, q_index, threads: int) -> Path:
    req = w.request
    t0 = time.time()
    terms = O.terms_for_request(req, q_index=q_index, threads=threads, precise=True)
    secs = time.time() - t0
    qi = list(range(req.nq)) if q_index is None else [int(i) for i in q_index]
    out = {
        "workload": w.name,
        "n_atoms": int(req.n_atoms),
        "qmin": req.qmin,
        "qmax": req.qmax,
        "nq": int(req.nq),
        "q_index": qi,
        "input_sha256": request_digest(req),
        "oracle": "compensated FP64 (long double accumulators), reference loop structure",
        "oracle_seconds": round(secs, 1),
        "oracle_threads": threads,
        "rows": ["atoms", "excluded", "hydration", "atom_excluded", "atom_hydration",
                 "excluded_hydration"],
        "oracle_terms": [[float(v) for v in row] for row in terms],
    }
    path = HERE / name
    path.write_text(json.dumps(out, indent=None) + "\n")
    return path


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("which", choices=["sphere10k", "ellipsoid100k", "sasa20k"])
    ap.add_argument("--threads", type=int, default=0, help="oracle threads (0: all cores)")
    ap.add_argument("--q-index", default=None,
                    help="comma-separated grid indices (ellipsoid100k only)")
    ap.add_argument("--append", action="store_true",
                    help="ellipsoid100k: add the points to an existing fixture of the same "
                         "inputs (the subset can be computed in several runs)")
    args = ap.parse_args(argv)
    if args.which == "sphere10k":
        w = workloads.sphere_solvent_10k("fp64")
        p = write("oracle_sphere_solvent_10k.json", w, None, args.threads)
    elif args.which == "sasa20k":
        w = workloads.ellipsoid_sasa_20k("fp64")
        p = write("oracle_ellipsoid_sasa_20k.json", w, np.array(DEFAULT_SASA20K), args.threads)
    else:
        qi = DEFAULT_100K if args.q_index is None else [int(s) for s in args.q_index.split(",")]
        w = workloads.ellipsoid_solvent_100k("fp64")
        name = "oracle_ellipsoid_solvent_100k.json"
        old = None
        if args.append and (HERE / name).exists():
            old = json.loads((HERE / name).read_text())
            if old["input_sha256"] != request_digest(w.request):
                sys.exit("the existing fixture was made from other inputs")
            qi = [i for i in qi if i not in old["q_index"]]
        p = write(name, w, np.array(qi), args.threads)
        if old is not None:
            new = json.loads(p.read_text())
            idx = old["q_index"] + new["q_index"]
            cols = [list(r_old) + list(r_new)
                    for r_old, r_new in zip(old["oracle_terms"], new["oracle_terms"])]
            order = np.argsort(idx, kind="stable")
            new["q_index"] = [idx[k] for k in order]
            new["oracle_terms"] = [[row[k] for k in order] for row in cols]
            new["oracle_seconds"] = round(old["oracle_seconds"] + new["oracle_seconds"], 1)
            p.write_text(json.dumps(new, indent=None) + "\n")
    print(p)


if __name__ == "__main__":
    main()
