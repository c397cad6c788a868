"""Generate the golden fixtures of the parity tests from the reference's test data.

    python tests/golden/make_golden.py /path/to/pripps

Reads (never at test time) the reference's lysozyme fixtures and assets:
  tests/lysozyme/4lzt.xyz        129 residue beads
  assets/poly_amino_acid.yaml    residue form factors (+ excluded_solvent)
  tests/lysozyme/pepsi.out/.log  PEPSI-SAXS I_at column and its intensity scale
and writes small JSON fixtures next to this script:

  pepsi_4lzt.json  positions, species (compact ids), the form-factor table on
                   the PEPSI q grid, the unscaled PEPSI I_at profile, the
                   reference test's tolerance (max rel < 0.04,
                   src/lib.rs:808-854), and the oracle's vacuum Debye profile
                   on the same inputs;
  solvent_4lzt.json  the same beads with the per-kind excluded solvent of
                   poly_amino_acid.yaml and a deterministic hydration weight
                   per bead, q ∈ [0, 0.3], nq = 20, with the oracle's six terms.

The form-factor tables are produced by pripps_b200.formfactor (the resolver
under test) and cross-checked against the oracle's C restatement of the
reference's polynomial evaluation before they are written.
"""
import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from pripps_b200.formfactor import Polynomial, linear_q_values, read_formfactors  # noqa: E402
from pripps_b200.structure import parse_xyz  # noqa: E402


def pepsi_scale(log_text):
    for line in log_text.splitlines():
        if "Intensity scaling" in line:
            return float(line.split()[-1])
    raise SystemExit("no intensity scaling in pepsi.log")


def pepsi_iat(out_text, scale):
    rows = []
    for line in out_text.splitlines():
        t = line.strip()
        if not t or t.startswith("#"):
            continue
        f = t.split()
        rows.append((float(f[0]), float(f[2]) / scale))
    return rows


def main(ref):
    ref = Path(ref)
    ffmap = read_formfactors(ref / "assets/poly_amino_acid.yaml")
    atoms = parse_xyz((ref / "tests/lysozyme/4lzt.xyz").read_text())
    names = {k.name: i for i, k in enumerate(ffmap.kinds())}
    ids = np.array([names[n] for n, _ in atoms])
    pos = np.array([p for _, p in atoms], dtype=np.float64)
    used = np.unique(ids)
    compact = np.searchsorted(used, ids)

    scale = pepsi_scale((ref / "tests/lysozyme/pepsi.log").read_text())
    prof = pepsi_iat((ref / "tests/lysozyme/pepsi.out").read_text(), scale)
    qmin, qmax, nq = prof[0][0], prof[-1][0], len(prof)
    qv = linear_q_values(qmin, qmax, nq)
    assert max(abs(a - b[0]) for a, b in zip(qv, prof)) < 1e-12
    table = ffmap.table(used, qv)
    # cross-check the resolver's polynomial evaluation against the oracle's
    for r, sid in enumerate(used):
        ff = ffmap.form_factor(int(sid))
        assert isinstance(ff, Polynomial)
        for k in (0, nq // 2, nq - 1):
            assert table[r, k] == O.eval_polynomial(qv[k], ff.coeff)
    vac = O.vacuum(pos, compact, table, qmin, qmax, nq)
    rel = max(abs(c - e) / e for c, e in zip(vac, (p[1] for p in prof)))
    print(f"oracle vs PEPSI I_at: max rel {rel:.4f} (reference bound 0.04)")
    json.dump({
        "source": "pripps tests/lysozyme/4lzt.xyz + assets/poly_amino_acid.yaml; "
                  "PEPSI I_at from tests/lysozyme/pepsi.out divided by the pepsi.log scale",
        "kinds": [ffmap.kind(int(i)).name for i in used],
        "positions": pos.tolist(), "species": compact.tolist(),
        "qmin": qmin, "qmax": qmax, "nq": nq, "ff_atoms": table.tolist(),
        "pepsi_iat": [p[1] for p in prof], "pepsi_rel_tol": 0.04,
        "oracle_vacuum": vac.tolist(),
    }, open(HERE / "pepsi_4lzt.json", "w"))

    # Solvent fixture: per-kind excluded solvent, deterministic weights.
    qmin2, qmax2, nq2 = 0.0, 0.3, 20
    qv2 = linear_q_values(qmin2, qmax2, nq2)
    ffA = ffmap.table(used, qv2)
    ffC = np.array([[ffmap.excluded_solvent(int(s)).eval(q) for q in qv2] for s in used])
    water = ffmap.form_factor_by_name("H2O")
    ffW = np.array([water.eval(q) for q in qv2])
    w = np.array([0.5 + 0.25 * math.sin(0.7 * i) ** 2 for i in range(len(ids))])
    w[::7] = 0.0  # buried beads
    terms = O.build_model(pos, compact, ffA, ffC, w, ffW, qmin2, qmax2, nq2).T
    json.dump({
        "source": "pripps tests/lysozyme/4lzt.xyz + assets/poly_amino_acid.yaml "
                  "(formfactor, excluded_solvent, H2O); weights 0.5+0.25 sin²(0.7 i), 0 for i%7==0",
        "positions": pos.tolist(), "species": compact.tolist(),
        "qmin": qmin2, "qmax": qmax2, "nq": nq2, "ff_atoms": ffA.tolist(),
        "ff_excluded": ffC.tolist(), "ff_water": ffW.tolist(), "hyd_weights": w.tolist(),
        "oracle_terms": terms.tolist(),
    }, open(HERE / "solvent_4lzt.json", "w"))
    print("wrote", HERE / "pepsi_4lzt.json", HERE / "solvent_4lzt.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/pripps (the reference checkout)")
    main(sys.argv[1])
