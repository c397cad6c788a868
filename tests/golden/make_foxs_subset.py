"""Regenerate foxs_elements.yaml from the reference's FoXS form-factor asset.

    python tests/golden/make_foxs_subset.py /path/to/pripps/assets/foxs_formfactors.yaml

Writes pripps_b200/data/foxs_elements.yaml (the form-factor input of the
synthetic workloads).

Keeps the entries the synthetic workloads use — the C/N/O/S elements (their
Cromer–Mann Gaussians, radii and displaced volumes) and H2O with the H it is
built from — in the same tagged YAML form, so that
``pripps_b200.formfactor.read_formfactors`` resolves them exactly as the
reference's resolver does (H2O: United O + 2·H at 0.9584 Å).
"""
import sys
from pathlib import Path

import yaml

KEEP = ("C", "N", "O", "S", "H", "H2O")


def _loader():
    class L(yaml.SafeLoader):
        pass

    def multi(loader, suffix, node):
        if isinstance(node, yaml.ScalarNode):
            v = loader.construct_scalar(node)
        elif isinstance(node, yaml.SequenceNode):
            v = loader.construct_sequence(node, deep=True)
        else:
            v = loader.construct_mapping(node, deep=True)
        return (suffix, v)

    L.add_multi_constructor("!", multi)
    return L


def _flow(v):
    if isinstance(v, dict):
        return "{ " + ", ".join(f"{k}: {_flow(x)}" for k, x in v.items()) + " }"
    if isinstance(v, (list, tuple)):
        return "[" + ", ".join(_flow(x) for x in v) + "]"
    return repr(v) if isinstance(v, float) else str(v)


def main(src):
    raw = yaml.load(Path(src).read_text(), Loader=_loader())
    lines = ["# FoXS element form factors (Cromer-Mann Gaussians, s^2 = (q/4pi)^2),",
             "# radii and displaced volumes; H2O is the United O + 2 H form factor.",
             "# Generated by make_foxs_subset.py from the pripps FoXS asset.", ""]
    for name in KEEP:
        spec = raw[name]
        parts = []
        for key in ("radius", "displaced_volume"):
            if key in spec:
                parts.append(f"{key}: {spec[key]!r}")
        tag, val = spec.get("ff", spec.get("formfactor"))
        parts.append(f"ff: !{tag} {_flow(val)}")
        lines.append(f"{name}: {{ " + ", ".join(parts) + " }")
    out = Path(__file__).resolve().parents[2] / "pripps_b200" / "data" / "foxs_elements.yaml"
    out.write_text("\n".join(lines) + "\n")
    print(out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_foxs_subset.py /path/to/pripps/assets/foxs_formfactors.yaml")
    main(sys.argv[1])
