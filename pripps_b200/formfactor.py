"""Form factors F(q): the per-species inputs of the Debye sum.

Host-side restatement of the reference's runtime form-factor model and its
YAML resolver (src/formfactor.rs). The Debye kernels never evaluate a form
factor: the host tabulates F_s(q_k) for every species s on the request's q
grid (``FormFactorMap.table``) and ships the [species × nq] FP64 table with the
request, so ``QOutOfRange`` is raised here, before any device work, exactly as
the reference raises it inside ``formfactor_by_index``
(src/formfactor.rs:528-544).

Variants (src/formfactor.rs:137-156):
  Constant(c)              F = c
  Polynomial(qrange, c_i)  F = Σ c_i q^i                  (:378-385)
  Table([(q, F)...])       binary search + linear interp  (:388-408)
  Gaussian(qrange, ab, c)  F = c + Σ a_i exp(-b_i s²), s² = q²/(16π²)  (:368-375)
  SingleGaussian(a, b)     F = a exp(-b q²)               (:196)
Symbolic YAML variants resolved at load time (:560-698):
  !Alias name, !Linear [[name, w]...] (100-point table), !United {center,
  orbit: [[name, offset, weight?]...]} (101-point table over the centre's
  range, q_max capped at 2 Å⁻¹ when infinite).
"""
from __future__ import annotations

import bisect
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .errors import InternalError, QOutOfRange, UndefinedFormFactor, ValidationError

__all__ = [
    "FormFactor", "Constant", "Polynomial", "Table", "Gaussian", "SingleGaussian",
    "AtomKind", "FormFactorMap", "read_formfactors", "formfactors_from_yaml_str",
    "linear_q_values", "sinc",
]


def sinc(x: float) -> float:
    """sin(x)/x with 1 for |x| < 1e-8 (src/debye.rs:17-24)."""
    if abs(x) < 1e-8:
        return 1.0
    return math.sin(x) / x


def linear_q_values(qmin: float, qmax: float, nq: int) -> np.ndarray:
    """Inclusive uniform grid, denominator (nq-1).max(1) (src/q_sampler.rs:24-29)."""
    denom = float(max(nq - 1, 1))
    return np.array([qmin + (qmax - qmin) * i / denom for i in range(nq)], dtype=np.float64)


class FormFactor:
    """Runtime form factor; ``eval`` raises QOutOfRange outside ``qrange``."""

    def qrange(self) -> Tuple[float, float]:  # pragma: no cover - abstract
        raise NotImplementedError

    def _eval(self, q: float) -> float:  # pragma: no cover - abstract
        raise NotImplementedError

    def eval(self, q: float) -> float:
        lo, hi = self.qrange()
        if not (lo <= q <= hi):
            raise QOutOfRange(q, lo, hi)
        return self._eval(float(q))

    def to_table(self, qvalues) -> List[Tuple[float, float]]:
        return [(float(q), self.eval(q)) for q in qvalues]


@dataclass
class Constant(FormFactor):
    c: float

    def qrange(self):
        return (0.0, math.inf)

    def _eval(self, q):
        return self.c


@dataclass
class Polynomial(FormFactor):
    qrange_: Tuple[float, float]
    coeff: List[float]

    def qrange(self):
        return tuple(self.qrange_)

    def _eval(self, q):
        # Σ c_i q^i with q^i by repeated multiplication (Rust powi).
        total = 0.0
        for i, c in enumerate(self.coeff):
            p = 1.0
            for _ in range(i):
                p *= q
            total += c * p
        return total


@dataclass
class Table(FormFactor):
    points: List[Tuple[float, float]]

    def __post_init__(self):
        if len(self.points) < 2:
            raise ValidationError("a tabulated form factor needs at least two points")
        self._xs = [p[0] for p in self.points]
        self._ys = [p[1] for p in self.points]

    def qrange(self):
        return (self._xs[0], self._xs[-1])

    def _eval(self, q):
        xs, ys = self._xs, self._ys
        # Binary search as src/formfactor.rs:394-403: an exact hit returns the
        # tabulated value; otherwise `low` is the right end of the interval.
        low, high = 0, len(xs) - 1
        while low < high:
            mid = (low + high) // 2
            if q < xs[mid]:
                high = mid
            elif q > xs[mid]:
                low = mid + 1
            else:
                return ys[mid]
        x0, y0, x1, y1 = xs[low - 1], ys[low - 1], xs[low], ys[low]
        return y0 + (q - x0) * (y1 - y0) / (x1 - x0)


@dataclass
class Gaussian(FormFactor):
    qrange_: Tuple[float, float]
    ab: List[Tuple[float, float]]
    c: float

    def qrange(self):
        return tuple(self.qrange_)

    def _eval(self, q):
        s2 = q * q / (16.0 * math.pi * math.pi)
        total = 0.0
        for a, b in self.ab:
            total += a * math.exp(-b * s2)
        return total + self.c


@dataclass
class SingleGaussian(FormFactor):
    a: float
    b: float

    def qrange(self):
        return (0.0, math.inf)

    def _eval(self, q):
        return self.a * math.exp(-self.b * q * q)


@dataclass
class AtomKind:
    """Species record (src/atomkind.rs:25): the YAML ``radius`` is kept as
    sigma = 2r, and ``displaced_volume`` defaults to 4/3·π·r³ when absent
    (src/formfactor.rs:350-362)."""

    name: str
    sigma: Optional[float] = None
    displaced_volume: Optional[float] = None

    @property
    def radius(self) -> Optional[float]:
        return None if self.sigma is None else 0.5 * self.sigma


@dataclass
class _Entry:
    kind: AtomKind
    formfactor: FormFactor
    excluded_solvent: Optional[FormFactor] = None


@dataclass
class FormFactorMap:
    """Species table in id order; ids are positions (src/formfactor.rs:37-129).
    YAML-loaded maps are in name order, as the reference's BTreeMap is."""

    entries: List[_Entry] = field(default_factory=list)

    @classmethod
    def from_entries(cls, entries: Sequence[Tuple[AtomKind, FormFactor]]) -> "FormFactorMap":
        return cls([_Entry(k, f) for k, f in entries])

    def __len__(self):
        return len(self.entries)

    def kind(self, idx: int) -> AtomKind:
        return self.entries[idx].kind

    def kinds(self) -> List[AtomKind]:
        return [e.kind for e in self.entries]

    def form_factor(self, idx: int) -> FormFactor:
        return self.entries[idx].formfactor

    def excluded_solvent(self, idx: int) -> Optional[FormFactor]:
        return self.entries[idx].excluded_solvent

    def id_of(self, name: str) -> int:
        for i, e in enumerate(self.entries):
            if e.kind.name == name:
                return i
        raise ValidationError(f"unknown atom kind '{name}'")

    def form_factor_by_name(self, name: str) -> Optional[FormFactor]:
        for e in self.entries:
            if e.kind.name == name:
                return e.formfactor
        return None

    def table(self, ids: Sequence[int], q_values: np.ndarray, ctx=None,
              grid: Optional[Tuple[float, float, int]] = None) -> np.ndarray:
        """[len(ids) × nq] FP64 table of F_id(q_k). Only the listed ids are
        evaluated, so unused species with narrower q ranges never raise
        (src/formfactor.rs:520-544). With a device context and the uniform
        grid (qmin, qmax, nq) that q_values holds, the table is evaluated on
        the device (pd_formfactor_tables)."""
        if ctx is not None and grid is not None:
            return device_tables([self.entries[i].formfactor for i in ids], grid[0], grid[1],
                                 grid[2], ctx)
        out = np.empty((len(ids), len(q_values)), dtype=np.float64)
        for r, idx in enumerate(ids):
            ff = self.entries[idx].formfactor
            out[r] = [ff.eval(q) for q in q_values]
        return out


# ---------------------------------------------------------------- YAML specs

def _spec_from_tag(tag: str, value):
    """Convert one tagged YAML node into a (kind, payload) spec tuple."""
    name = tag.lstrip("!")
    if name in ("Constant", "Alias", "Table", "Linear"):
        return (name, value)
    if name in ("Polynomial", "Gaussian", "United"):
        return (name, dict(value))
    raise ValidationError(f"unknown form-factor tag '{tag}'")


def _make_loader():
    import yaml

    class _Loader(yaml.SafeLoader):
        pass

    def _multi(loader, tag_suffix, node):
        if isinstance(node, yaml.ScalarNode):
            value = loader.construct_scalar(node)
            if tag_suffix == "Constant":
                value = float(value)
        elif isinstance(node, yaml.SequenceNode):
            value = loader.construct_sequence(node, deep=True)
        else:
            value = loader.construct_mapping(node, deep=True)
        return _spec_from_tag(tag_suffix, value)

    _Loader.add_multi_constructor("!", _multi)
    return _Loader


def _spec_qrange(spec) -> Tuple[float, float]:
    kind, v = spec
    if kind == "Constant":
        return (0.0, math.inf)
    if kind in ("Gaussian", "Polynomial"):
        lo, hi = v["qrange"]
        return (float(lo), float(hi))
    if kind == "Table":
        return (float(v[0][0]), float(v[-1][0]))
    return (0.0, math.inf)  # unresolved symbolic variants


def _spec_to_runtime(spec) -> FormFactor:
    kind, v = spec
    if kind == "Constant":
        return Constant(float(v))
    if kind == "Polynomial":
        return Polynomial(tuple(float(x) for x in v["qrange"]), [float(c) for c in v["coeff"]])
    if kind == "Gaussian":
        return Gaussian(tuple(float(x) for x in v["qrange"]),
                        [(float(a), float(b)) for a, b in v["ab"]], float(v["c"]))
    if kind == "Table":
        return Table([(float(q), float(f)) for q, f in v])
    raise InternalError(f"unresolved {kind} form factor reached conversion boundary")


def _spec_eval(spec, q: float) -> float:
    lo, hi = _spec_qrange(spec)
    if not (lo <= q <= hi):
        raise QOutOfRange(q, lo, hi)
    return _spec_to_runtime(spec)._eval(q)


def _resolve(specs: Dict[str, dict], role: str) -> None:
    """Alias, then Linear, then United (src/formfactor.rs:560-564)."""

    def plain(kind_filter):
        return {n: s[role] for n, s in specs.items()
                if s.get(role) is not None and s[role][0] != kind_filter}

    # Alias (:618-640)
    table = plain("Alias")
    for n, s in specs.items():
        sp = s.get(role)
        if sp is not None and sp[0] == "Alias":
            if sp[1] not in table:
                raise UndefinedFormFactor(sp[1])
            s[role] = table[sp[1]]

    # Linear (:566-616): 100-point table over the intersection of ranges.
    table = plain("Linear")
    for n, s in specs.items():
        sp = s.get(role)
        if sp is None or sp[0] != "Linear":
            continue
        comps = [(str(c[0]), float(c[1])) for c in sp[1]]
        for cname, _ in comps:
            if cname not in table:
                raise UndefinedFormFactor(cname)
        qmin, qmax = 0.0, 2.0
        for cname, _ in comps:
            lo, hi = _spec_qrange(table[cname])
            qmin, qmax = max(lo, qmin), min(hi, qmax)
        pts = []
        for q in linear_q_values(qmin, qmax, 100):
            f = 0.0
            for cname, w in comps:
                f += w * _spec_eval(table[cname], float(q))
            pts.append((float(q), f))
        s[role] = ("Table", pts)

    # United (:642-698): 101 points over the centre's range.
    table = plain("United")
    for n, s in specs.items():
        sp = s.get(role)
        if sp is None or sp[0] != "United":
            continue
        center = sp[1]["center"]
        if center not in table:
            raise UndefinedFormFactor(center)
        cff = table[center]
        qmin, qmax = _spec_qrange(cff)
        if math.isinf(qmax):
            qmax = 2.0
        qs = [qmin + (qmax - qmin) * i / 100.0 for i in range(101)]
        pts = [[q, _spec_eval(cff, q)] for q in qs]
        for orbit in sp[1].get("orbit", []):
            oname, offset = str(orbit[0]), float(orbit[1])
            weight = float(orbit[2]) if len(orbit) > 2 and orbit[2] is not None else 1.0
            if oname not in table:
                raise UndefinedFormFactor(oname)
            for p in pts:
                p[1] += weight * _spec_eval(table[oname], p[0]) * sinc(p[0] * offset)
        s[role] = ("Table", [(p[0], p[1]) for p in pts])


def _finalize(raw: Dict[str, dict]) -> FormFactorMap:
    specs = {}
    for name, spec in raw.items():
        spec = dict(spec)
        if "ff" in spec and "formfactor" not in spec:
            spec["formfactor"] = spec.pop("ff")
        specs[str(name)] = spec
    _resolve(specs, "formfactor")
    _resolve(specs, "excluded_solvent")
    entries = []
    for name in sorted(specs):  # BTreeMap order = kind ids
        s = specs[name]
        radius = s.get("radius")
        dv = s.get("displaced_volume")
        if dv is None and radius is not None:
            dv = (4.0 / 3.0) * math.pi * (float(radius) ** 3)
        kind = AtomKind(name, None if radius is None else 2.0 * float(radius),
                        None if dv is None else float(dv))
        exc = s.get("excluded_solvent")
        entries.append(_Entry(kind, _spec_to_runtime(s["formfactor"]),
                              None if exc is None else _spec_to_runtime(exc)))
    return FormFactorMap(entries)


def formfactors_from_yaml_str(text: str) -> FormFactorMap:
    """Parse a form-factor YAML document (src/formfactor.rs:456-459)."""
    import yaml
    return _finalize(yaml.load(text, Loader=_make_loader()))


def read_formfactors(path) -> FormFactorMap:
    """Read a form-factor YAML file (src/formfactor.rs:446-454)."""
    with open(path, "r", encoding="utf-8") as fh:
        return formfactors_from_yaml_str(fh.read())


# ------------------------------------------------------ device evaluation
# Kind codes of pd_formfactor (include/pripps_debye.h).
PD_FF_CODES = {"Constant": 0, "Gaussian": 1, "SingleGaussian": 2, "Polynomial": 3, "Table": 4}


def device_descriptor(ff: FormFactor):
    """(type, n, qlo, qhi, params) of a runtime form factor for
    pd_formfactor_tables."""
    lo, hi = ff.qrange()
    if isinstance(ff, Constant):
        return 0, 1, lo, hi, [float(ff.c)]
    if isinstance(ff, Gaussian):
        return 1, len(ff.ab), lo, hi, [float(ff.c)] + [float(x) for ab in ff.ab for x in ab]
    if isinstance(ff, SingleGaussian):
        return 2, 1, lo, hi, [float(ff.a), float(ff.b)]
    if isinstance(ff, Polynomial):
        return 3, len(ff.coeff), lo, hi, [float(c) for c in ff.coeff]
    if isinstance(ff, Table):
        return 4, len(ff._xs), lo, hi, [float(x) for x in ff._xs] + [float(y) for y in ff._ys]
    raise ValidationError(f"form factor {type(ff).__name__} has no device form")


def device_tables(ffs: Sequence[FormFactor], qmin: float, qmax: float, nq: int, ctx) -> np.ndarray:
    """[len(ffs) × nq] F(q_k) on the uniform grid, evaluated on the device
    (pd_formfactor_tables); a grid point outside a form factor's range raises
    QOutOfRange, as FormFactor::eval does (src/formfactor.rs:188-193)."""
    import ctypes as C
    from . import _lib
    descs = (_lib.PdFormFactor * len(ffs))()
    keep = []
    for k, ff in enumerate(ffs):
        t, n, lo, hi, par = device_descriptor(ff)
        arr = np.ascontiguousarray(par, dtype=np.float64)
        keep.append(arr)
        descs[k].type, descs[k].n, descs[k].qlo, descs[k].qhi = t, n, lo, hi
        descs[k].params = _lib.dptr(arr)
    out = np.empty((len(ffs), int(nq)), dtype=np.float64)
    rc = _lib.lib().pd_formfactor_tables(ctx.handle, descs, len(ffs), float(qmin), float(qmax),
                                         int(nq), _lib.dptr(out))
    if rc == _lib.PD_EINVAL and "QOutOfRange" in _lib.last_error(ctx.handle):
        q = linear_q_values(qmin, qmax, nq)
        for ff in ffs:  # name the first failing point as the host evaluator would
            for x in q:
                ff.eval(float(x))
    _lib.check(rc, ctx.handle)
    return out
