"""Direct (explicit q-vector) transform of a periodic box on the B200.

Host mirror of the reference's DirectTransform and DirectModel
(src/explicit.rs): a box of side lengths L is sampled at reciprocal-lattice
vectors q = 2π·n/L (integer n), by default the 13 [100], [110], [111]
directions times p = 1..p_max (src/explicit.rs:46-60, :275-292). For each
vector the device (``pd_direct``) forms the amplitude
A(q) = Σ_j f_j(|q|)·e^{i q·r_j} in FP64 and, for a box of N identical
contiguous molecules, the self term Σ_m |F_m|²; here the rows are grouped by
|q| exactly as the reference does (1e-6 bins, mean per bin, sorted;
src/explicit.rs:372-405), giving I(q), the per-molecule form factor
P = self/N and the effective structure factor S_eff = I/self
(src/lib.rs:510-526). With a solvent model the atoms, excluded-volume dummies
and hydration dummies each get their amplitudes, cached in a DirectModel
that recombines |A − v·C + c·B|² per vector before grouping
(src/explicit.rs:296-357).

The q grids (src/q_grid.rs) are restated in QGrid: the Miller grid, and the
lattice grid of every reciprocal-lattice vector up to q_max in |q| bins
(exact shells, evenly spread subsets of large bins, spherical-Fibonacci
sampling of bins beyond ~20,000 vectors).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .debye import Contributions, Intensity
from .errors import UsageError, ValidationError
from .formfactor import FormFactorMap
from .solvent import SolventConfig, distinct_dummy_sets, excluded_table, sasa_weights
from .structure import Structure

# src/explicit.rs:46-60
MILLER_INDEX = np.array([
    [1, 0, 0], [0, 1, 0], [0, 0, 1],
    [1, 1, 0], [0, 1, 1], [1, 0, 1],
    [-1, 1, 0], [-1, 0, 1], [0, -1, 1],
    [1, 1, 1], [-1, 1, 1], [1, -1, 1], [1, 1, -1],
], dtype=np.int64)


def miller_indices(p_max: int) -> np.ndarray:
    """p·(h, k, l) for the 13 directions (outer) and p = 1..p_max (inner),
    src/explicit.rs:275-283."""
    return np.array([p * d for d in MILLER_INDEX for p in range(1, int(p_max) + 1)],
                    dtype=np.int64).reshape(-1, 3)


def q_vectors(indices: np.ndarray, box_sides) -> np.ndarray:
    """(2π·n) / L component-wise (to_directions + component_div,
    src/explicit.rs:286-292, :211)."""
    n = np.asarray(indices, dtype=np.float64).reshape(-1, 3)
    return (2.0 * math.pi * n) / np.asarray(box_sides, dtype=np.float64)


def q_bin(q: float) -> int:
    """round(q·1e6) with halves away from zero (src/explicit.rs:372-377)."""
    x = q * 1e6
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def average_by_qnorm(qs: np.ndarray, values: np.ndarray):
    """Mean of the rows of each |q| bin, bins sorted by their first q
    (average_by_qnorm, src/explicit.rs:379-405). values is [rows, C]."""
    groups = {}
    for r, q in enumerate(qs):
        groups.setdefault(q_bin(float(q)), []).append(r)
    out_q, out_v = [], []
    for rows in groups.values():
        acc = np.zeros(values.shape[1])
        for r in rows:
            acc = acc + values[r]
        out_q.append(float(qs[rows[0]]))
        out_v.append(acc / float(len(rows)))
    order = sorted(range(len(out_q)), key=lambda k: out_q[k])
    return np.array([out_q[k] for k in order]), np.array([out_v[k] for k in order])


def amplitudes(xyz: np.ndarray, kind: np.ndarray, ff: np.ndarray, qvec: Optional[np.ndarray],
               n_molecules: int = 1, weight: Optional[np.ndarray] = None,
               ctx: Optional[_lib.Context] = None, hkl: Optional[np.ndarray] = None,
               box=None) -> np.ndarray:
    """[n_vectors, 4] = (Re A, Im A, |A|², Σ_m |F_m|²): pd_direct at the
    q-vectors qvec, or, given integer lattice indices hkl and the box sides,
    pd_direct_lattice at q = 2π·hkl/box (per-point phase tables on the
    device, the reference's PhaseTable, src/explicit.rs:85-135)."""
    ctx = ctx or _lib.default_context()
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    kind = np.ascontiguousarray(kind, dtype=np.uint32)
    ff = np.ascontiguousarray(ff, dtype=np.float64)
    if hkl is not None:
        hkl = np.asarray(hkl).reshape(-1, 3)
        if np.any(np.abs(hkl) > np.iinfo(np.int32).max):
            raise ValidationError("lattice indices beyond the int32 range")
        hkl = np.ascontiguousarray(hkl, dtype=np.int32)
        box = np.ascontiguousarray(box, dtype=np.float64).reshape(3)
        n_vec = len(hkl)
    else:
        qvec = np.ascontiguousarray(qvec, dtype=np.float64).reshape(-1, 3)
        n_vec = len(qvec)
    w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
    r = _lib.PdDirectRequest()
    r.n_points = len(kind)
    r.xyz = _lib.dptr(xyz)
    r.kind = _lib.u32ptr(kind)
    r.n_kinds = int(ff.shape[0])
    r.reserved = 0
    r.ff = _lib.dptr(ff)
    r.n_vectors = n_vec
    r.qvec = _lib.dptr(qvec if hkl is None else None)
    r.n_molecules = int(n_molecules)
    r.weight = _lib.dptr(w)
    out = np.empty((n_vec, 4), dtype=np.float64)
    if hkl is None:
        _lib.check(_lib.lib().pd_direct(ctx.handle, C.byref(r), _lib.dptr(out)), ctx.handle)
    else:
        _lib.check(_lib.lib().pd_direct_lattice(
            ctx.handle, C.byref(r), hkl.ctypes.data_as(C.POINTER(C.c_int32)), _lib.dptr(box),
            _lib.dptr(out)), ctx.handle)
    return out


def _kind_table(used: np.ndarray, formfactors: FormFactorMap, qnorm: np.ndarray) -> np.ndarray:
    """[len(used), n_vec]: each species' form factor at each vector's |q|
    (eval_atom_form_factors, src/explicit.rs:360-370)."""
    return formfactors.table(used, qnorm)


class DirectModel:
    """Cached amplitudes of atoms, excluded volume and hydration per q-vector
    (src/explicit.rs:296-357)."""

    def __init__(self, qnorm: np.ndarray, a: np.ndarray, c: np.ndarray, b: np.ndarray):
        self._qnorm = np.asarray(qnorm, dtype=np.float64)
        self._a, self._c, self._b = a, c, b  # complex [n_vec]
        self._q_values, _ = average_by_qnorm(self._qnorm, np.zeros((len(self._qnorm), 1)))

    @property
    def q_values(self) -> np.ndarray:
        return self._q_values

    def intensity(self, volume_scale: float = 1.0, contrast_density: float = 0.03) -> Intensity:
        v, c = float(volume_scale), float(contrast_density)
        tot = self._a - v * self._c + c * self._b
        cols = np.stack([tot.real ** 2 + tot.imag ** 2,
                         self._a.real ** 2 + self._a.imag ** 2,
                         self._c.real ** 2 + self._c.imag ** 2,
                         self._b.real ** 2 + self._b.imag ** 2], axis=1)
        q, g = average_by_qnorm(self._qnorm, cols)
        return Intensity(q, g[:, 0], Contributions(g[:, 1], g[:, 2], g[:, 3]))


class DirectTransform:
    """I(q) of a periodic box at explicit q-vectors (src/explicit.rs:62-247)."""

    def __init__(self, formfactors: FormFactorMap, p_max: int = 6,
                 solvent: Optional[SolventConfig] = None, num_molecules: Optional[int] = None,
                 indices: Optional[np.ndarray] = None, ctx: Optional[_lib.Context] = None,
                 grid: Optional["QGrid"] = None):
        self.formfactors = formfactors
        self.grid = grid
        if grid is not None:
            self.indices = grid.indices()
        else:
            self.indices = (miller_indices(p_max) if indices is None
                            else np.asarray(indices, dtype=np.int64).reshape(-1, 3))
        self.solvent = solvent if (solvent is not None and solvent.is_active()) else None
        self.num_molecules = num_molecules
        self._ctx = ctx

    @property
    def ctx(self):
        return self._ctx or _lib.default_context()

    def calc_intensities(self, structure: Structure, box_sides) -> Intensity:
        if box_sides is None:
            raise UsageError("direct Fourier transform requires box side lengths on the structure")
        if self.grid is not None:
            self.grid.check_box(box_sides)
        qvec = q_vectors(self.indices, box_sides)
        qnorm = np.sqrt(np.sum(qvec * qvec, axis=1))
        if self.solvent is not None:
            return self.build_model(structure, box_sides).intensity(
                self.solvent.excluded.effective_volume_scale(),
                self.solvent.hydration.effective_contrast_density())
        used = np.unique(structure.ids)
        kind = np.searchsorted(used, structure.ids)
        ff = _kind_table(used, self.formfactors, qnorm)
        n = self.num_molecules or 1
        rows = amplitudes(structure.pos, kind, ff, None, n, ctx=self.ctx, hkl=self.indices,
                          box=box_sides)
        if self.grid is not None:
            q, g = self.grid.group(qnorm, rows[:, 2:4])
        else:
            q, g = average_by_qnorm(qnorm, rows[:, 2:4])
        out = Intensity(q, g[:, 0].copy())
        if self.num_molecules:
            self_term = g[:, 1]
            out.form_factor = self_term / float(n)
            out.effective_structure_factor = np.where(
                self_term > 0.0, g[:, 0] / np.where(self_term > 0.0, self_term, 1.0), np.nan)
        return out

    def build_model(self, structure: Structure, box_sides) -> DirectModel:
        """Amplitudes of the three sets per q-vector (src/explicit.rs:249-299),
        on the unit basis (the knobs are applied in DirectModel.intensity)."""
        cfg = self.solvent if self.solvent is not None else SolventConfig()
        qvec = q_vectors(self.indices, box_sides)
        qnorm = np.sqrt(np.sum(qvec * qvec, axis=1))
        used = np.unique(structure.ids)
        kind = np.searchsorted(used, structure.ids)
        ctx = self.ctx

        def amp(xyz, knd, table, weight=None):
            if len(knd) == 0:
                return np.zeros(len(qvec), dtype=np.complex128)
            r = amplitudes(xyz, knd, table, None, 1, weight, ctx, hkl=self.indices, box=box_sides)
            return r[:, 0] + 1j * r[:, 1]

        a = amp(structure.pos, kind, _kind_table(used, self.formfactors, qnorm))
        exc, hyd = distinct_dummy_sets(cfg, structure.pos, structure.ids, self.formfactors)
        if cfg.excluded.at_atoms():
            c = amp(structure.pos, kind, excluded_table(cfg.excluded.unit_scale(),
                                                        self.formfactors, used, qnorm,
                                                        cfg.bulk_electron_density))
        elif exc is not None:
            idx, rows = exc.rows(qnorm)
            c = amp(exc.positions, idx, rows)
        else:
            c = np.zeros(len(qvec), dtype=np.complex128)
        if cfg.hydration.at_atoms():
            w = sasa_weights(cfg.hydration, self.formfactors, structure.ids)
            water = self.formfactors.form_factor_by_name("H2O")
            table = np.array([[water.eval(float(q)) for q in qnorm]])
            b = amp(structure.pos, np.zeros(len(w), dtype=np.int64), table, w)
        elif hyd is not None:
            table = np.array([[hyd.form_factors[0].eval(float(q)) for q in qnorm]])
            b = amp(hyd.positions, np.zeros(len(hyd), dtype=np.int64), table, hyd.weights)
        else:
            b = np.zeros(len(qvec), dtype=np.complex128)
        return DirectModel(qnorm, a, c, b)


def check_num_molecules(structure: Structure, n: Optional[int], solvent_active: bool) -> None:
    """The reference's guards on --num-molecules (src/lib.rs:368-411)."""
    if n is None:
        return
    if n == 0:
        raise UsageError("--num-molecules must be at least 1")
    if solvent_active:
        raise UsageError("--num-molecules supports vacuum runs only (no excluded-volume/"
                         "hydration model)")
    if len(structure.pos) % n:
        raise ValidationError(f"box atom count ({len(structure.pos)}) is not a multiple of "
                              f"--num-molecules ({n})")
    m = len(structure.pos) // n
    ids = structure.ids
    if m > 0 and not all(np.array_equal(ids[k * m:(k + 1) * m], ids[:m]) for k in range(n)):
        raise ValidationError(f"--num-molecules {n} does not partition the box into {n} "
                              "identical contiguous molecules: the atom composition differs "
                              "between blocks")


# ------------------------------------------------------------------ q grids
EXACT_BIN_LIMIT = 20_000.0               # src/q_grid.rs:170-173
GOLDEN_ANGLE = 2.399_963_229_728_653     # src/q_grid.rs:306


def _round(x: float) -> int:
    """f64::round: halves away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def _bin_width(box) -> float:
    return 2.0 * math.pi / max(0.0, *box)


def _expected_count(box, k: int) -> float:
    """src/q_grid.rs:179-184"""
    width = _bin_width(box)
    volume = box[0] * box[1] * box[2]
    return 2.0 * math.pi * (k * width) ** 2 * width * volume / (2.0 * math.pi) ** 3


def _largest_exact_bin(box) -> int:
    k = 1
    while not _expected_count(box, k + 1) > EXACT_BIN_LIMIT:
        k += 1
    return k


def _upper_half(n) -> bool:
    h, k, l = n
    return h > 0 or (h == 0 and (k > 0 or (k == 0 and l > 0)))


def _norm(box, n) -> float:
    s = 0.0
    for a in range(3):
        s += (2.0 * math.pi * n[a] / box[a]) ** 2
    return math.sqrt(s)


def _exact_shells(box, q_max: float):
    """src/q_grid.rs:315-344: every upper-half lattice vector with
    |q| <= q_max in the exactly enumerated bins, grouped by bin."""
    width = _bin_width(box)
    last_exact = _largest_exact_bin(box)
    q_max = min(q_max, (last_exact + 0.5) * width)
    n_max = [int(math.floor(q_max * (1.0 + 1e-12) * l / (2.0 * math.pi))) for l in box]
    bins = {}
    for h in range(-n_max[0], n_max[0] + 1):
        for k in range(-n_max[1], n_max[1] + 1):
            for l in range(-n_max[2], n_max[2] + 1):
                n = (h, k, l)
                if not _upper_half(n):
                    continue
                q = _norm(box, n)
                b = _round(q / width)
                if q <= q_max * (1.0 + 1e-12) and b <= last_exact:
                    bins.setdefault(b, []).append((n, q))
    return [bins[b] for b in sorted(bins)]


def _direction_key(n) -> float:
    x, y, z = (float(c) for c in n)
    norm = math.sqrt(x * x + y * y + z * z)
    band = math.floor((z / norm + 1.0) * 8.0)
    return band * 10.0 + math.atan2(y, x)


def _spread_subset(shell, cap: int):
    """src/q_grid.rs:351-359"""
    if len(shell) <= cap:
        return list(shell)
    shell.sort(key=lambda v: _direction_key(v[0]))
    return [shell[i * len(shell) // cap] for i in range(cap)]


def _shell_holds(box, a, b, n) -> bool:
    length = _norm(box, n)
    return a <= length < b


def _shell_any_vector(box, a, b):
    """src/q_grid.rs:279-303"""
    step = [2.0 * math.pi / l for l in box]
    n_max = [int(math.floor(b / s)) for s in step]
    for h in range(0, n_max[0] + 1):
        for k in range(-n_max[1], n_max[1] + 1):
            planar = (h * step[0]) ** 2 + (k * step[1]) ** 2
            if planar >= b * b:
                continue
            l0 = int(math.ceil(math.sqrt(max(a * a - planar, 0.0)) / step[2]))
            for l in (l0 - 1, l0, l0 + 1):
                n = (h, k, l) if _upper_half((h, k, l)) else (-h, -k, -l)
                if _upper_half(n) and _shell_holds(box, a, b, n):
                    return n
    return None


def _sampled_shell(box, k: int, q_max: float, cap: int):
    """src/q_grid.rs:194-262: spherical-Fibonacci directions at radii uniform
    in the shell volume, snapped to the lattice and deduplicated."""
    width = _bin_width(box)
    a, b = (k - 0.5) * width, min((k + 0.5) * width, q_max)
    if b <= a:
        return None
    q = 0.75 * (b ** 4 - a ** 4) / (b ** 3 - a ** 3)
    sb = min((k + 0.5) * width, q_max * (1.0 + 1e-12))
    wanted = min(cap, int(EXACT_BIN_LIMIT))
    attempts = 2 * wanted + 16
    seen, vectors = set(), []
    for i in range(attempts):
        z = 1.0 - (2 * i + 1) / attempts
        sn, cs = math.sin(i * GOLDEN_ANGLE), math.cos(i * GOLDEN_ANGLE)
        rho = math.sqrt(1.0 - z * z)
        tt = i * 0.618_033_988_749_895
        t = tt - math.trunc(tt)
        r = math.cbrt(a ** 3 + t * (b ** 3 - a ** 3))
        direction = (rho * cs, rho * sn, z)
        n = tuple(_round(r * direction[ax] * box[ax] / (2.0 * math.pi)) for ax in range(3))
        if not _upper_half(n):
            n = tuple(-c for c in n)
        if _upper_half(n) and _shell_holds(box, a, sb, n) and n not in seen:
            seen.add(n)
            vectors.append(n)
    if not vectors:
        v = _shell_any_vector(box, a, sb)
        return None if v is None else (q, [v])
    m = min(wanted, len(vectors))
    return q, [vectors[i * len(vectors) // m] for i in range(m)]


class QGrid:
    """Which q-vectors a periodic box is sampled at (src/q_grid.rs): the 13
    Miller directions × p, or every reciprocal-lattice vector up to q_max in
    |q| bins of width 2π/max(L) (exact bins up to ~20,000 vectors, sampled
    beyond; bins over `max_per_bin` keep an evenly spread subset)."""

    def __init__(self, p_max: Optional[int] = None, box=None, vectors=None, bins=None, q=None):
        self.p_max, self.box = p_max, box
        self._vectors, self._bins, self._q = vectors, bins, q

    @classmethod
    def miller(cls, p_max: int) -> "QGrid":
        return cls(p_max=int(p_max))

    @classmethod
    def lattice(cls, box_sides, q_max: float, max_per_bin: int) -> "QGrid":
        box = [float(l) for l in box_sides]
        if not all(math.isfinite(l) and l > 0.0 for l in box):
            raise UsageError(f"invalid box sides {box}")
        if not (math.isfinite(q_max) and q_max > 0.0):
            raise UsageError(f"invalid q_max {q_max} Å⁻¹")
        shells = _exact_shells(box, float(q_max))
        if not shells:
            raise UsageError(f"q_max {q_max} Å⁻¹ is below the shortest lattice vector of box "
                             f"{box}")
        cap = max(int(max_per_bin), 1)
        vectors, bins, qs = [], [], []
        for shell in shells:
            q = sum(v[1] for v in shell) / len(shell)
            b = len(qs)
            qs.append(q)
            for n, _ in _spread_subset(shell, cap):
                vectors.append(n)
                bins.append(b)
        width = _bin_width(box)
        first_sampled = _largest_exact_bin(box) + 1
        last = _round(q_max / width)
        for k in range(first_sampled, last + 1):
            got = _sampled_shell(box, k, float(q_max), cap)
            if got is not None:
                b = len(qs)
                qs.append(got[0])
                for n in got[1]:
                    vectors.append(n)
                    bins.append(b)
        return cls(box=box, vectors=np.array(vectors, dtype=np.int64).reshape(-1, 3),
                   bins=np.array(bins, dtype=np.int64), q=np.array(qs))

    @property
    def is_lattice(self) -> bool:
        return self._vectors is not None

    def indices(self) -> np.ndarray:
        return self._vectors if self.is_lattice else miller_indices(self.p_max)

    def q(self) -> np.ndarray:
        return self._q if self.is_lattice else np.zeros(0)

    def vectors_per_bin(self):
        if not self.is_lattice:
            return []
        return np.bincount(self._bins, minlength=len(self._q)).tolist()

    def check_box(self, box_sides) -> None:
        if not self.is_lattice:
            return
        if not all(abs(box_sides[a] - self.box[a]) <= 1e-9 * self.box[a] for a in range(3)):
            raise UsageError(f"box {list(box_sides)} differs from the {self.box} the q-grid was "
                             "built for")

    def group(self, qnorm: np.ndarray, values: np.ndarray):
        """Mean of the rows per |q| group (src/q_grid.rs:140-157)."""
        if not self.is_lattice:
            return average_by_qnorm(qnorm, values)
        sums = np.zeros((len(self._q), values.shape[1]))
        for r, b in enumerate(self._bins):
            sums[b] = sums[b] + values[r]
        counts = np.array(self.vectors_per_bin(), dtype=np.float64)
        return self._q.copy(), sums / counts[:, None]
