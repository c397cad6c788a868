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

The reference's lattice q-grid builder (QGrid::lattice, src/q_grid.rs) is not
restated: a caller with such a grid passes its integer indices directly.
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


def amplitudes(xyz: np.ndarray, kind: np.ndarray, ff: np.ndarray, qvec: np.ndarray,
               n_molecules: int = 1, weight: Optional[np.ndarray] = None,
               ctx: Optional[_lib.Context] = None) -> np.ndarray:
    """pd_direct: [n_vectors, 4] = (Re A, Im A, |A|², Σ_m |F_m|²)."""
    ctx = ctx or _lib.default_context()
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    kind = np.ascontiguousarray(kind, dtype=np.uint32)
    ff = np.ascontiguousarray(ff, dtype=np.float64)
    qvec = np.ascontiguousarray(qvec, dtype=np.float64).reshape(-1, 3)
    w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
    r = _lib.PdDirectRequest()
    r.n_points = len(kind)
    r.xyz = _lib.dptr(xyz)
    r.kind = _lib.u32ptr(kind)
    r.n_kinds = int(ff.shape[0])
    r.reserved = 0
    r.ff = _lib.dptr(ff)
    r.n_vectors = len(qvec)
    r.qvec = _lib.dptr(qvec)
    r.n_molecules = int(n_molecules)
    r.weight = _lib.dptr(w)
    out = np.empty((len(qvec), 4), dtype=np.float64)
    _lib.check(_lib.lib().pd_direct(ctx.handle, C.byref(r), _lib.dptr(out)), ctx.handle)
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
                 indices: Optional[np.ndarray] = None, ctx: Optional[_lib.Context] = None):
        self.formfactors = formfactors
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
        rows = amplitudes(structure.pos, kind, ff, qvec, n, ctx=self.ctx)
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
            r = amplitudes(xyz, knd, table, qvec, 1, weight, ctx)
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
