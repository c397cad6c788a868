"""Solvent dummy scatterers at their own positions.

The grid models of the reference place their scatterers on a Cartesian grid
instead of at the atoms:

  grid_excluded_dummies   ExcludedVolume::Grid (src/solvent/grid_excluded.rs):
      every grid point inside the molecular envelope (distance to the nearest
      atom surface <= 0) carries the Fraser form factor of one grid cell,
      ρ·V·exp(-V^{2/3} q²/4π), V = spacing³, weight 1
  grid_hydration_dummies  Hydration::Grid (src/solvent/grid.rs):
      every grid point with probe < d < probe + thickness (d = distance to the
      nearest atom surface) carries the H2O form factor times the number of
      water molecules per cell, (spacing / 3.10516)³

A ``DummySet`` (src/solvent/mod.rs:202-374) is positions plus either one form
factor per dummy (PerDummy) or one shared form factor times per-dummy weights
(Weighted). Callers with their own generators (e.g. the Voronoi models, whose
tessellation library is not available here) can build one directly.

On the device the three sets (atoms A, excluded-volume dummies C, hydration
dummies B) become one point set whose classes each carry one set's factor, so
a single pass over all unordered pairs yields the reference's three self sums
and three cross sums (see ``pripps_b200.debye.union_request``).
"""
from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np

from .errors import InternalError, ValidationError
from .formfactor import FormFactor, FormFactorMap, SingleGaussian

PEPSI_DENOMINATOR = 4.0 * math.pi   # src/solvent/fraser.rs:29
WATER_KIND_NAME = "H2O"             # src/solvent/mod.rs:43
WATER_SPACING = 3.10516             # Å per water molecule at 30 Å³, src/solvent/grid.rs:86-94


class DummySet:
    """Dummy scatterers: positions [n, 3] Å and their form factors, either
    ``per_dummy`` (one FormFactor per dummy, given as a list of distinct form
    factors and an index per dummy) or ``weighted`` (one FormFactor, scaled by
    a weight per dummy)."""

    def __init__(self, positions, *, form_factors: Sequence[FormFactor],
                 kinds: Optional[np.ndarray] = None, weights: Optional[np.ndarray] = None,
                 lattice: Optional[tuple] = None):
        self.positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        # (origin [3], spacing, extent [3]) when every dummy sits on the grid
        # origin + spacing·(i, j, k), 0 <= i < extent[0], ...: the device then
        # sums the set's self pairs from exact counts per squared offset
        self.lattice = lattice
        self.form_factors = list(form_factors)
        n = len(self.positions)
        if (kinds is None) == (weights is None):
            raise InternalError("DummySet: give exactly one of kinds (per dummy) or weights")
        if weights is not None:
            self.weights = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
            self.kinds = None
            if len(self.form_factors) != 1:
                raise InternalError("DummySet: a weighted set has one shared form factor")
            if len(self.weights) != n:
                # src/solvent/mod.rs:309-315
                raise InternalError(f"DummySet: positions ({n}) and weights "
                                    f"({len(self.weights)}) length mismatch")
        else:
            self.kinds = np.ascontiguousarray(kinds, dtype=np.int64).reshape(-1)
            self.weights = None
            if len(self.kinds) != n:
                raise InternalError(f"DummySet: positions ({n}) and form_factors "
                                    f"({len(self.kinds)}) length mismatch")
            if n and (self.kinds.min() < 0 or self.kinds.max() >= len(self.form_factors)):
                raise InternalError("DummySet: form factor index out of range")

    @classmethod
    def weighted(cls, positions, form_factor: FormFactor, weights,
                 lattice: Optional[tuple] = None) -> "DummySet":
        return cls(positions, form_factors=[form_factor], weights=weights, lattice=lattice)

    @classmethod
    def per_dummy(cls, positions, form_factors: Sequence[FormFactor], kinds) -> "DummySet":
        return cls(positions, form_factors=form_factors, kinds=kinds)

    def __len__(self):
        return len(self.positions)

    def form_factors_at(self, q: float) -> np.ndarray:
        """F_i(q) of every dummy (DummySet::form_factors_at, src/solvent/mod.rs:357-374)."""
        if self.weights is not None:
            shared = self.form_factors[0].eval(float(q))
            return self.weights * shared
        vals = np.array([f.eval(float(q)) for f in self.form_factors])
        return vals[self.kinds]

    def rows(self, q_values: np.ndarray):
        """Per-dummy form factors as (row index per dummy [n], rows [R, nq]):
        one row per distinct (form factor, weight); the reference evaluates
        each dummy's form factor, which is the row's value at every q."""
        q_values = np.asarray(q_values, dtype=np.float64)
        if self.weights is not None:
            base = np.array([self.form_factors[0].eval(float(q)) for q in q_values])
            uniq, idx = np.unique(self.weights, return_inverse=True)
            return idx.astype(np.int64), uniq[:, None] * base[None, :]
        tabs = np.array([[f.eval(float(q)) for q in q_values] for f in self.form_factors])
        used, idx = np.unique(self.kinds, return_inverse=True)
        return idx.astype(np.int64), tabs[used].reshape(len(used), len(q_values))


def atom_radii(ids: np.ndarray, formfactors: FormFactorMap, caller: str) -> np.ndarray:
    """Per-atom radius from the kind's YAML ``radius`` (src/solvent/mod.rs:57-78)."""
    out = np.empty(len(ids), dtype=np.float64)
    cache = {}
    for i, sid in enumerate(np.asarray(ids).tolist()):
        r = cache.get(sid)
        if r is None:
            kind = formfactors.kind(int(sid))
            if kind.radius is None:
                raise ValidationError(f"atom kind {kind.name} has no `radius`; required by "
                                      f"{caller}")
            r = cache[sid] = float(kind.radius)
        out[i] = r
    return out


def grid_steps(lo: float, hi: float, spacing: float) -> int:
    """ceil((hi - lo) / spacing) + 1 (src/solvent/grid.rs:35-37)."""
    return int(math.ceil((hi - lo) / spacing)) + 1


def _grid(lo: np.ndarray, hi: np.ndarray, spacing: float):
    """Grid points lo + i·spacing in the reference's loop order (x outer,
    z inner), [nx·ny·nz, 3], and the lattice (lo, spacing, (nx, ny, nz))."""
    ext = tuple(grid_steps(lo[d], hi[d], spacing) for d in range(3))
    axes = [lo[d] + np.arange(ext[d], dtype=np.float64) * spacing for d in range(3)]
    gx, gy, gz = np.meshgrid(*axes, indexing="ij")
    pts = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    return pts, (tuple(float(v) for v in lo), float(spacing), ext)


def nearest_surface_distance(points: np.ndarray, centers: np.ndarray, radii: np.ndarray,
                             cutoff: float) -> np.ndarray:
    """min over atoms of |p - c| - r for every point (src/solvent/grid.rs:
    26-32), with the distance evaluated exactly as the reference does
    (component differences, sqrt of x² + y² + z² in that order, minus r).
    Exact wherever the minimum is at most `cutoff`; points whose nearest
    surface is farther get +inf (every caller compares against a threshold
    no larger than `cutoff`). Candidate atoms come from a k-d tree query of
    radius cutoff + max(r): an atom farther away has |p - c| - r > cutoff."""
    from scipy.spatial import cKDTree

    n = len(points)
    out = np.full(n, np.inf)
    if n == 0 or len(centers) == 0:
        return out
    reach = float(cutoff + radii.max())
    tp, ta = cKDTree(points), cKDTree(centers)
    pairs = tp.sparse_distance_matrix(ta, reach * (1 + 1e-12) + 1e-9, output_type="ndarray")
    if len(pairs) == 0:
        return out
    pi = pairs["i"].astype(np.int64)
    ai = pairs["j"].astype(np.int64)
    d = points[pi] - centers[ai]
    dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]) - radii[ai]
    np.minimum.at(out, pi, dist)
    out[out > cutoff] = np.inf
    return out


def grid_excluded_dummies(pos: np.ndarray, ids: np.ndarray, formfactors: FormFactorMap,
                          bulk_electron_density: float, spacing: float) -> DummySet:
    """Excluded-volume grid dummies (src/solvent/grid_excluded.rs:34-73)."""
    if not spacing > 0:
        raise ValidationError("grid spacing must be positive")
    radii = atom_radii(ids, formfactors, "ExcludedVolume::Grid")
    cell_volume = spacing ** 3
    ff = SingleGaussian(bulk_electron_density * cell_volume,
                        cell_volume ** (2.0 / 3.0) / PEPSI_DENOMINATOR)
    if len(pos) == 0:
        return DummySet.weighted(np.zeros((0, 3)), ff, np.zeros(0))
    margin = float(radii.max()) + spacing
    lo, hi = pos.min(axis=0) - margin, pos.max(axis=0) + margin
    pts, lattice = _grid(lo, hi, spacing)
    d = nearest_surface_distance(pts, pos, radii, 0.0)
    keep = pts[d <= 0.0]
    return DummySet.weighted(keep, ff, np.ones(len(keep)), lattice)


def grid_hydration_dummies(pos: np.ndarray, ids: np.ndarray, formfactors: FormFactorMap,
                           spacing: float, thickness: float, probe: float) -> DummySet:
    """Hydration-shell grid dummies (src/solvent/grid.rs:40-95)."""
    if not spacing > 0:
        raise ValidationError("grid spacing must be positive")
    radii = atom_radii(ids, formfactors, "Hydration::Grid")
    water = formfactors.form_factor_by_name(WATER_KIND_NAME)
    if water is None:
        raise ValidationError(f"Hydration::Grid requires an `{WATER_KIND_NAME}` entry in the "
                              "form-factor YAML")
    per_cell = (spacing / WATER_SPACING) ** 3
    if len(pos) == 0:
        return DummySet.weighted(np.zeros((0, 3)), water, np.zeros(0))
    margin = float(radii.max()) + probe + thickness + spacing
    lo, hi = pos.min(axis=0) - margin, pos.max(axis=0) + margin
    pts, lattice = _grid(lo, hi, spacing)
    outer = probe + thickness
    d = nearest_surface_distance(pts, pos, radii, outer)
    keep = pts[(d > probe) & (d < outer)]
    return DummySet.weighted(keep, water, np.full(len(keep), per_cell), lattice)
