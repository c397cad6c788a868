"""Solvent models of the Debye path: excluded volume (C) and hydration (B).

Host-side restatement of the reference's solvent configuration
(src/solvent/mod.rs) for the models whose dummy scatterers sit at the atom
positions — the ones the CUDA backend's colocated form serves:

  ExcludedVolume.Fraser / FraserFoxs  one Gaussian dummy per atom,
      C_i(q) = ρ·V·exp(-V^{2/3} q²/D), V = volume_scale·displaced_volume,
      D = 4π (PepsiSAXS) or 16π (FoXS)      (src/solvent/fraser.rs:26-100)
  ExcludedVolume.PerKind  per-species ``excluded_solvent`` form factor
                                              (src/solvent/per_kind_excluded.rs)
  Hydration.Sasa  B_i(q) = w_i·F_H2O(q), w_i = clamp(area_i, 0, 4π(r+p)²)·3/30
                                              (src/solvent/sasa.rs:47-70)

Models whose dummies sit at their own positions (pripps_b200.dummies):

  ExcludedVolume.Grid     grid cells inside the envelope   (src/solvent/grid_excluded.rs)
  Hydration.Grid          grid points in a shell around it  (src/solvent/grid.rs)
  ExcludedVolume.custom / Hydration.custom   a caller-built DummySet

The SASA areas and the Voronoi models come from voronota-ltr in the
reference, a dependency that is not available here; callers supply per-atom
areas (or weights) for SASA, and Voronoi dummies as a custom DummySet.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .dummies import DummySet, grid_excluded_dummies, grid_hydration_dummies
from .errors import UsageError, ValidationError
from .formfactor import FormFactorMap

WATER_KIND_NAME = "H2O"          # src/solvent/mod.rs:43
WATER_VOLUME = 30.0              # Å³, src/solvent/mod.rs:46
SHELL_THICKNESS = 3.0            # Å, src/solvent/sasa.rs:32
PEPSI_DENOMINATOR = 4.0 * math.pi   # src/solvent/fraser.rs:29
FOXS_DENOMINATOR = 16.0 * math.pi   # src/solvent/fraser.rs:39
DEFAULT_BULK_DENSITY = 0.334     # e/Å³, src/solvent/mod.rs:113-120


# ----------------------------------------------------------- excluded volume
@dataclass(frozen=True)
class ExcludedVolume:
    kind: str = "disabled"        # disabled | fraser | fraser_foxs | per_kind | grid | custom
    volume_scale: float = 1.0
    spacing: float = 1.0          # grid: cell edge (Å), src/cli.rs:98-100
    dummy_set: Optional[DummySet] = field(default=None, compare=False)

    @staticmethod
    def disabled() -> "ExcludedVolume":
        return ExcludedVolume("disabled", 0.0)

    @staticmethod
    def fraser(volume_scale: float = 1.0) -> "ExcludedVolume":
        return ExcludedVolume("fraser", float(volume_scale))

    @staticmethod
    def fraser_foxs(volume_scale: float = 1.0) -> "ExcludedVolume":
        return ExcludedVolume("fraser_foxs", float(volume_scale))

    @staticmethod
    def per_kind(volume_scale: float = 1.0) -> "ExcludedVolume":
        return ExcludedVolume("per_kind", float(volume_scale))

    @staticmethod
    def grid(spacing: float = 1.0, volume_scale: float = 1.0) -> "ExcludedVolume":
        """Grid cells filling the envelope (src/solvent/grid_excluded.rs)."""
        return ExcludedVolume("grid", float(volume_scale), float(spacing))

    @staticmethod
    def custom(dummies: DummySet, volume_scale: float = 1.0) -> "ExcludedVolume":
        """Caller-built excluded-volume dummies (unit basis; the scale is
        applied when the six profiles are combined)."""
        return ExcludedVolume("custom", float(volume_scale), dummy_set=dummies)

    def at_atoms(self) -> bool:
        """Whether the dummies sit at the atom positions (one per atom)."""
        return self.kind in ("fraser", "fraser_foxs", "per_kind")

    def is_active(self) -> bool:
        return self.kind != "disabled"

    def effective_volume_scale(self) -> float:
        """0 for Disabled (src/solvent/mod.rs:131-143)."""
        return 0.0 if self.kind == "disabled" else self.volume_scale

    def unit_scale(self) -> "ExcludedVolume":
        """The unit basis cached models are built on (src/solvent/mod.rs:385-403)."""
        return self if self.kind == "disabled" else ExcludedVolume(self.kind, 1.0, self.spacing,
                                                                    self.dummy_set)


def fraser_form_factor(q: float, volume: float, rho: float, denominator: float) -> float:
    """ρV·exp(-(V^{2/3}/D)·q·q) (src/solvent/fraser.rs:48-57 + SingleGaussian)."""
    a = rho * volume
    b = volume ** (2.0 / 3.0) / denominator
    return a * math.exp(-b * q * q)


def excluded_table(cfg: ExcludedVolume, formfactors: FormFactorMap, species: np.ndarray,
                   q_values: np.ndarray, bulk_electron_density: float) -> Optional[np.ndarray]:
    """[len(species) × nq] C_s(q_k) table for the listed species ids, or None.

    Always the unit basis (volume_scale = 1): the scale is applied when the
    six terms are combined, as the reference builds its dummies through
    unit_scale_dummies for both the cached and the one-shot Debye path
    (src/debye.rs:62-66, :83-87)."""
    if cfg.kind == "disabled" or not cfg.at_atoms():
        return None
    out = np.empty((len(species), len(q_values)), dtype=np.float64)
    if cfg.kind in ("fraser", "fraser_foxs"):
        denom = PEPSI_DENOMINATOR if cfg.kind == "fraser" else FOXS_DENOMINATOR
        for r, sid in enumerate(species):
            kind = formfactors.kind(int(sid))
            if kind.displaced_volume is None:
                raise ValidationError(
                    f"atom kind {kind.name} has no `displaced_volume`; required by "
                    "ExcludedVolume::Fraser")
            vol = 1.0 * kind.displaced_volume
            out[r] = [fraser_form_factor(float(q), vol, bulk_electron_density, denom)
                      for q in q_values]
        return out
    if cfg.kind == "per_kind":
        for r, sid in enumerate(species):
            ff = formfactors.excluded_solvent(int(sid))
            if ff is None:
                raise ValidationError(
                    f"atom kind {formfactors.kind(int(sid)).name} has no `excluded_solvent` "
                    "form factor; required by ExcludedVolume::PerKind")
            out[r] = [ff.eval(float(q)) for q in q_values]
        return out
    raise UsageError(f"excluded volume '{cfg.kind}' places dummies away from the atoms; "
                     "the CUDA Debye backend serves colocated dummies only")


# ----------------------------------------------------------------- hydration
@dataclass(frozen=True)
class Hydration:
    kind: str = "disabled"            # disabled | sasa | grid | custom
    probe: float = 1.8
    contrast_density: float = 0.0
    areas: Optional[tuple] = None     # per-atom SAS areas (Å²), or
    weights: Optional[tuple] = None   # per-atom shell weights directly
    spacing: float = 3.10516          # grid: point spacing (Å), src/cli.rs:112-116
    thickness: float = 3.0            # grid: shell thickness (Å), src/cli.rs:117-119
    dummy_set: Optional[DummySet] = field(default=None, compare=False)

    @staticmethod
    def disabled() -> "Hydration":
        return Hydration()

    @staticmethod
    def sasa(contrast_density: float = 0.03, probe: float = 1.8, *, areas=None,
             weights=None) -> "Hydration":
        return Hydration("sasa", float(probe), float(contrast_density),
                         None if areas is None else tuple(np.asarray(areas, dtype=float)),
                         None if weights is None else tuple(np.asarray(weights, dtype=float)))

    @staticmethod
    def grid(contrast_density: float = 0.03, spacing: float = 3.10516, thickness: float = 3.0,
             probe: float = 1.8) -> "Hydration":
        """Grid points in a shell around the envelope (src/solvent/grid.rs)."""
        return Hydration("grid", float(probe), float(contrast_density), spacing=float(spacing),
                         thickness=float(thickness))

    @staticmethod
    def custom(dummies: DummySet, contrast_density: float = 0.03) -> "Hydration":
        """Caller-built hydration dummies (e.g. a Voronoi shell)."""
        return Hydration("custom", 0.0, float(contrast_density), dummy_set=dummies)

    def at_atoms(self) -> bool:
        return self.kind == "sasa"

    def is_active(self) -> bool:
        return self.kind != "disabled"

    def effective_contrast_density(self) -> float:
        return 0.0 if self.kind == "disabled" else self.contrast_density


def sasa_weights(hyd: Hydration, formfactors: FormFactorMap, ids: np.ndarray) -> np.ndarray:
    """Per-atom shell weights: clamp(area, 0, 4π(r+probe)²)·3/30 where r is the
    kind's YAML radius (src/solvent/sasa.rs:47-61)."""
    n = len(ids)
    if hyd.weights is not None:
        w = np.asarray(hyd.weights, dtype=np.float64)
        if len(w) != n:
            raise ValidationError(f"hydration weights ({len(w)}) do not match atoms ({n})")
        return w
    if hyd.areas is None:
        raise UsageError("Hydration.sasa needs per-atom SAS areas (the voronota-ltr "
                         "tessellation is not available); pass areas= or weights=")
    areas = np.asarray(hyd.areas, dtype=np.float64)
    if len(areas) != n:
        raise ValidationError(f"SAS areas ({len(areas)}) do not match atoms ({n})")
    out = np.empty(n, dtype=np.float64)
    for i, sid in enumerate(ids):
        kind = formfactors.kind(int(sid))
        if kind.radius is None:
            raise ValidationError(
                f"atom kind {kind.name} has no `radius`; required by Hydration::Sasa")
        rp = kind.radius + hyd.probe
        full = 4.0 * math.pi * (rp * rp)
        a = min(max(areas[i], 0.0), full)
        out[i] = a * SHELL_THICKNESS / WATER_VOLUME
    return out


def full_shell_weight(radius: float, probe: float = 1.8) -> float:
    """Weight of an atom whose whole shell is exposed: 4π(r+p)²·3/30."""
    rp = radius + probe
    return 4.0 * math.pi * (rp * rp) * SHELL_THICKNESS / WATER_VOLUME


def water_table(formfactors: FormFactorMap, q_values: np.ndarray) -> np.ndarray:
    ff = formfactors.form_factor_by_name(WATER_KIND_NAME)
    if ff is None:
        raise ValidationError(
            f"Hydration::Sasa requires an `{WATER_KIND_NAME}` entry in the form-factor YAML")
    return np.array([ff.eval(float(q)) for q in q_values], dtype=np.float64)


# --------------------------------------------------------------- top level
@dataclass(frozen=True)
class SolventConfig:
    excluded: ExcludedVolume = ExcludedVolume()
    hydration: Hydration = Hydration()
    bulk_electron_density: float = DEFAULT_BULK_DENSITY

    def is_active(self) -> bool:
        """src/solvent/mod.rs:123-128"""
        return self.excluded.is_active() or self.hydration.is_active()


def distinct_dummy_sets(cfg: "SolventConfig", pos: np.ndarray, ids: np.ndarray,
                        formfactors: FormFactorMap):
    """(excluded DummySet or None, hydration DummySet or None) for the models
    whose dummies sit at their own positions; both None for colocated models
    (src/solvent/mod.rs:405-470, unit basis)."""
    exc = hyd = None
    e, h = cfg.excluded, cfg.hydration
    if e.kind == "grid":
        exc = grid_excluded_dummies(pos, ids, formfactors, cfg.bulk_electron_density, e.spacing)
    elif e.kind == "custom":
        exc = e.dummy_set
    if h.kind == "grid":
        hyd = grid_hydration_dummies(pos, ids, formfactors, h.spacing, h.thickness, h.probe)
    elif h.kind == "custom":
        hyd = h.dummy_set
    if hyd is not None and hyd.weights is None:
        raise UsageError("hydration dummies must be a weighted DummySet (one shared form "
                         "factor, per-dummy weights)")
    return exc, hyd
