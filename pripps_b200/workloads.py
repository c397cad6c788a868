"""The Debye workloads, built from seeded synthetic globules.

  sphere_vacuum_1k     1,000 atoms, sphere R = 16 Å, vacuum, q ∈ [0, 0.5], nq = 500
  sphere_solvent_10k   10,000 atoms, sphere R = 35 Å, FoXS Fraser excluded volume
                       + Bernoulli(0.35) surface hydration, q ∈ [0, 0.5], nq = 500
  ellipsoid_solvent_100k  100,000 atoms, prolate ellipsoid 80×40×40 Å, solvent as
                       above, q ∈ [0, 1.0], nq = 1,000
  ellipsoid_solvent_20k / ellipsoid_sasa_20k  20,000 atoms at the 100k density,
                       nq = 512; the second with a continuous hydration weight
                       per atom (SASA-like: weighted mode)
  trajectory_5k_256    256 frames of a 5,000-atom sphere (R = 25 Å), σ = 0.5 Å,
                       Dirichlet(1) frame weights, vacuum, q ∈ [0, 0.5], nq = 300
  stream               Poisson requests, N log-uniform 500–50,000 (sphere at the
                       1k/16 Å density), nq 100–1000, qmax 0.3–1.0, 70 % solvent

Form factors: the FoXS Cromer–Mann elements (data/foxs_elements.yaml), FoXS
Fraser dummies ρ·V·exp(-V^{2/3} q²/16π) with ρ = 0.334 and the YAML displaced
volumes (S: 4/3·π·1.68³), and the United H2O table for hydration.
"""
from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache
from pathlib import Path
from typing import Optional

import numpy as np

from . import synth
from .debye import DebyeRequest
from .formfactor import FormFactorMap, linear_q_values, read_formfactors
from .solvent import (DEFAULT_BULK_DENSITY, ExcludedVolume, excluded_table, full_shell_weight,
                      water_table)

DATA = Path(__file__).resolve().parent / "data"


@lru_cache(maxsize=1)
def foxs() -> FormFactorMap:
    return read_formfactors(DATA / "foxs_elements.yaml")


def element_ids() -> np.ndarray:
    m = foxs()
    return np.array([m.id_of(e) for e in synth.ELEMENTS], dtype=np.int64)


def tables(qv: np.ndarray, solvent: bool):
    """Per-element (C, N, O, S) tables on the grid: F, C (FoXS Fraser) and
    F_H2O; plus the fully-exposed shell weight of each element."""
    m = foxs()
    ids = element_ids()
    ffA = m.table(ids, qv)
    if not solvent:
        return ffA, None, None, None
    ffC = excluded_table(ExcludedVolume.fraser_foxs(1.0), m, ids, qv, DEFAULT_BULK_DENSITY)
    ffW = water_table(m, qv)
    wfull = np.array([full_shell_weight(m.kind(int(i)).radius, synth.PROBE) for i in ids])
    return ffA, ffC, ffW, wfull


def globule_request(g: synth.Globule, qmin: float, qmax: float, nq: int, solvent: bool,
                    precision: str = "fp32", frames=None, frame_weights=None) -> DebyeRequest:
    qv = linear_q_values(qmin, qmax, nq)
    ffA, ffC, ffW, wfull = tables(qv, solvent)
    hw = None
    if solvent:
        hw = np.where(g.exposed, wfull[g.elements], 0.0)
    xyz = g.pos if frames is None else frames
    return DebyeRequest(xyz, g.elements.astype(np.uint32), ffA, ffC, hw, ffW, qmin, qmax, nq,
                        frame_weights, precision)


@dataclass
class Workload:
    name: str
    request: DebyeRequest
    globule: synth.Globule

    def with_grid(self, nq: int, precision: str) -> DebyeRequest:
        """The same structure and solvent model on another q grid (same
        range) and precision form."""
        r = self.request
        if self.name == "sphere_grid_solvent_10k":
            return grid_solvent_request(self.globule, r.qmin, r.qmax, nq, precision)
        frames = r.xyz if r.xyz.ndim == 3 else None  # a trajectory keeps its frames
        return globule_request(self.globule, r.qmin, r.qmax, nq, r.ff_excluded is not None,
                               precision, frames, r.frame_weights)

    @property
    def pairs(self) -> int:
        n = self.request.n_atoms
        return n * (n - 1) // 2

    @property
    def pair_q(self) -> int:
        return self.pairs * self.request.nq * self.request.n_frames


@lru_cache(maxsize=8)
def _globule(n, axes, seed):
    return synth.globule(n, axes, seed)


def sphere_vacuum_1k(precision="fp64") -> Workload:
    g = _globule(1000, (16.0, 16.0, 16.0), 0)
    return Workload("sphere_vacuum_1k", globule_request(g, 0.0, 0.5, 500, False, precision), g)


def sphere_solvent_10k(precision="fp32") -> Workload:
    g = _globule(10_000, (35.0, 35.0, 35.0), 1)
    return Workload("sphere_solvent_10k", globule_request(g, 0.0, 0.5, 500, True, precision), g)


def ellipsoid_solvent_100k(precision="fp32") -> Workload:
    g = _globule(100_000, (80.0, 40.0, 40.0), 2)
    return Workload("ellipsoid_solvent_100k",
                    globule_request(g, 0.0, 1.0, 1000, True, precision), g)


def ellipsoid_solvent_20k(precision="fp32") -> Workload:
    """A fifth of the 100k workload at the same density (axes × 0.2^{1/3}),
    nq = 512: the size used for detailed kernel profiles."""
    f = 0.2 ** (1.0 / 3.0)
    g = _globule(20_000, (80.0 * f, 40.0 * f, 40.0 * f), 12)
    return Workload("ellipsoid_solvent_20k",
                    globule_request(g, 0.0, 1.0, 512, True, precision), g)


def ellipsoid_sasa_20k(precision="fp32") -> Workload:
    """The 20,000-atom ellipsoid with a hydration weight per atom, as pripps'
    SASA hydration gives (area × shell thickness / water volume, a continuous
    value): each exposed atom's full-shell weight times a seeded exposed
    fraction in [0.05, 1). With thousands of distinct weights the kernels run
    in weighted mode (two accumulators per q)."""
    w = ellipsoid_solvent_20k(precision)
    req = w.request
    rng = np.random.default_rng(20)
    req.hyd_weights = req.hyd_weights * rng.uniform(0.05, 1.0, req.n_atoms)
    return Workload("ellipsoid_sasa_20k", req, w.globule)


def trajectory_5k_256(precision="fp32", n_frames: int = 256) -> Workload:
    g = _globule(5000, (25.0, 25.0, 25.0), 3)
    frames, w = synth.trajectory(g.pos, n_frames, 0.5, 3)
    return Workload("trajectory_5k_256",
                    globule_request(g, 0.0, 0.5, 300, False, precision, frames, w), g)


def grid_solvent_request(g: synth.Globule, qmin: float, qmax: float, nq: int,
                         precision: str = "fp32", excluded_spacing: float = 1.0,
                         hydration_spacing: float = 3.10516):
    """Atoms plus grid solvent dummies at their own positions: excluded-volume
    cells of `excluded_spacing` Å filling the envelope (FoXS radii) and
    hydration points of `hydration_spacing` Å in the 1.8-4.8 Å shell around it,
    as one union request (see pripps_b200.debye.union_request)."""
    from .debye import make_request
    from .solvent import ExcludedVolume, Hydration, SolventConfig
    from .structure import Structure
    cfg = SolventConfig(ExcludedVolume.grid(excluded_spacing),
                        Hydration.grid(0.03, spacing=hydration_spacing))
    q = linear_q_values(qmin, qmax, nq)
    s = Structure(g.pos, element_ids()[g.elements])
    return make_request(s, foxs(), q, qmin, qmax, cfg, precision)


def grid_solvent_sets(req: DebyeRequest, n_atoms: int):
    """Split a union request (atoms first, then excluded-volume dummies, then
    hydration dummies) back into the three sets, as the oracle's
    build_model_sets takes them: (atoms xyz, species, ffA, excluded xyz,
    excluded rows, ffC, hydration xyz, hydration weights, F_water)."""
    S_atoms = int(req.species[:n_atoms].max()) + 1
    sp = req.species.astype(np.int64)
    exc = (sp >= S_atoms) & (req.hyd_weights == 0)
    hyd = req.hyd_weights > 0
    hyd[:n_atoms] = False
    exc[:n_atoms] = False
    return (req.xyz[:n_atoms], req.species[:n_atoms], req.ff_atoms[:S_atoms],
            req.xyz[exc], sp[exc], req.ff_excluded, req.xyz[hyd], req.hyd_weights[hyd],
            req.ff_water)


def sphere_grid_solvent_10k(precision="fp32") -> Workload:
    """The 10,000-atom sphere with grid excluded volume (1 Å cells) and a
    grid hydration shell: ~111,000 points, nq = 500 on [0, 0.5]."""
    g = _globule(10_000, (35.0, 35.0, 35.0), 1)
    return Workload("sphere_grid_solvent_10k", grid_solvent_request(g, 0.0, 0.5, 500, precision),
                    g)


def stream_request(sr: synth.StreamRequest, precision="fp32") -> Workload:
    r = synth.sphere_radius_for(sr.n_atoms)
    g = synth.globule(sr.n_atoms, (r, r, r), sr.seed)
    return Workload(f"stream_{sr.n_atoms}",
                    globule_request(g, 0.0, sr.qmax, sr.nq, sr.solvent, precision), g)


class GlobulePool:
    """Compact sub-globules for long request streams: a few RSA globules at
    log-spaced sizes, atoms sorted by distance from the centre; a request of N
    atoms takes the N innermost atoms of the smallest pool globule that has
    them (the same packing density as a globule built for N, without an RSA
    run per request), with surface exposure redrawn for its own envelope."""

    def __init__(self, n_min: int = 500, n_max: int = 50_000, size: int = 24, seed: int = 40):
        self.globules = []
        for k, n in enumerate(np.unique(np.geomspace(n_min, n_max, size).astype(np.int64))):
            r = synth.sphere_radius_for(int(n))
            g = synth.globule(int(n), (r, r, r), seed + k)
            c = g.pos.mean(axis=0)
            order = np.argsort(np.linalg.norm(g.pos - c, axis=1), kind="stable")
            self.globules.append((int(n), g.pos[order] - c, g.elements[order]))

    def take(self, n: int, seed: int) -> synth.Globule:
        for size, pos, el in self.globules:
            if size >= n:
                break
        p, e = pos[:n], el[:n]
        rad = np.linalg.norm(p, axis=1)
        rng = np.random.default_rng(seed)
        exposed = (rad >= rad.max() - 3.0) & (rng.random(n) < synth.EXPOSED_PROB)
        return synth.Globule(p.copy(), e.copy(), exposed, (rad.max(),) * 3)


def stream_request_pooled(sr: synth.StreamRequest, pool: GlobulePool,
                          precision="fp32") -> Workload:
    g = pool.take(sr.n_atoms, sr.seed)
    return Workload(f"stream_{sr.n_atoms}",
                    globule_request(g, 0.0, sr.qmax, sr.nq, sr.solvent, precision), g)


def small_globule(n: int, seed: int, nq: int = 40, qmax: float = 0.5, solvent: bool = True,
                  precision: str = "fp32", radius: Optional[float] = None) -> Workload:
    r = radius if radius is not None else synth.sphere_radius_for(max(n, 8))
    g = synth.globule(n, (r, r, r), seed)
    return Workload(f"small_{n}", globule_request(g, 0.0, qmax, nq, solvent, precision), g)


WORKLOADS = {
    "sphere_grid_solvent_10k": sphere_grid_solvent_10k,
    "sphere_vacuum_1k": sphere_vacuum_1k,
    "sphere_solvent_10k": sphere_solvent_10k,
    "ellipsoid_solvent_100k": ellipsoid_solvent_100k,
    "ellipsoid_solvent_20k": ellipsoid_solvent_20k,
    "ellipsoid_sasa_20k": ellipsoid_sasa_20k,
    "trajectory_5k_256": trajectory_5k_256,
}
