"""Debye scattering on the B200: the six cached profiles and what sits on them.

Host-side mirror of the reference's Debye calculator (src/debye.rs), cached
model (``DebyeModel``, src/debye.rs:138-174), library entry points
(``Pripps.debye_model`` / ``Pripps.intensity``, src/lib.rs:287-303, 344-528)
and trajectory averaging (src/trajectory.rs:167-251). The pair sum itself —
the per-q body of ``build_model`` (src/debye.rs:90-130) — runs in
libpripps_debye through ``pd_solve``; nothing here computes a pair term.

``DebyeModel.intensity(volume_scale, contrast_density)`` recombines the six
cached terms exactly as ``DebyeTerms::combine`` does (src/debye.rs:187-194),
so fits and the one-shot path share one kernel result.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .dummies import DummySet
from .errors import ValidationError
from .formfactor import FormFactorMap, linear_q_values, read_formfactors
from .solvent import (SolventConfig, distinct_dummy_sets, excluded_table, sasa_weights,
                      water_table)
from .structure import Structure, structure_from_xyz

TERM_NAMES = ("atoms", "excluded", "hydration", "atom_excluded", "atom_hydration",
              "excluded_hydration")


@dataclass
class Contributions:
    """Unscaled self profiles (src/lib.rs:113-121)."""
    atoms: np.ndarray
    excluded: np.ndarray
    hydration: np.ndarray

    def __eq__(self, other):
        return (isinstance(other, Contributions) and np.array_equal(self.atoms, other.atoms)
                and np.array_equal(self.excluded, other.excluded)
                and np.array_equal(self.hydration, other.hydration))


@dataclass
class Intensity:
    """I(q) on a q grid (src/lib.rs:89-109). form_factor and
    effective_structure_factor are set by the direct transform of a box of
    identical molecules (src/lib.rs:510-526)."""
    q: np.ndarray
    total: np.ndarray
    contributions: Optional[Contributions] = None
    form_factor: Optional[np.ndarray] = None
    effective_structure_factor: Optional[np.ndarray] = None


def combine(terms: np.ndarray, volume_scale: float, contrast_density: float) -> np.ndarray:
    """AA + v²CC + c²BB − 2v·AC + 2c·AB − 2vc·CB per q, in the reference's
    operation order (src/debye.rs:187-194)."""
    t = np.asarray(terms, dtype=np.float64)
    v, c = float(volume_scale), float(contrast_density)
    return (t[0] + v * v * t[1] + c * c * t[2] - 2.0 * v * t[3] + 2.0 * c * t[4]
            - 2.0 * v * c * t[5])


class DebyeModel:
    """Cached six-profile Debye state for solvent fitting (src/debye.rs:138-174)."""

    def __init__(self, q_values: np.ndarray, terms: np.ndarray):
        self._q = np.asarray(q_values, dtype=np.float64)
        self.terms = np.asarray(terms, dtype=np.float64).reshape(6, -1)

    @property
    def q_values(self) -> np.ndarray:
        return self._q

    def intensity(self, volume_scale: float = 1.0, contrast_density: float = 0.03) -> Intensity:
        total = combine(self.terms, volume_scale, contrast_density)
        return Intensity(self._q.copy(), total,
                         Contributions(self.terms[0].copy(), self.terms[1].copy(),
                                       self.terms[2].copy()))

    def fit(self, q, intensity, sigma=None, *, method="nelder-mead", c1_points=151,
            c2_points=101, c1_bounds=None, c2_bounds=None):
        """Fit (volume_scale, contrast_density) to experimental data, as the
        pyo3 ``cached_model!`` fit does (pripps-py/src/lib.rs:619-646)."""
        from . import fit as _fit
        exp = _fit.ExpData.from_arrays(q, intensity, [] if sigma is None else sigma)
        c1b = _fit.DEFAULT_C1_BOUNDS if c1_bounds is None else tuple(c1_bounds)
        c2b = _fit.DEFAULT_C2_BOUNDS if c2_bounds is None else tuple(c2_bounds)
        ev = lambda c1, c2: self.intensity(c1, c2)
        m = str(method).lower().replace("_", "-")
        if m in ("nelder-mead", "neldermead"):
            return _fit.fit_parameters_with_bounds(exp, ev, c1b, c2b)
        if m == "grid":
            return _fit.fit_parameters_grid_with_bounds(exp, ev, c1_points, c2_points, c1b, c2b)
        raise ValidationError(f"unknown fit method {method!r}")


# ------------------------------------------------------------------ requests
@dataclass
class DebyeRequest:
    """Host arrays of one pd_request (see include/pripps_debye.h)."""
    xyz: np.ndarray                    # [F, N, 3] or [N, 3] float64
    species: np.ndarray                # [N] uint32, compact ids
    ff_atoms: np.ndarray               # [S, nq]
    ff_excluded: Optional[np.ndarray]  # [S, nq] or None
    hyd_weights: Optional[np.ndarray]  # [N] or None
    ff_water: Optional[np.ndarray]     # [nq] or None
    qmin: float
    qmax: float
    nq: int
    frame_weights: Optional[np.ndarray] = None
    precision: str = "fp32"
    # lattice sets: (species, origin [3], spacing, extent [3]) per set whose
    # points all sit on that lattice (see pd_lattice in pripps_debye.h)
    lattices: Optional[list] = None

    def __post_init__(self):
        self.xyz = np.ascontiguousarray(self.xyz, dtype=np.float64)
        self.species = np.ascontiguousarray(self.species, dtype=np.uint32)
        self.ff_atoms = np.ascontiguousarray(self.ff_atoms, dtype=np.float64)
        if self.ff_excluded is not None:
            self.ff_excluded = np.ascontiguousarray(self.ff_excluded, dtype=np.float64)
        if self.hyd_weights is not None:
            self.hyd_weights = np.ascontiguousarray(self.hyd_weights, dtype=np.float64)
            self.ff_water = np.ascontiguousarray(self.ff_water, dtype=np.float64)
        if self.frame_weights is not None:
            self.frame_weights = np.ascontiguousarray(self.frame_weights, dtype=np.float64)

    @property
    def n_atoms(self) -> int:
        return int(self.species.shape[0])

    @property
    def n_frames(self) -> int:
        return int(self.xyz.shape[0]) if self.xyz.ndim == 3 else 1

    def c_struct(self) -> _lib.PdRequest:
        r = _lib.PdRequest()
        r.n_atoms = self.n_atoms
        r.xyz = _lib.dptr(self.xyz)
        r.species = _lib.u32ptr(self.species)
        r.n_species = int(self.ff_atoms.shape[0])
        r.precision = _lib.PRECISIONS[self.precision]
        r.ff_atoms = _lib.dptr(self.ff_atoms)
        r.ff_excluded = _lib.dptr(self.ff_excluded)
        r.hyd_weights = _lib.dptr(self.hyd_weights)
        r.ff_water = _lib.dptr(self.ff_water)
        r.qmin = float(self.qmin)
        r.qmax = float(self.qmax)
        r.nq = int(self.nq)
        r.n_frames = self.n_frames if self.xyz.ndim == 3 else 0
        r.frame_weights = _lib.dptr(self.frame_weights)
        r.flags = 0
        lats = self.lattices or []
        r.n_lattices = len(lats)
        if lats:
            arr = (_lib.PdLattice * len(lats))()
            for k, (sp, origin, spacing, extent) in enumerate(lats):
                arr[k].species = int(sp)
                arr[k].origin[:] = [float(v) for v in origin]
                arr[k].spacing = float(spacing)
                arr[k].extent[:] = [int(v) for v in extent]
            self._lattice_array = arr  # keep alive as long as the struct is used
            r.lattices = C.cast(arr, C.POINTER(_lib.PdLattice))
        return r


def make_request(structure: Structure, formfactors: FormFactorMap, q_values: np.ndarray,
                 qmin: float, qmax: float, solvent: Optional[SolventConfig],
                 precision: str = "fp32", frames: Optional[np.ndarray] = None,
                 frame_weights: Optional[np.ndarray] = None) -> DebyeRequest:
    """Tabulate the per-species inputs of a solve on the host. Form factors are
    evaluated only for the species the structure uses, so a QOutOfRange is
    raised here exactly when the reference's formfactor_by_index would raise
    it (src/formfactor.rs:520-544)."""
    ids = structure.ids
    used = np.unique(ids)
    compact = np.searchsorted(used, ids).astype(np.uint32)
    ffA = formfactors.table(used, q_values)
    ffC = hw = ffW = None
    exc = hyd = None
    if solvent is not None and solvent.is_active():
        ffC = excluded_table(solvent.excluded, formfactors, used, q_values,
                             solvent.bulk_electron_density)
        if solvent.hydration.at_atoms():
            hw = sasa_weights(solvent.hydration, formfactors, ids)
            ffW = water_table(formfactors, q_values)
        if frames is None:
            exc, hyd = distinct_dummy_sets(solvent, structure.pos, ids, formfactors)
        elif not (solvent.excluded.at_atoms() or solvent.excluded.kind == "disabled") or \
                not (solvent.hydration.at_atoms() or solvent.hydration.kind == "disabled"):
            raise ValidationError("dummies away from the atoms depend on each frame; solve "
                                  "the frames one at a time")
    xyz = structure.pos if frames is None else np.asarray(frames, dtype=np.float64)
    if exc is None and hyd is None:
        return DebyeRequest(xyz, compact, ffA, ffC, hw, ffW, qmin, qmax, len(q_values),
                            frame_weights, precision)
    return union_request(structure.pos, compact, ffA, ffC, hw, ffW, exc, hyd, q_values, qmin,
                         qmax, precision)


def union_request(pos: np.ndarray, species: np.ndarray, ffA: np.ndarray,
                  ffC: Optional[np.ndarray], hw: Optional[np.ndarray], ffW: Optional[np.ndarray],
                  exc: Optional[DummySet], hyd: Optional[DummySet], q_values: np.ndarray,
                  qmin: float, qmax: float, precision: str = "fp32") -> DebyeRequest:
    """One request over atoms, excluded-volume dummies and hydration dummies
    as a single point set (the reference's build_model with dummies at their
    own positions, src/debye.rs:83-130).

    Species rows are extended so that each point carries only its own set's
    factor: atoms keep their A rows (and their C rows / SASA weights when those
    models sit at the atoms), excluded dummies get A = 0 and one C row per
    distinct dummy form factor, hydration dummies get A = C = 0 and
    B = w·F_water through the hydration weights. The sum over all unordered
    pairs of the union then splits exactly into the reference's three self
    sums (pairs within a set) and three cross sums (pairs across sets), and the
    i = j terms of the cross profiles vanish, as they must for distinct
    points."""
    S, nq = ffA.shape
    n = len(pos)
    xyz, sp, rows_a, rows_c, wts = [pos], [np.asarray(species, dtype=np.int64)], [ffA], [], []
    rows_c.append(ffC if ffC is not None else np.zeros((S, nq)))
    wts.append(hw if hw is not None else np.zeros(n))
    has_c, water = ffC is not None, ffW
    nxt = S
    if exc is not None and len(exc):
        idx, rows = exc.rows(q_values)
        xyz.append(exc.positions)
        sp.append(nxt + idx)
        rows_a.append(np.zeros_like(rows))
        rows_c.append(rows)
        wts.append(np.zeros(len(exc)))
        nxt += rows.shape[0]
        has_c = True
    has_b = hw is not None
    lattices = []
    if exc is not None and len(exc) and exc.lattice is not None and len(rows_c[-1]) == 1:
        lattices.append((nxt - 1,) + tuple(exc.lattice))
    if hyd is not None and len(hyd):
        xyz.append(hyd.positions)
        sp.append(np.full(len(hyd), nxt, dtype=np.int64))
        rows_a.append(np.zeros((1, nq)))
        rows_c.append(np.zeros((1, nq)))
        wts.append(hyd.weights)
        water = np.array([hyd.form_factors[0].eval(float(q)) for q in q_values])
        if hyd.lattice is not None and np.all(hyd.weights == hyd.weights[0]):
            lattices.append((nxt,) + tuple(hyd.lattice))
        nxt += 1
        has_b = True
    return DebyeRequest(np.concatenate(xyz), np.concatenate(sp).astype(np.uint32),
                        np.vstack(rows_a), np.vstack(rows_c) if has_c else None,
                        np.concatenate(wts) if has_b else None, water if has_b else None,
                        qmin, qmax, len(q_values), None, precision, lattices or None)


def solve(req: DebyeRequest, ctx: Optional[_lib.Context] = None) -> np.ndarray:
    """Blocking pd_solve: the [6, nq] terms (frame-weighted mean for batches)."""
    ctx = ctx or _lib.default_context()
    out = np.empty((6, req.nq), dtype=np.float64)
    r = req.c_struct()
    _lib.check(_lib.lib().pd_solve(ctx.handle, C.byref(r), _lib.dptr(out)), ctx.handle)
    return out


# ------------------------------------------------------------------ facade
class Pripps:
    """High-level entry points over a form-factor table (src/lib.rs:212-250)."""

    def __init__(self, formfactors: FormFactorMap, *, precision: str = "fp32",
                 ctx: Optional[_lib.Context] = None):
        if precision not in _lib.PRECISIONS:
            raise ValidationError(f"precision must be one of {sorted(_lib.PRECISIONS)}")
        self.formfactors = formfactors
        self.precision = precision
        self._ctx = ctx

    @classmethod
    def from_yaml(cls, path, **kw) -> "Pripps":
        return cls(read_formfactors(path), **kw)

    @property
    def ctx(self) -> _lib.Context:
        return self._ctx or _lib.default_context()

    def _structure(self, structure) -> Structure:
        if isinstance(structure, Structure):
            return structure
        return structure_from_xyz(structure, self.formfactors)

    def debye_model(self, structure, qmin: float = 0.0, qmax: float = 0.5, nq: int = 100,
                    solvent: Optional[SolventConfig] = None) -> DebyeModel:
        """Cached six-profile model (src/lib.rs:287-303 → src/debye.rs:78-136).
        Built on the unit basis; the knobs are applied in ``intensity``."""
        s = self._structure(structure)
        q = linear_q_values(qmin, qmax, nq)
        cfg = solvent if solvent is not None else SolventConfig()
        req = make_request(s, self.formfactors, q, qmin, qmax, cfg, self.precision)
        return DebyeModel(q, solve(req, self.ctx))

    def intensity(self, structure, qmin: float = 0.0, qmax: float = 0.5, nq: int = 100,
                  solvent: Optional[SolventConfig] = None, *, frames=None, frame_weights=None,
                  stride: int = 1) -> Intensity:
        """One-shot Debye intensity (src/debye.rs:56-69). Vacuum returns AA with
        no contributions; an active solvent builds the six terms and combines
        them at the configured knobs. With ``frames`` ([F, N, 3] Å), the
        weighted mean over frames[::stride] (src/trajectory.rs:167-251)."""
        s = self._structure(structure)
        q = linear_q_values(qmin, qmax, nq)
        active = solvent if (solvent is not None and solvent.is_active()) else None
        if frames is not None:
            return self._trajectory(s, q, qmin, qmax, active, frames, frame_weights, stride)
        req = make_request(s, self.formfactors, q, qmin, qmax, active, self.precision)
        terms = solve(req, self.ctx)
        if active is None:
            return Intensity(q, terms[0].copy(), None)
        model = DebyeModel(q, terms)
        return model.intensity(active.excluded.effective_volume_scale(),
                               active.hydration.effective_contrast_density())

    def direct_intensity(self, structure, p_max: int, box_sides,
                         solvent: Optional[SolventConfig] = None,
                         num_molecules: Optional[int] = None, indices=None,
                         grid=None) -> Intensity:
        """I(q) of a periodic box by the direct transform (IntensityScheme::
        Direct, src/lib.rs:424-431 with the --num-molecules guards and
        derivations, :365-411 and :510-526). ``indices`` replaces the Miller
        vectors with any integer reciprocal-lattice list."""
        from .direct import DirectTransform, check_num_molecules
        s = self._structure(structure)
        active = solvent if (solvent is not None and solvent.is_active()) else None
        check_num_molecules(s, num_molecules, active is not None)
        t = DirectTransform(self.formfactors, p_max, active, num_molecules, indices, self._ctx,
                            grid)
        return t.calc_intensities(s, box_sides)

    def direct_model(self, structure, p_max: int, box_sides, solvent: SolventConfig):
        """Cached direct-transform amplitudes for fitting (src/lib.rs:305-342)."""
        from .direct import DirectTransform
        s = self._structure(structure)
        t = DirectTransform(self.formfactors, p_max, solvent, None, None, self._ctx)
        return t.build_model(s, box_sides)

    def _trajectory(self, s, q, qmin, qmax, active, frames, frame_weights, stride):
        if not isinstance(frames, (np.ndarray, list, tuple)):
            return self._trajectory_stream(s, q, qmin, qmax, active, frames, frame_weights,
                                           stride)
        frames = np.asarray(frames, dtype=np.float64)
        if frames.ndim != 3 or frames.shape[1:] != (len(s), 3):
            raise ValidationError(
                f"frames must be [F, {len(s)}, 3]; got {tuple(frames.shape)}")
        n_all = frames.shape[0]
        if frame_weights is None:
            w_all = np.ones(n_all)
        else:
            w_all = np.asarray(frame_weights, dtype=np.float64)
            if len(w_all) != n_all:
                raise ValidationError(
                    f"number of weights ({len(w_all)}) does not match number of frames in "
                    f"trajectory ({n_all})")
            tot = float(np.sum(w_all))
            if not np.isfinite(tot) or tot == 0.0 or abs(tot) < np.finfo(float).tiny:
                raise ValidationError("sum of weights is zero or infinite")
        if stride < 1:
            raise ValidationError("stride must be >= 1")
        sel = frames[::stride]
        w = w_all[::stride]
        wsum = float(np.sum(w))
        if not np.isfinite(wsum) or wsum == 0.0 or abs(wsum) < np.finfo(float).tiny:
            raise ValidationError(
                f"weights of the {len(w)} averaged frames sum to {wsum}; cannot normalize")
        per_frame = active is not None and not (
            active.excluded.kind == "disabled" or active.excluded.at_atoms()) or (
            active is not None and not (active.hydration.kind == "disabled" or
                                        active.hydration.at_atoms()))
        if per_frame:
            # Dummies away from the atoms are rebuilt from every frame
            # (src/trajectory.rs:198-223 runs the calculator per frame): the
            # frames go to the request loop together and their totals are
            # averaged with the frame weights.
            from .serving import Server
            srv = Server(self.ctx)
            tickets = []
            for fr in sel:
                sf = Structure(fr, s.ids)
                tickets.append(srv.submit(make_request(sf, self.formfactors, q, qmin, qmax,
                                                       active, self.precision)))
            vs = active.excluded.effective_volume_scale()
            cd = active.hydration.effective_contrast_density()
            total = np.zeros(len(q))
            for wf, t in zip(w, tickets):
                total += wf * combine(srv.wait(t), vs, cd)
            return Intensity(q, total / wsum, None)
        req = make_request(s, self.formfactors, q, qmin, qmax, active, self.precision,
                           frames=sel, frame_weights=w)
        terms = solve(req, self.ctx)
        if active is None:
            return Intensity(q, terms[0].copy(), None)
        return Intensity(q, combine(terms, active.excluded.effective_volume_scale(),
                                    active.hydration.effective_contrast_density()), None)

    def _trajectory_stream(self, s, q, qmin, qmax, active, frames, frame_weights, stride,
                           frames_per_batch: int = 64):
        """Frames from an iterable (a reader), solved in pinned batches while
        later frames are still being read (pd_stream_*)."""
        if stride < 1:
            raise ValidationError("stride must be >= 1")
        req = make_request(s, self.formfactors, q, qmin, qmax, active, self.precision)
        if req.lattices:
            raise ValidationError("dummies away from the atoms depend on each frame; pass the "
                                  "frames as an array")
        st = TrajectoryStream(req, frames_per_batch, self.ctx)
        buf, wts = [], []
        for fr, w in _frame_pairs(frames, frame_weights, stride):
            buf.append(np.asarray(fr, dtype=np.float64).reshape(len(s), 3))
            wts.append(w)
            if len(buf) == frames_per_batch:
                st.push(np.stack(buf), np.array(wts))
                buf, wts = [], []
        if buf:
            st.push(np.stack(buf), np.array(wts))
        terms = st.finish()
        if active is None:
            return Intensity(q, terms[0].copy(), None)
        return Intensity(q, combine(terms, active.excluded.effective_volume_scale(),
                                    active.hydration.effective_contrast_density()), None)


def _frame_pairs(frames, frame_weights, stride):
    """(frame, weight) of every stride-th frame of an iterable, with the weight
    of the original frame index (src/trajectory.rs:56-61)."""
    wit = iter(frame_weights) if frame_weights is not None else None
    for k, fr in enumerate(frames):
        w = 1.0 if wit is None else float(next(wit))
        if k % stride == 0:
            yield fr, w


class TrajectoryStream:
    """A trajectory average fed frame by frame (pd_stream_*): the frame loop of
    trajectory_average (src/trajectory.rs:198-248) for trajectories too long to
    hold at once. ``push`` takes [F, N, 3] Å frames (and weights); pinned
    batches of ``frames_per_batch`` frames are uploaded while the previous
    batch is solved; ``finish`` returns the [6, nq] weighted mean of the six
    profiles."""

    def __init__(self, topology: DebyeRequest, frames_per_batch: int = 64,
                 ctx: Optional[_lib.Context] = None):
        self.ctx = ctx or _lib.default_context()
        self._req = topology
        self._nq = topology.nq
        self._n = topology.n_atoms
        self._h = C.c_void_p()
        r = topology.c_struct()
        _lib.check(_lib.lib().pd_stream_open(self.ctx.handle, C.byref(r), int(frames_per_batch),
                                             C.byref(self._h)), self.ctx.handle)

    def push(self, frames, weights=None) -> None:
        fr = np.ascontiguousarray(frames, dtype=np.float64).reshape(-1, self._n, 3)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        if w is not None and len(w) != len(fr):
            raise ValidationError(f"{len(w)} weights for {len(fr)} frames")
        _lib.check(_lib.lib().pd_stream_push(self.ctx.handle, self._h, _lib.dptr(fr),
                                             _lib.dptr(w), len(fr)), self.ctx.handle)

    def finish(self) -> np.ndarray:
        out = np.empty((6, self._nq), dtype=np.float64)
        h, self._h = self._h, C.c_void_p()
        _lib.check(_lib.lib().pd_stream_finish(self.ctx.handle, h, _lib.dptr(out)),
                   self.ctx.handle)
        return out

    def __del__(self):  # pragma: no cover - an unfinished stream is released
        try:
            if self._h:
                _lib.lib().pd_stream_finish(self.ctx.handle, self._h, None)
        except Exception:
            pass
