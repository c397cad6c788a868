"""Grid solvent dummies (excluded-volume cells and hydration shell points) and
the union request that carries them to the device.

The generators restate src/solvent/grid_excluded.rs and src/solvent/grid.rs;
here they are checked against a loop-for-loop restatement of the reference's
brute-force generators on small structures (same points, same order), against
the reference's own unit tests of those files, and the union request is
checked against the oracle's build_model with separate dummy sets.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from pripps_b200 import workloads
from pripps_b200.debye import make_request, union_request
from pripps_b200.dummies import (DummySet, WATER_SPACING, grid_excluded_dummies,
                                 grid_hydration_dummies, grid_steps, nearest_surface_distance)
from pripps_b200.formfactor import (AtomKind, Constant, FormFactorMap, SingleGaussian,
                                    linear_q_values)
from pripps_b200.solvent import ExcludedVolume, Hydration, SolventConfig
from pripps_b200.structure import Structure


def _one_atom_map(with_water=True):
    kind = AtomKind("C", sigma=2.0 * 1.7)
    entries = [(kind, Constant(6.0))]
    if with_water:
        entries.append((AtomKind("H2O"), Constant(10.0)))
    return FormFactorMap.from_entries(entries)


def _brute_grid(pos, radii, spacing, margin, keep):
    """The reference's triple loop (src/solvent/grid.rs:52-77)."""
    lo = [min(p[d] for p in pos) - margin for d in range(3)]
    hi = [max(p[d] for p in pos) + margin for d in range(3)]
    n = [grid_steps(lo[d], hi[d], spacing) for d in range(3)]
    out = []
    for ix in range(n[0]):
        x = lo[0] + ix * spacing
        for iy in range(n[1]):
            y = lo[1] + iy * spacing
            for iz in range(n[2]):
                z = lo[2] + iz * spacing
                d = math.inf
                for (cx, cy, cz), r in zip(pos, radii):
                    dx, dy, dz = x - cx, y - cy, z - cz
                    d = min(d, math.sqrt(dx * dx + dy * dy + dz * dz) - r)
                if keep(d):
                    out.append((x, y, z))
    return np.array(out).reshape(-1, 3)


@pytest.mark.parametrize("seed", [0, 1])
def test_grid_generators_match_the_reference_loops(seed):
    m = workloads.foxs()
    g = workloads.small_globule(40, seed).globule
    ids = workloads.element_ids()[g.elements]
    radii = [m.kind(int(i)).radius for i in ids]
    pos = g.pos
    exc = grid_excluded_dummies(pos, ids, m, 0.334, 1.1)
    ref = _brute_grid(pos.tolist(), radii, 1.1, max(radii) + 1.1, lambda d: d <= 0.0)
    assert np.array_equal(exc.positions, ref)
    hyd = grid_hydration_dummies(pos, ids, m, 2.3, 3.0, 1.8)
    ref = _brute_grid(pos.tolist(), radii, 2.3, max(radii) + 1.8 + 3.0 + 2.3,
                      lambda d: 1.8 < d < 4.8)
    assert np.array_equal(hyd.positions, ref)
    assert np.all(hyd.weights == (2.3 / WATER_SPACING) ** 3)
    assert np.all(exc.weights == 1.0)


def test_single_atom_shell_is_spherical():
    """src/solvent/grid.rs:109-129"""
    shell = grid_hydration_dummies(np.zeros((1, 3)), np.array([0]), _one_atom_map(), 1.5, 3.0,
                                   1.4)
    assert len(shell) > 50
    r = np.linalg.norm(shell.positions, axis=1)
    assert np.all(r > 3.0) and np.all(r < 6.2)


def test_no_shell_points_inside_protein():
    """src/solvent/grid.rs:131-151"""
    pos = np.array([[0.0, 0, 0], [2.0, 0, 0]])
    shell = grid_hydration_dummies(pos, np.array([0, 0]), _one_atom_map(), 1.5, 3.0, 1.4)
    d = nearest_surface_distance(shell.positions, pos, np.array([1.7, 1.7]), 10.0)
    assert np.all(d > 1.39)


def test_grid_excluded_single_atom_and_volume():
    """src/solvent/grid_excluded.rs:94-138: every cell inside the atom, and the
    cell volume sum within 15 % of the sphere at 0.3 Å spacing."""
    m = _one_atom_map(False)
    d = grid_excluded_dummies(np.zeros((1, 3)), np.array([0]), m, 0.334, 0.5)
    assert len(d) > 10
    assert np.all(np.linalg.norm(d.positions, axis=1) - 1.7 <= 0.0)
    d = grid_excluded_dummies(np.zeros((1, 3)), np.array([0]), m, 0.334, 0.3)
    ratio = len(d) * 0.3 ** 3 / (4.0 / 3.0 * math.pi * 1.7 ** 3)
    assert 0.85 < ratio < 1.15


def test_grid_excluded_form_factor_at_zero_and_empty():
    """src/solvent/grid_excluded.rs:140-166: F(0) = ρ·V_cell; no atoms, no cells."""
    m = _one_atom_map(False)
    d = grid_excluded_dummies(np.zeros((1, 3)), np.array([0]), m, 0.334, 1.0)
    assert np.all(np.abs(d.form_factors_at(0.0) - 0.334 * 1.0) < 1e-10)
    e = grid_excluded_dummies(np.zeros((0, 3)), np.zeros(0, dtype=np.int64),
                              FormFactorMap.from_entries([]), 0.334, 1.0)
    assert len(e) == 0


def test_dummyset_length_checks():
    from pripps_b200.errors import InternalError
    with pytest.raises(InternalError):
        DummySet.weighted(np.zeros((3, 3)), Constant(1.0), np.ones(2))
    with pytest.raises(InternalError):
        DummySet.per_dummy(np.zeros((3, 3)), [Constant(1.0)], np.zeros(2))


def _grid_case(n, seed, nq=24, qmax=0.6):
    m = workloads.foxs()
    g = workloads.small_globule(n, seed).globule
    ids = workloads.element_ids()[g.elements]
    q = linear_q_values(0.0, qmax, nq)
    return m, Structure(g.pos, ids), q


@pytest.mark.parametrize("excluded,hydration", [
    ("grid", "grid"), ("grid", "disabled"), ("disabled", "grid"), ("foxs", "grid"),
    ("grid", "sasa")])
def test_union_request_equals_separate_sets_on_the_oracle(excluded, hydration):
    """The union request, summed by the oracle as one colocated point set,
    equals the oracle's build_model over the three separate sets (the
    decomposition the device relies on), term by term."""
    m, s, q = _grid_case(30, 4)
    exc = {"grid": ExcludedVolume.grid(1.4), "disabled": ExcludedVolume.disabled(),
           "foxs": ExcludedVolume.fraser_foxs(1.0)}[excluded]
    w = np.where(np.arange(len(s)) % 3 == 0, 2.5, 0.0)
    hyd = {"grid": Hydration.grid(0.03, spacing=2.5), "disabled": Hydration.disabled(),
           "sasa": Hydration.sasa(0.03, weights=w)}[hydration]
    cfg = SolventConfig(exc, hyd)
    req = make_request(s, m, q, 0.0, 0.6, cfg, "fp64")
    union = O.terms_for_request(req, precise=True)

    # the same model with the sets kept apart
    from pripps_b200.solvent import distinct_dummy_sets, excluded_table, water_table
    used = np.unique(s.ids)
    sp = np.searchsorted(used, s.ids)
    ffA = m.table(used, q)
    e_set, h_set = distinct_dummy_sets(cfg, s.pos, s.ids, m)
    if excluded == "foxs":
        exc_xyz, exc_kind, ffC = s.pos, sp, excluded_table(exc, m, used, q, 0.334)
    elif e_set is not None:
        idx, rows = e_set.rows(q)
        exc_xyz, exc_kind, ffC = e_set.positions, idx, rows
    else:
        exc_xyz = exc_kind = ffC = None
    if hydration == "sasa":
        hyd_xyz, hyd_w, ffW = s.pos, w, water_table(m, q)
    elif h_set is not None:
        hyd_xyz, hyd_w = h_set.positions, h_set.weights
        ffW = np.array([h_set.form_factors[0].eval(x) for x in q])
    else:
        hyd_xyz = hyd_w = ffW = None
    sets = O.build_model_sets(s.pos, sp, ffA, exc_xyz, exc_kind, ffC, hyd_xyz, hyd_w, ffW,
                              0.0, 0.6, len(q), precise=True).T
    scale = np.maximum(np.abs(sets), 1e-300)
    for r in range(6):
        if np.all(sets[r] == 0):
            assert np.all(union[r] == 0), r
        else:
            assert np.max(np.abs(union[r] - sets[r]) / np.max(scale[r])) < 1e-12, r


def test_union_request_layout():
    m, s, q = _grid_case(50, 2)
    cfg = SolventConfig(ExcludedVolume.grid(1.2), Hydration.grid(0.03))
    req = make_request(s, m, q, 0.0, 0.6, cfg, "fp32")
    S = len(np.unique(s.ids))
    n = len(s)
    assert req.ff_atoms.shape[0] == S + 2  # one excluded row (weights all 1), one water row
    assert np.all(req.ff_atoms[S:] == 0) and np.all(req.ff_excluded[:S] == 0)
    assert np.all(req.hyd_weights[:n] == 0)
    assert np.all(req.species[:n] < S)


def _inspect(req):
    import ctypes as C
    from pripps_b200 import _lib
    r = req.c_struct()
    out = [C.c_uint64() for _ in range(4)]
    rc = _lib.lib().pd_plan_inspect(None, C.byref(r), *[C.byref(o) for o in out])
    return rc, [o.value for o in out]


def test_union_request_marks_grid_sets_as_lattices_and_covers_every_pair():
    """Both grid sets travel as lattice sets (one species each, the grid's
    origin, spacing and extents); the plan's pair tiles plus the lattice
    pair counts cover every unordered pair of the union exactly once, with
    far fewer tiles than without the lattices."""
    m, s, q = _grid_case(200, 6)
    cfg = SolventConfig(ExcludedVolume.grid(1.0), Hydration.grid(0.03))
    req = make_request(s, m, q, 0.0, 0.6, cfg, "fp32")
    S = len(np.unique(s.ids))
    assert [l[0] for l in req.lattices] == [S, S + 1]
    for sp, origin, spacing, extent in req.lattices:
        pts = req.xyz[req.species == sp]
        idx = (pts - np.array(origin)) / spacing
        assert np.all(np.abs(idx - np.rint(idx)) < 1e-9)
        assert np.all(np.rint(idx) >= 0) and np.all(np.rint(idx) < np.array(extent))
    rc, (ncls, npad, ntiles, covered) = _inspect(req)
    assert rc == 0
    n = req.n_atoms
    assert covered == n * (n - 1) // 2
    plain = make_request(s, m, q, 0.0, 0.6, cfg, "fp32")
    plain.lattices = None
    rc, (_, _, ntiles_plain, covered_plain) = _inspect(plain)
    assert rc == 0 and covered_plain == covered
    assert ntiles < ntiles_plain / 2


def test_lattice_validation():
    from pripps_b200 import _lib
    m, s, q = _grid_case(60, 1)
    cfg = SolventConfig(ExcludedVolume.grid(1.2), Hydration.grid(0.03))
    good = make_request(s, m, q, 0.0, 0.6, cfg, "fp32")
    assert _inspect(good)[0] == 0
    sp, origin, spacing, extent = good.lattices[0]
    for bad in [(sp, origin, -1.0, extent), (sp, origin, spacing, (0, 1, 1)),
                (999, origin, spacing, extent), (sp, (np.nan, 0, 0), spacing, extent),
                (sp, origin, spacing, (5000, 5000, 5000))]:
        r = make_request(s, m, q, 0.0, 0.6, cfg, "fp32")
        r.lattices = [bad]
        assert _inspect(r)[0] == _lib.PD_EINVAL, bad
    r = make_request(s, m, q, 0.0, 0.6, cfg, "fp32")
    r.lattices = [good.lattices[0], good.lattices[0]]
    assert _inspect(r)[0] == _lib.PD_EINVAL
    # a lattice species whose points carry two hydration weights
    r = make_request(s, m, q, 0.0, 0.6, cfg, "fp32")
    hyd_sp = good.lattices[1][0]
    k = np.flatnonzero(r.species == hyd_sp)[0]
    r.hyd_weights[k] *= 2.0
    assert _inspect(r)[0] == _lib.PD_EINVAL
