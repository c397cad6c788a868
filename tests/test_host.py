"""Host logic on the CPU: recombination, fitting, synthetic inputs, request
construction. No GPU."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from pripps_b200 import (DebyeModel, ExcludedVolume, Hydration, QOutOfRange, SolventConfig,
                         Structure, UsageError, ValidationError, combine, synth, workloads)
from pripps_b200 import fit as F
from pripps_b200.debye import make_request
from pripps_b200.formfactor import FormFactorMap, AtomKind, Constant, Polynomial, linear_q_values


def test_combine_is_the_reference_order():
    rng = np.random.default_rng(0)
    t = rng.normal(size=(6, 13))
    got = combine(t, 0.9, 0.05)
    for k in range(13):
        assert got[k] == O.combine(t[:, k].copy(), 0.9, 0.05)


def test_model_intensity_knobs():
    rng = np.random.default_rng(1)
    t = np.abs(rng.normal(size=(6, 9)))
    m = DebyeModel(np.linspace(0, 0.4, 9), t)
    zero = m.intensity(0.0, 0.0)
    assert np.array_equal(zero.total, zero.contributions.atoms)
    a = m.intensity(1.0, 0.0)
    b = m.intensity(1.0, 0.0)
    assert np.array_equal(a.total, b.total)
    assert not np.array_equal(m.intensity(1.0, 0.1).total, a.total)


def test_cubic_spline_reproduces_nodes_and_cubics():
    xs = np.linspace(0, 1, 11)
    ys = np.sin(3 * xs)
    sp = F.CubicSpline(xs, ys)
    for x, y in zip(xs, ys):
        assert abs(sp.eval(x) - y) < 1e-14
    assert abs(sp.eval(0.55) - math.sin(1.65)) < 2e-3
    assert sp.eval(-1.0) == ys[0] and sp.eval(2.0) == ys[-1]


def test_chi2_scale_invariance_and_zero_at_truth():
    q = np.linspace(0.01, 0.5, 60)
    theory = type("T", (), {})()
    theory.q = q
    theory.total = 100.0 / (1 + 30 * q ** 2)
    exp = F.ExpData.from_arrays(q, 3.0 * theory.total, 0.01 * theory.total)
    assert F.chi2_per_point(theory, exp) < 1e-20
    assert abs(F.compute_scale(theory, exp) - 3.0) < 1e-12


def test_nelder_mead_and_grid_recover_knobs():
    """Fit the knobs back from a curve generated at known knobs."""
    q = np.linspace(0.0, 0.5, 41)
    rng = np.random.default_rng(5)
    t = np.vstack([1e4 * np.exp(-20 * q ** 2), 3e3 * np.exp(-15 * q ** 2),
                   2e2 * np.exp(-5 * q ** 2), 4e3 * np.exp(-18 * q ** 2),
                   -3e2 * np.exp(-9 * q ** 2), -1e2 * np.exp(-8 * q ** 2)])
    m = DebyeModel(q, t)
    truth = m.intensity(1.12, 0.04).total
    qe = np.linspace(0.02, 0.48, 50)
    sp = F.CubicSpline(q, truth)
    ie = np.array([sp.eval(x) for x in qe])
    r = m.fit(qe, 2.5 * ie, 0.01 * ie)
    assert abs(r.volume_scale - 1.12) < 2e-3 and abs(r.contrast_density - 0.04) < 2e-3
    assert abs(r.scale - 2.5) < 1e-3 * 2.5  # scale·I_th ≈ I_exp
    g = m.fit(qe, ie, None, method="grid", c1_points=151, c2_points=101)
    assert abs(g.volume_scale - 1.12) <= 0.01 and abs(g.contrast_density - 0.04) <= 0.001 + 1e-12
    with pytest.raises(ValidationError):
        m.fit(qe, ie, method="grid", c1_points=1)


def test_expdata_validation():
    with pytest.raises(ValidationError):
        F.ExpData.from_arrays([], [], [])
    with pytest.raises(ValidationError):
        F.ExpData.from_arrays([0.1, 0.2], [1.0], [])
    e = F.ExpData.from_arrays([0.1, 0.2], [1.0, 2.0])
    assert e.sigma == [1.0, 1.0]


def test_rsa_spacing_and_shape():
    rng = np.random.default_rng(2)
    p = synth.rsa_points(3000, (20.0, 12.0, 12.0), rng)
    from scipy.spatial import cKDTree
    d, _ = cKDTree(p).query(p, k=2)
    assert d[:, 1].min() >= synth.D_MIN
    assert np.all(np.sum((p / np.array([20.0, 12.0, 12.0])) ** 2, axis=1) <= 1.0)


def test_surface_distance_ellipsoid():
    axes = (8.0, 4.0, 4.0)
    pts = np.array([[0.0, 0.0, 0.0], [7.0, 0.0, 0.0], [0.0, 3.5, 0.0], [0.0, 0.0, 1.0]])
    d = synth.surface_distance(pts, axes)
    assert abs(d[1] - 1.0) < 1e-9 and abs(d[2] - 0.5) < 1e-9 and abs(d[3] - 3.0) < 1e-9
    assert abs(d[0] - 4.0) < 1e-5  # off-axis closest point, found after the nudge


def test_globule_distributions():
    g = synth.globule(20_000, (30.0, 30.0, 30.0), 7)
    frac = np.bincount(g.elements, minlength=4) / len(g.elements)
    assert np.allclose(frac, synth.ELEMENT_PROBS, atol=0.01)
    near = synth.surface_distance(g.pos, g.axes) <= 3.0
    assert not np.any(g.exposed & ~near)
    assert abs(g.exposed[near].mean() - 0.35) < 0.03
    # deterministic from the seed
    g2 = synth.globule(20_000, (30.0, 30.0, 30.0), 7)
    assert np.array_equal(g.pos, g2.pos) and np.array_equal(g.exposed, g2.exposed)


def test_trajectory_weights_dirichlet():
    base = np.zeros((10, 3))
    f, w = synth.trajectory(base, 256, 0.5, 3)
    assert f.shape == (256, 10, 3)
    assert abs(w.sum() - 1.0) < 1e-12 and np.all(w > 0)
    assert abs(np.std(f) - 0.5) < 0.02


def test_stream_distribution():
    rs = synth.request_stream(4000, 50.0, 1)
    ns = np.array([r.n_atoms for r in rs])
    assert ns.min() >= 500 and ns.max() <= 50_000
    assert abs(np.median(np.log(ns)) - 0.5 * (math.log(500) + math.log(50_000))) < 0.15
    arr = np.array([r.arrival for r in rs])
    assert np.all(np.diff(arr) > 0)
    assert abs(np.mean(np.diff(arr)) - 1 / 50.0) < 0.002
    assert abs(np.mean([r.solvent for r in rs]) - 0.7) < 0.03


def test_workload_requests():
    w = workloads.sphere_solvent_10k()
    r = w.request
    assert r.n_atoms == 10_000 and r.nq == 500 and r.ff_excluded is not None
    # hydration weights: exposed surface atoms only, the full-shell weight of
    # their element
    wfull = workloads.tables(np.array([0.0]), True)[3]
    exp = w.globule.exposed
    assert np.all(r.hyd_weights[~exp] == 0)
    assert np.allclose(r.hyd_weights[exp], wfull[w.globule.elements[exp]])
    # the same structure on another grid keeps its solvent model
    g = w.with_grid(64, "fp64")
    assert g.nq == 64 and g.precision == "fp64" and np.array_equal(g.xyz, r.xyz)
    assert np.array_equal(g.hyd_weights, r.hyd_weights)


def test_trajectory_workload_on_another_grid_keeps_its_frames():
    w = workloads.trajectory_5k_256(n_frames=6)
    g = w.with_grid(24, "fp64")
    assert g.n_frames == 6 and np.array_equal(g.xyz, w.request.xyz)
    assert np.array_equal(g.frame_weights, w.request.frame_weights)


def _tiny_map():
    a = AtomKind("A", 3.0, 10.0)
    b = AtomKind("B", 2.0, None)
    return FormFactorMap.from_entries([(a, Polynomial((0.0, 0.4), [5.0, 0.0, -1.0])),
                                       (b, Constant(2.0))])


def test_make_request_tables_and_errors():
    m = _tiny_map()
    s = Structure(np.array([[0, 0, 0], [1.0, 0, 0], [0, 2.0, 0]]), np.array([1, 0, 1]))
    q = linear_q_values(0.0, 0.3, 4)
    r = make_request(s, m, q, 0.0, 0.3, None)
    assert list(r.species) == [1, 0, 1] and r.ff_atoms.shape == (2, 4)
    # unused species are not evaluated: a structure of B atoms only at q > 0.4
    s_b = Structure(np.zeros((2, 3)), np.array([1, 1]))
    qb = linear_q_values(0.0, 1.0, 3)
    r = make_request(s_b, m, qb, 0.0, 1.0, None)
    assert r.ff_atoms.shape == (1, 3)
    with pytest.raises(QOutOfRange):
        make_request(s, m, qb, 0.0, 1.0, None)
    # Fraser needs a displaced volume on every used kind
    cfg = SolventConfig(ExcludedVolume.fraser(1.0))
    with pytest.raises(ValidationError):
        make_request(s, m, q, 0.0, 0.3, cfg)
    s_a = Structure(np.zeros((1, 3)), np.array([0]))
    r = make_request(s_a, m, q, 0.0, 0.3, cfg)
    assert abs(r.ff_excluded[0, 0] - 0.334 * 10.0) < 1e-12
    # hydration without areas: the tessellation is unavailable
    with pytest.raises(UsageError):
        make_request(s_a, m, q, 0.0, 0.3, SolventConfig(hydration=Hydration.sasa(0.03)))
