"""The FP64 oracle against the reference's golden vectors and known answers.

These pin the oracle before any GPU result is compared with it:
  * PEPSI I_at on 4lzt (src/lib.rs:808-854, max rel < 0.04),
  * I(0) = (Σf)² (src/multipole/mod.rs:908-940),
  * two atoms at 4 Å: 2 + 2·sinc(4q) (src/multipole/mod.rs:943-967),
  * Fraser F(0) = ρV and linearity in the volume (src/solvent/fraser.rs:142-163),
  * the fully-exposed SASA weight (src/solvent/sasa.rs:101-118),
  * inclusive q-grid endpoints (src/q_sampler.rs:173-185),
  * cross sum includes coincident pairs (src/debye.rs:236-250).
"""
import math

import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O


def test_pepsi_iat_golden():
    g = load_golden("pepsi_4lzt.json")
    vac = O.vacuum(np.array(g["positions"]), np.array(g["species"]), np.array(g["ff_atoms"]),
                   g["qmin"], g["qmax"], g["nq"])
    ref = np.array(g["pepsi_iat"])
    rel = np.max(np.abs(vac - ref) / ref)
    assert rel < g["pepsi_rel_tol"], rel
    # the committed oracle output is reproduced bit for bit
    assert np.array_equal(vac, np.array(g["oracle_vacuum"]))


def test_intensity_at_q_zero_is_sum_squared():
    xyz = np.array([[0, 0, 0], [2, 0, 0], [0, 3, 0], [0, 0, 1.5]], dtype=float)
    v = O.vacuum(xyz, np.zeros(4), np.ones((1, 5)), 0.0, 0.1, 5)
    assert abs(v[0] - 16.0) < 1e-10


def test_two_atoms_closed_form():
    xyz = np.array([[0, 0, 0], [4.0, 0, 0]])
    q = O.linear_q_values(0.01, 0.5, 20)
    v = O.vacuum(xyz, np.zeros(2), np.ones((1, 20)), 0.01, 0.5, 20)
    exact = 2 + 2 * np.sin(4 * q) / (4 * q)
    assert np.max(np.abs(v - exact) / exact) < 1e-14


def test_sinc_threshold():
    assert O.sinc(0.0) == 1.0
    assert O.sinc(0.9e-8) == 1.0
    assert O.sinc(1e-3) == math.sin(1e-3) / 1e-3


def test_q_grid_inclusive():
    q = O.linear_q_values(0.0, 1.0, 11)
    assert q[0] == 0.0 and q[10] == 1.0
    assert list(O.linear_q_values(0.42, 0.42, 1)) == [0.42]


def test_fraser_q0_and_linearity():
    rho, v = 0.334, 16.43
    assert O.fraser(0.0, v, rho, 4 * math.pi) == rho * v
    assert O.fraser(0.0, 2 * v, rho, 4 * math.pi) == 2 * O.fraser(0.0, v, rho, 4 * math.pi)
    # FoXS (16π) decays more slowly than PepsiSAXS (4π)
    assert O.fraser(0.5, v, rho, 16 * math.pi) > O.fraser(0.5, v, rho, 4 * math.pi)


def test_sasa_full_weight():
    w = O.sasa_full_weight(1.7, 1.4)
    assert abs(w - 4 * math.pi * 3.1 ** 2 * 3 / 30) < 1e-12


def test_cross_includes_coincident_pairs():
    xyz = np.array([[0, 0, 0], [3.0, 0, 0]])
    fa = np.array([2.0, 3.0])
    fb = np.array([5.0, 7.0])
    q = 0.2
    s = math.sin(q * 3) / (q * 3)
    expect = 2 * 5 + 3 * 7 + (2 * 7 + 3 * 5) * s
    assert abs(O.cross_intensity(xyz, fa, xyz, fb, q) - expect) < 1e-12


def test_build_model_rows_consistent():
    """Self rows equal the vacuum sum with the same per-atom factors, and the
    six terms combine like DebyeTerms::combine."""
    rng = np.random.default_rng(3)
    xyz = rng.uniform(-6, 6, (40, 3))
    sp = rng.integers(0, 3, 40)
    ffA = rng.uniform(1, 8, (3, 9))
    ffC = rng.uniform(0.5, 3, (3, 9))
    w = rng.uniform(0, 1, 40)
    fw = rng.uniform(5, 10, 9)
    t = O.build_model(xyz, sp, ffA, ffC, w, fw, 0.0, 0.4, 9)
    vac = O.vacuum(xyz, sp, ffA, 0.0, 0.4, 9)
    assert np.array_equal(t[:, 0], vac)
    vacC = O.vacuum(xyz, sp, ffC, 0.0, 0.4, 9)
    assert np.array_equal(t[:, 1], vacC)
    for k in range(9):
        v, c = 1.3, 0.07
        tt = t[k]
        expect = tt[0] + v * v * tt[1] + c * c * tt[2] - 2 * v * tt[3] + 2 * c * tt[4] - 2 * v * c * tt[5]
        assert O.combine(tt, v, c) == expect


def test_solvent_golden_reproduced():
    g = load_golden("solvent_4lzt.json")
    t = O.build_model(np.array(g["positions"]), np.array(g["species"]), np.array(g["ff_atoms"]),
                      np.array(g["ff_excluded"]), np.array(g["hyd_weights"]),
                      np.array(g["ff_water"]), g["qmin"], g["qmax"], g["nq"]).T
    assert np.array_equal(t, np.array(g["oracle_terms"]))
    # q = 0: every sinc is 1, so AA(0) = (ΣA)², AC(0) = ΣA·ΣC
    sp = np.array(g["species"])
    A0 = np.array(g["ff_atoms"])[sp, 0]
    C0 = np.array(g["ff_excluded"])[sp, 0]
    assert abs(t[0, 0] - A0.sum() ** 2) < 1e-9 * A0.sum() ** 2
    assert abs(t[3, 0] - A0.sum() * C0.sum()) < 1e-9 * abs(A0.sum() * C0.sum())
