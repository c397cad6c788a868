"""Host-side form-factor model and YAML resolver (src/formfactor.rs),
checked against hand-computed values and the oracle's C restatement."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from pripps_b200 import QOutOfRange
from pripps_b200.formfactor import (Constant, Gaussian, Polynomial, SingleGaussian, Table,
                                    formfactors_from_yaml_str, linear_q_values)
from pripps_b200 import workloads


def test_polynomial_and_range():
    ff = Polynomial((0.0, 1.0), [2.0, -1.0, 0.5, 3.0])
    assert ff.eval(0.0) == 2.0
    assert abs(ff.eval(1.0) - 4.5) < 1e-15
    assert ff.eval(0.3) == O.eval_polynomial(0.3, [2.0, -1.0, 0.5, 3.0])
    with pytest.raises(QOutOfRange):
        ff.eval(1.5)


def test_table_interpolation():
    ff = Table([(0.0, 2.0), (1.0, 4.0), (2.0, 10.0)])
    assert ff.eval(1.0) == 4.0
    assert ff.eval(0.5) == 3.0
    assert ff.eval(1.5) == 7.0
    xs, ys = [0.0, 1.0, 2.0], [2.0, 4.0, 10.0]
    for x in (0.25, 1.0, 1.75, 2.0):
        assert ff.eval(x) == O.interpolate(xs, ys, x)
    with pytest.raises(QOutOfRange):
        ff.eval(-0.01)


def test_gaussian_s2_convention():
    ff = Gaussian((0.0, math.inf), [(4.0, 12.0)], 0.5)
    s2 = 0.36 / (16 * math.pi ** 2)
    assert ff.eval(0.6) == 4.0 * math.exp(-12.0 * s2) + 0.5
    assert ff.eval(0.6) == O.eval_gaussian(0.6, [(4.0, 12.0)], 0.5)


def test_single_gaussian_q2_convention():
    ff = SingleGaussian(3.0, 0.2)
    assert ff.eval(0.0) == 3.0
    assert ff.eval(0.5) == 3.0 * math.exp(-0.2 * 0.25)


YAML = """
A:  { radius: 1.5, ff: !Constant 2.0, excluded_solvent: !Constant 0.5 }
B:  { displaced_volume: 7.0, ff: !Constant 5.0, excluded_solvent: !Constant 1.5 }
AL: { ff: !Constant 1.0, excluded_solvent: !Alias A }
LI: { ff: !Constant 1.0, excluded_solvent: !Linear [[A, 2.0], [B, 4.0]] }
UN: { ff: !United { center: B, orbit: [[A, 1.2, 3]] }, excluded_solvent: !United { center: B, orbit: [[A, 0.8]] } }
"""


def test_symbolic_resolution():
    m = formfactors_from_yaml_str(YAML)
    names = [k.name for k in m.kinds()]
    assert names == sorted(names)  # BTreeMap order
    exc = lambda n: m.excluded_solvent(m.id_of(n)).eval(0.0)
    assert exc("AL") == 0.5
    assert abs(exc("LI") - (2 * 0.5 + 4 * 1.5)) < 1e-12
    assert abs(exc("UN") - (1.5 + 0.5)) < 1e-12  # weight defaults to 1, sinc(0) = 1
    un = m.form_factor(m.id_of("UN"))
    q = 1.0
    assert abs(un.eval(q) - (5.0 + 3 * 2.0 * math.sin(1.2) / 1.2)) < 1e-12  # a grid point
    # displaced volume from the radius when absent: 4/3 π r³
    assert abs(m.kind(m.id_of("A")).displaced_volume - 4 / 3 * math.pi * 1.5 ** 3) < 1e-12
    assert m.kind(m.id_of("B")).displaced_volume == 7.0


def test_foxs_elements_asset():
    m = workloads.foxs()
    for name in ("C", "N", "O", "S", "H2O"):
        assert m.form_factor_by_name(name) is not None
    # S has no displaced volume in the asset: 4/3 π 1.68³
    s = m.kind(m.id_of("S"))
    assert abs(s.displaced_volume - 4 / 3 * math.pi * 1.68 ** 3) < 1e-12
    h2o = m.form_factor_by_name("H2O")
    assert h2o.qrange() == (0.0, 6.0)
    # United H2O at q = 0: F_O(0) + 2 F_H(0)
    o0 = m.form_factor_by_name("O").eval(0.0)
    h0 = m.form_factor_by_name("H").eval(0.0)
    assert abs(h2o.eval(0.0) - (o0 + 2 * h0)) < 1e-12
    # The tables the workloads feed the kernels: C/N/O/S Gaussians in range
    q = linear_q_values(0.0, 1.0, 11)
    ffA, ffC, ffW, wfull = workloads.tables(q, True)
    assert ffA.shape == (4, 11) and ffC.shape == (4, 11) and ffW.shape == (11,)
    assert abs(ffC[0, 0] - 0.334 * 16.44) < 1e-12
    assert abs(wfull[0] - O.sasa_full_weight(1.58, 1.8)) < 1e-12
