"""Form factors evaluated on the device (pd_formfactor_tables) against the
host evaluator that restates FormFactor::eval (src/formfactor.rs:188-201):
every kind of the reference, the FoXS element table (Gaussians) and the
United H2O table, and QOutOfRange outside a form factor's range."""
import numpy as np
import pytest

from pripps_b200 import _lib, workloads
from pripps_b200.errors import QOutOfRange
from pripps_b200.formfactor import (Constant, Gaussian, Polynomial, SingleGaussian, Table,
                                    device_tables, linear_q_values)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("qmin,qmax,nq", [(0.0, 0.5, 500), (0.0, 1.0, 1000), (0.1, 2.0, 37),
                                          (0.3, 0.3, 1)])
def test_device_tables_match_host(gpu_ctx, qmin, qmax, nq):
    m = workloads.foxs()
    ffs = [m.entries[i].formfactor for i in range(len(m))]
    ffs += [Constant(3.5), SingleGaussian(5.486, 0.42),
            Polynomial((0.0, 3.0), [1.0, -0.5, 0.25, 0.01]),
            Table([(0.0, 9.0), (0.7, 7.5), (1.5, 4.0), (2.5, 2.2)]),
            Gaussian((0.0, 6.0), [(2.31, 20.8439), (1.02, 10.2075)], 0.2156)]
    got = device_tables(ffs, qmin, qmax, nq, gpu_ctx)
    q = linear_q_values(qmin, qmax, nq)
    ref = np.array([[ff.eval(float(x)) for x in q] for ff in ffs])
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) < 1e-14


def test_device_tables_raise_qoutofrange(gpu_ctx):
    ffs = [Constant(1.0), Table([(0.0, 1.0), (0.5, 0.5)])]
    with pytest.raises(QOutOfRange):
        device_tables(ffs, 0.0, 0.8, 20, gpu_ctx)
    assert np.all(np.isfinite(device_tables(ffs, 0.0, 0.5, 20, gpu_ctx)))
