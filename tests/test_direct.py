"""Direct transform host logic and its oracle (no GPU): Miller vectors, |q|
grouping, the --num-molecules guards, and the oracle's amplitude rows on
closed forms."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from pripps_b200.direct import (average_by_qnorm, check_num_molecules, miller_indices, q_bin,
                                q_vectors)
from pripps_b200.errors import UsageError, ValidationError
from pripps_b200.structure import Structure


def test_miller_indices_order_and_count():
    """13 directions (outer) × p = 1..p_max (inner), src/explicit.rs:275-283."""
    n = miller_indices(3)
    assert n.shape == (39, 3)
    assert n[:3].tolist() == [[1, 0, 0], [2, 0, 0], [3, 0, 0]]
    assert n[-1].tolist() == [3, 3, -3]
    q = q_vectors(n, [10.0, 20.0, 40.0])
    assert np.allclose(q[1], [2 * 2 * math.pi / 10.0, 0, 0])


def test_average_duplicates_golden():
    """The reference's test_average_duplicates (src/explicit.rs:470-475)."""
    qs = np.array([1.0, 3.0, 2.0, 2.0, 1.0])
    v = np.array([[1.0], [0.1], [3.0], [4.0], [2.0]])
    q, g = average_by_qnorm(qs, v)
    assert q.tolist() == [1.0, 2.0, 3.0]
    assert g[:, 0].tolist() == [1.5, 3.5, 0.1]
    assert q_bin(0.1234565) == 123457 and q_bin(2.5e-6) == 3


def test_oracle_rows_closed_forms():
    """One scatterer: |A|² = f²; two scatterers: f1² + f2² + 2 f1 f2 cos(q·Δr);
    two molecules of one atom each: self = f1² + f2²."""
    qv = q_vectors(miller_indices(4), [30.0, 30.0, 30.0])
    xyz = np.array([[1.0, 2.0, 3.0], [4.0, -1.0, 0.5]])
    ff = np.array([np.full(len(qv), 2.0), np.full(len(qv), 3.0)])
    one = O.direct_rows(xyz[:1], [0], ff, qv)
    assert np.allclose(one[:, 2], 4.0) and np.allclose(one[:, 3], 4.0)
    two = O.direct_rows(xyz, [0, 1], ff, qv, 2)
    ph = qv @ (xyz[1] - xyz[0])
    assert np.allclose(two[:, 2], 4.0 + 9.0 + 12.0 * np.cos(ph), atol=1e-12)
    assert np.allclose(two[:, 3], 13.0)
    w = O.direct_rows(xyz, [0, 1], ff, qv, 1, weight=[0.5, 2.0])
    assert np.allclose(w[:, 2], 1.0 + 36.0 + 12.0 * np.cos(ph), atol=1e-12)


def test_num_molecules_guards():
    """src/lib.rs:368-411 (and the guards of num_molecules_* tests, :1160-1232)."""
    two = Structure(np.array([[0, 0, -3], [0, 0, 3], [50, 0, -3], [50, 0, 3.0]]), [0, 0, 0, 0])
    check_num_molecules(two, 2, False)
    with pytest.raises(ValidationError):
        check_num_molecules(two, 3, False)
    with pytest.raises(UsageError):
        check_num_molecules(two, 0, False)
    with pytest.raises(UsageError):
        check_num_molecules(two, 2, True)
    mismatch = Structure(np.array([[0, 0, 0], [1, 0, 0], [50, 0, 0], [51, 0, 0.0]]), [0, 1, 1, 0])
    with pytest.raises(ValidationError):
        check_num_molecules(mismatch, 2, False)
