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


# ---------------------------------------------------------------- q grids
# The reference's own q-grid tests (src/q_grid.rs:362-485), restated.
from pripps_b200.direct import QGrid

L = 405.0


def test_first_bin_holds_the_unit_and_face_diagonal_vectors():
    grid = QGrid.lattice([L] * 3, 0.023, 10 ** 9)
    assert grid.vectors_per_bin() == [9]
    expected = 2.0 * math.pi / L * (3.0 + 6.0 * math.sqrt(2.0)) / 9.0
    assert abs(grid.q()[0] - expected) <= 1e-12 * expected


def test_bin_counts_match_a_brute_force_count():
    grid = QGrid.lattice([L] * 3, 0.5, 10 ** 9)
    assert grid.vectors_per_bin()[:8] == [9, 31, 49, 105, 175, 225, 301, 381]


def test_the_cap_thins_large_bins_only_and_keeps_their_q():
    full = QGrid.lattice([L] * 3, 0.5, 10 ** 9)
    capped = QGrid.lattice([L] * 3, 0.5, 100)
    for a, k in zip(full.vectors_per_bin(), capped.vectors_per_bin()):
        assert k == min(a, 100)
    assert np.array_equal(full.q(), capped.q())


def _assert_isotropic(grid, b, eps):
    picked = grid.indices()[grid._bins == b].astype(np.float64)
    norm2 = (picked * picked).sum(axis=1)
    tensor = (picked[:, :, None] * picked[:, None, :] / norm2[:, None, None]).sum(axis=0)
    tensor /= len(picked)
    assert np.all(np.abs(tensor - np.eye(3) / 3.0) <= eps), tensor


def test_a_capped_bin_still_spans_the_sphere():
    grid = QGrid.lattice([L] * 3, 0.5, 50)
    _assert_isotropic(grid, len(grid.q()) - 1, 0.03)


def test_sampled_bins_span_the_sphere_and_share_q_across_caps():
    """a_sampled_bin_spans_the_sphere and huge_boxes_are_sampled_not_enumerated
    (src/q_grid.rs:430-484), with the reference's box and q_max."""
    l = 6900.0
    small = QGrid.lattice([l] * 3, 0.5, 16)
    large = QGrid.lattice([l] * 3, 0.5, 200)
    assert np.array_equal(small.q(), large.q())
    assert np.all(np.diff(small.q()) > 0)
    counts = small.vectors_per_bin()
    assert all(n <= 16 for n in counts)
    assert sum(1 for n in counts if n < 12) < 3
    _assert_isotropic(large, len(large.q()) - 2, 0.03)
    width = 2.0 * math.pi / l
    qm = small.q()[len(small.q()) // 2]
    k = round(qm / width)
    expected = 0.75 * ((k + 0.5) ** 4 - (k - 0.5) ** 4) / ((k + 0.5) ** 3 - (k - 0.5) ** 3) * width
    assert abs(qm - expected) <= 1e-6 * expected


def test_impossible_grids_are_errors():
    for box, q in [([L] * 3, 0.01), ([L, 0.0, L], 0.5), ([L, float("nan"), L], 0.5),
                   ([L] * 3, float("inf")), ([L] * 3, float("nan")), ([L] * 3, -0.5)]:
        with pytest.raises(UsageError):
            QGrid.lattice(box, q, 10)


def test_a_narrow_last_bin_survives_any_cap():
    q_max = 0.054_190_196_758_008_29
    small = QGrid.lattice([6900.0] * 3, q_max, 16)
    large = QGrid.lattice([6900.0] * 3, q_max, 200)
    assert np.array_equal(small.q(), large.q())
