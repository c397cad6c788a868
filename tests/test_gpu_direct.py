"""Direct transform on the device (pd_direct) against the oracle's restated
rows (src/explicit.rs:138-147, :208-230), FP64: every row within 1e-12 of
(Σ_j |w_j f_j|)², the largest |A|² can be, and the reference's own facts on
molecule boxes (src/lib.rs:1102-1150)."""
import numpy as np
import pytest

from oracle import oracle as O
from pripps_b200 import workloads
from pripps_b200.direct import amplitudes, miller_indices, q_vectors
from pripps_b200.formfactor import formfactors_from_yaml_str

pytestmark = pytest.mark.gpu


def _box(n, seed, L=60.0, kinds=3):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, L, (n, 3)), rng.integers(0, kinds, n), L


@pytest.mark.parametrize("n,n_mol,p_max,weighted", [
    (1, 1, 5, False), (7, 7, 9, False), (1000, 1, 6, False), (2048, 4, 12, True),
    (4500, 3, 8, False), (3000, 1, 20, True), (6000, 2000, 4, False), (2053, 1, 3, False)])
def test_pd_direct_matches_oracle(gpu_ctx, n, n_mol, p_max, weighted):
    xyz, kind, L = _box(n, n + p_max)
    qv = q_vectors(miller_indices(p_max), [L, L * 1.1, L * 0.9])
    rng = np.random.default_rng(1)
    ff = rng.uniform(0.5, 8.0, (3, len(qv)))
    w = rng.uniform(0.0, 2.0, n) if weighted else None
    got = amplitudes(xyz, kind, ff, qv, n_mol, w, gpu_ctx)
    ref = O.direct_rows(xyz, kind, ff, qv, n_mol, w)
    fmax = (np.abs(ff).max(axis=0) * (np.abs(w).sum() if weighted else n)) ** 2
    for c in range(4):
        scale = fmax if c >= 2 else np.sqrt(fmax)
        assert np.max(np.abs(got[:, c] - ref[:, c]) / scale) < 1e-12, c


@pytest.mark.parametrize("n,n_mol,kinds", [(1000, 40, 3), (777, 1, 40), (2100, 7, 17)])
def test_pd_direct_kinds_and_molecule_ends_across_stages(gpu_ctx, n, n_mol, kinds):
    """Form factors of more kinds than the kernel keeps in shared memory (read
    from global memory instead), and molecules that end inside and across the
    kernel's shared-memory stages of points."""
    xyz, kind, L = _box(n, n + kinds, kinds=kinds)
    qv = q_vectors(miller_indices(7), [L, L, L * 1.2])
    rng = np.random.default_rng(2)
    ff = rng.uniform(0.5, 8.0, (kinds, len(qv)))
    w = rng.uniform(0.0, 2.0, n)
    got = amplitudes(xyz, kind, ff, qv, n_mol, w, gpu_ctx)
    ref = O.direct_rows(xyz, kind, ff, qv, n_mol, w)
    fmax = (np.abs(ff).max(axis=0) * np.abs(w).sum()) ** 2
    for c in range(4):
        scale = fmax if c >= 2 else np.sqrt(fmax)
        assert np.max(np.abs(got[:, c] - ref[:, c]) / scale) < 1e-12, c


def _rows_close(got, ref, ff, w, n):
    fmax = (np.abs(ff).max(axis=0) * (np.abs(w).sum() if w is not None else n)) ** 2
    for c in range(4):
        scale = fmax if c >= 2 else np.sqrt(fmax)
        assert np.max(np.abs(got[:, c] - ref[:, c]) / scale) < 1e-12, c


@pytest.mark.parametrize("n,n_mol,p_max,weighted,kinds", [
    (1, 1, 5, False, 3), (1000, 1, 6, False, 3), (2048, 4, 12, True, 3), (4500, 3, 100, False, 3),
    (3000, 1, 40, True, 20), (6000, 2000, 4, False, 3), (2053, 1, 3, False, 1)])
def test_pd_direct_lattice_phase_tables_match_oracle(gpu_ctx, n, n_mol, p_max, weighted, kinds):
    """pd_direct_lattice (per-point phase tables, negative indices by
    conjugation) against the oracle's rows at q = 2π·hkl/L, on a box that is
    not cubic, and against pd_direct at the same vectors."""
    xyz, kind, L = _box(n, n + p_max, kinds=kinds)
    box = [L, L * 1.1, L * 0.9]
    hkl = miller_indices(p_max)
    qv = q_vectors(hkl, box)
    rng = np.random.default_rng(1)
    ff = rng.uniform(0.5, 8.0, (kinds, len(qv)))
    w = rng.uniform(0.0, 2.0, n) if weighted else None
    got = amplitudes(xyz, kind, ff, None, n_mol, w, gpu_ctx, hkl=hkl, box=box)
    _rows_close(got, O.direct_rows(xyz, kind, ff, qv, n_mol, w), ff, w, n)
    _rows_close(got, amplitudes(xyz, kind, ff, qv, n_mol, w, gpu_ctx), ff, w, n)


def test_pd_direct_lattice_arbitrary_indices_and_the_sincos_fallback(gpu_ctx):
    """Unsorted lattice vectors with mixed signs and the zero vector; indices
    beyond the table bound (600) take the sincos kernel; both match the
    oracle."""
    xyz, kind, L = _box(1500, 7, kinds=4)
    box = [L, L * 1.3, L * 0.7]
    rng = np.random.default_rng(5)
    for hmax in (30, 600):
        hkl = rng.integers(-hmax, hmax + 1, (700, 3))
        hkl[0] = 0
        qv = q_vectors(hkl, box)
        ff = rng.uniform(0.5, 8.0, (4, len(qv)))
        got = amplitudes(xyz, kind, ff, None, 3, None, gpu_ctx, hkl=hkl, box=box)
        _rows_close(got, O.direct_rows(xyz, kind, ff, qv, 3), ff, None, len(kind))


def test_single_molecule_box_and_two_identical_molecules(gpu_ctx):
    """N = 1: S_eff ≡ 1 and P ≡ total; two well-separated identical dumbbells:
    the per-molecule form factor equals the one-molecule intensity
    (num_molecules_* test, src/lib.rs:1102-1150)."""
    from pripps_b200 import Pripps, Structure
    ff = formfactors_from_yaml_str("X: { formfactor: !Constant 1.0 }\n"
                                   "Y: { formfactor: !Constant 1.0 }\n")
    pr = Pripps(ff, ctx=gpu_ctx)
    one = Structure(np.array([[0, 0, -3], [0, 0, 3.0]]), [0, 0])
    two = Structure(np.array([[0, 0, -3], [0, 0, 3], [50, 0, -3], [50, 0, 3.0]]), [0, 0, 0, 0])
    single = pr.direct_intensity(one, 30, [200.0] * 3, num_molecules=1)
    assert np.allclose(single.effective_structure_factor, 1.0, atol=1e-9)
    assert np.allclose(single.form_factor, single.total, atol=1e-9)
    box2 = pr.direct_intensity(two, 30, [200.0] * 3, num_molecules=2)
    assert len(box2.form_factor) == len(single.total)
    assert np.allclose(box2.form_factor, single.total, atol=1e-6)


def test_direct_model_with_solvent_matches_oracle_amplitudes(gpu_ctx):
    """DirectModel: cached atom / excluded-volume / hydration amplitudes,
    combined as |A − v·C + c·B|² per vector before the |q| grouping
    (src/explicit.rs:296-357)."""
    from pripps_b200 import ExcludedVolume, Hydration, Pripps, SolventConfig, Structure
    from pripps_b200.direct import average_by_qnorm
    from pripps_b200.solvent import excluded_table
    g = workloads.small_globule(400, 5).globule
    ids = workloads.element_ids()[g.elements]
    s = Structure(g.pos + 40.0, ids)
    m = workloads.foxs()
    box = [90.0, 90.0, 90.0]
    cfg = SolventConfig(ExcludedVolume.fraser_foxs(1.0), Hydration.grid(0.03, spacing=3.1))
    pr = Pripps(m, ctx=gpu_ctx)
    model = pr.direct_model(s, 5, box, cfg)
    got = model.intensity(1.03, 0.02)
    # oracle: the three amplitude sets from the restated rows
    qv = q_vectors(miller_indices(5), box)
    qn = np.sqrt((qv * qv).sum(axis=1))
    used = np.unique(ids)
    kind = np.searchsorted(used, ids)
    A = O.direct_rows(s.pos, kind, m.table(used, qn), qv)
    Cr = O.direct_rows(s.pos, kind, excluded_table(cfg.excluded, m, used, qn, 0.334), qv)
    from pripps_b200.dummies import grid_hydration_dummies
    h = grid_hydration_dummies(s.pos, ids, m, 3.1, 3.0, 1.8)
    water = np.array([[m.form_factor_by_name("H2O").eval(float(q)) for q in qn]])
    B = O.direct_rows(h.positions, np.zeros(len(h), dtype=np.int64), water, qv, 1, h.weights)
    a, c, b = (r[:, 0] + 1j * r[:, 1] for r in (A, Cr, B))
    tot = a - 1.03 * c + 0.02 * b
    q, ref = average_by_qnorm(qn, np.stack([np.abs(tot) ** 2, np.abs(a) ** 2], axis=1))
    assert np.allclose(got.q, q)
    scale = np.abs(a).max() ** 2
    assert np.max(np.abs(got.total - ref[:, 0]) / scale) < 1e-12
    assert np.max(np.abs(got.contributions.atoms - ref[:, 1]) / scale) < 1e-12


def test_lattice_grid_direct_intensity_matches_oracle(gpu_ctx):
    """A lattice q-grid (QGrid.lattice): per-vector |A|² from the device,
    averaged per bin as the reference's QGrid::group (src/q_grid.rs:140-157)."""
    from pripps_b200 import Pripps, Structure
    from pripps_b200.direct import QGrid
    g = workloads.small_globule(300, 3).globule
    ids = workloads.element_ids()[g.elements]
    L = 120.0
    s = Structure(g.pos + L / 2, ids)
    m = workloads.foxs()
    grid = QGrid.lattice([L] * 3, 0.35, 40)
    got = Pripps(m, ctx=gpu_ctx).direct_intensity(s, 0, [L] * 3, grid=grid)
    qv = q_vectors(grid.indices(), [L] * 3)
    qn = np.sqrt((qv * qv).sum(axis=1))
    used = np.unique(ids)
    rows = O.direct_rows(s.pos, np.searchsorted(used, ids), m.table(used, qn), qv)
    q, ref = grid.group(qn, rows[:, 2:3])
    assert np.array_equal(got.q, q)
    assert np.max(np.abs(got.total - ref[:, 0]) / np.abs(ref[:, 0]).max()) < 1e-12
