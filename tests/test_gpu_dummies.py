"""Solvent dummies at their own positions on the device: the union request
(atoms + grid excluded-volume cells + grid hydration points) through the C
ABI against the oracle's build_model with the three sets kept apart
(src/debye.rs:83-130), in both precision forms. The grid sets travel as
lattice sets: their self sums come from exact pair counts per squared
lattice offset, everything else from the pair kernels.

Tolerances as for the colocated path: FP64 form 1e-10, FP32 form 1e-5 per
profile (cross profiles normalised by sqrt(self_a·self_b))."""
import numpy as np
import pytest

from conftest import term_errors
from oracle import oracle as O
from pripps_b200 import workloads
from pripps_b200.debye import solve

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-5}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n,seed,spacing,nq,qmax", [(300, 3, 1.3, 60, 0.6), (120, 8, 1.0, 37, 0.9),
                                                    (700, 5, 1.6, 130, 0.5)])
def test_grid_solvent_against_separate_sets(gpu_ctx, precision, n, seed, spacing, nq, qmax):
    g = workloads.small_globule(n, seed).globule
    req = workloads.grid_solvent_request(g, 0.0, qmax, nq, precision, spacing)
    t = solve(req, gpu_ctx)
    sets = workloads.grid_solvent_sets(req, n)
    ref = O.build_model_sets(*sets, 0.0, qmax, nq, precise=True).T
    err = term_errors(t, ref)
    assert np.all(err < TOL[precision]), err


def test_grid_solvent_10k_fp32_vs_fp64(gpu_ctx):
    """The 10,000-atom sphere with 1 Å grid excluded volume and a grid
    hydration shell (~111,000 points, nq = 500): FP32 form within 1e-5 of the
    FP64 form at every q; FP64 form against the oracle's separate-set sums
    on a spread of grid points."""
    w32 = workloads.sphere_grid_solvent_10k("fp32")
    w64 = workloads.sphere_grid_solvent_10k("fp64")
    t32, t64 = solve(w32.request, gpu_ctx), solve(w64.request, gpu_ctx)
    assert np.all(term_errors(t32, t64) < 1e-5), term_errors(t32, t64)
    # q = 0: each self profile is the square of its set's summed weights
    req = w64.request
    n = w64.globule.pos.shape[0]
    a_xyz, a_sp, ffA, c_xyz, c_kind, ffC, b_xyz, b_w, ffW = workloads.grid_solvent_sets(req, n)
    sa = np.sum(ffA[a_sp, 0], dtype=np.longdouble)
    sc = np.sum(ffC[c_kind, 0], dtype=np.longdouble)
    sb = np.sum(b_w * ffW[0], dtype=np.longdouble)
    exact = [sa * sa, sc * sc, sb * sb, sa * sc, sa * sb, sc * sb]
    for t in (t32, t64):
        for r in range(6):
            assert abs(t[r, 0] - float(exact[r])) <= 1e-12 * abs(float(exact[r])), r


def test_trajectory_with_grid_solvent_rebuilds_dummies_per_frame(gpu_ctx):
    """With dummies away from the atoms every frame gets its own dummy sets
    (src/trajectory.rs:198-223 runs the calculator per frame); the weighted
    mean of the per-frame totals equals the frames solved one by one."""
    from pripps_b200 import ExcludedVolume, Hydration, Pripps, SolventConfig, Structure
    from pripps_b200.debye import combine, make_request
    from pripps_b200.formfactor import linear_q_values
    g = workloads.small_globule(200, 12).globule
    ids = workloads.element_ids()[g.elements]
    s = Structure(g.pos, ids)
    rng = np.random.default_rng(5)
    frames = g.pos[None] + rng.normal(0, 0.4, (4, len(ids), 3))
    wts = np.array([0.1, 0.4, 0.2, 0.3])
    cfg = SolventConfig(ExcludedVolume.grid(1.4, volume_scale=1.05),
                        Hydration.grid(0.02, spacing=2.8))
    pr = Pripps(workloads.foxs(), precision="fp64", ctx=gpu_ctx)
    got = pr.intensity(s, 0.0, 0.5, 30, cfg, frames=frames, frame_weights=wts)
    q = linear_q_values(0.0, 0.5, 30)
    ref = np.zeros(30)
    for f, wf in zip(frames, wts):
        req = make_request(Structure(f, ids), workloads.foxs(), q, 0.0, 0.5, cfg, "fp64")
        ref += wf * combine(solve(req, gpu_ctx), 1.05, 0.02)
    ref /= wts.sum()
    assert np.max(np.abs(got.total - ref) / np.abs(ref)) < 1e-12


def test_point_off_its_lattice_is_refused(gpu_ctx):
    """A lattice species with a point moved off the grid: the device flags it
    and the solve returns PD_EINVAL instead of a result."""
    from pripps_b200.errors import ValidationError
    g = workloads.small_globule(150, 2).globule
    req = workloads.grid_solvent_request(g, 0.0, 0.5, 20, "fp32", 1.2)
    sp = req.lattices[1][0]
    k = np.flatnonzero(req.species == sp)[3]
    req.xyz[k, 0] += 0.01
    with pytest.raises(ValidationError):
        solve(req, gpu_ctx)
    # and a correct request on the same context still solves
    ok = workloads.grid_solvent_request(g, 0.0, 0.5, 20, "fp32", 1.2)
    assert np.all(np.isfinite(solve(ok, gpu_ctx)))


def test_lattice_sums_equal_pair_kernel_sums_in_fp64(gpu_ctx):
    """The lattice path against the plain FP64 pair kernel on the same union
    (lattices removed from the request): every profile within 1e-12."""
    g = workloads.small_globule(500, 4).globule
    req = workloads.grid_solvent_request(g, 0.0, 0.7, 90, "fp64", 1.1)
    a = solve(req, gpu_ctx)
    req.lattices = None
    b = solve(req, gpu_ctx)
    assert np.all(term_errors(a, b) < 1e-12), term_errors(a, b)
