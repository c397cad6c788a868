"""Streamed trajectory averages (pd_stream_*) against the one-shot batched
solve of the same frames: the frame loop of trajectory_average
(src/trajectory.rs:198-248) fed frame by frame."""
import numpy as np
import pytest

from conftest import term_errors
from pripps_b200 import _lib, workloads
from pripps_b200.debye import DebyeRequest, TrajectoryStream, solve
from pripps_b200.errors import ValidationError

pytestmark = pytest.mark.gpu


def _frames(n_atoms=800, n_frames=70, seed=3, solvent=False, precision="fp64"):
    w = workloads.small_globule(n_atoms, seed, nq=45, solvent=solvent, precision=precision)
    rng = np.random.default_rng(seed)
    frames = w.request.xyz[None] + rng.normal(0, 0.4, (n_frames, n_atoms, 3))
    weights = rng.exponential(1.0, n_frames)
    return w.request, frames, weights


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("solvent", [False, True])
@pytest.mark.parametrize("batch,chunk", [(16, 7), (32, 32), (1, 5), (64, 70)])
def test_stream_equals_batched_solve(gpu_ctx, precision, solvent, batch, chunk):
    req, frames, weights = _frames(solvent=solvent, precision=precision)
    ref = solve(DebyeRequest(frames, req.species, req.ff_atoms, req.ff_excluded, req.hyd_weights,
                             req.ff_water, req.qmin, req.qmax, req.nq, weights, precision),
                gpu_ctx)
    st = TrajectoryStream(req, batch, gpu_ctx)
    for a in range(0, len(frames), chunk):
        st.push(frames[a:a + chunk], weights[a:a + chunk])
    got = st.finish()
    # same per-frame terms, summed in another grouping: FP64 rounding only
    assert np.all(term_errors(got, ref) < 1e-12), term_errors(got, ref)


def test_stream_through_pripps_with_a_frame_iterator(gpu_ctx):
    """Pripps.intensity with a generator of frames streams them; stride and
    per-original-frame weights as in the reference (src/trajectory.rs:56-61)."""
    from pripps_b200 import Pripps, Structure
    w = workloads.small_globule(500, 2)
    g = w.globule
    ids = workloads.element_ids()[g.elements]
    rng = np.random.default_rng(1)
    frames = g.pos[None] + rng.normal(0, 0.3, (21, len(ids), 3))
    wts = rng.random(21) + 0.1
    pr = Pripps(workloads.foxs(), precision="fp64", ctx=gpu_ctx)
    s = Structure(g.pos, ids)
    arr = pr.intensity(s, 0.0, 0.4, 25, frames=frames, frame_weights=wts, stride=2)
    it = pr.intensity(s, 0.0, 0.4, 25, frames=(f for f in frames), frame_weights=iter(wts),
                      stride=2)
    assert np.max(np.abs(arr.total - it.total) / np.abs(arr.total)) < 1e-12


def test_stream_rejects_zero_weight_sum_and_empty(gpu_ctx):
    req, frames, _ = _frames(n_atoms=100, n_frames=4)
    st = TrajectoryStream(req, 8, gpu_ctx)
    st.push(frames[:2], np.array([1.0, -1.0]))
    with pytest.raises(ValidationError):
        st.finish()
    st = TrajectoryStream(req, 8, gpu_ctx)
    with pytest.raises(ValidationError):
        st.finish()
    st = TrajectoryStream(req, 8, gpu_ctx)
    bad = frames[:1].copy()
    bad[0, 3, 1] = np.nan
    with pytest.raises(ValidationError):
        st.push(bad)
    st.push(frames[:3])
    assert np.all(np.isfinite(st.finish()))
