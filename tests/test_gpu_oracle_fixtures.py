"""The solvent workloads against the CPU oracle itself, through the C ABI.

Fixtures (tests/golden/make_oracle_fixtures.py, compensated FP64 oracle):
  oracle_sphere_solvent_10k.json      10,000 atoms, nq = 500: the whole grid
  oracle_ellipsoid_solvent_100k.json  100,000 atoms, nq = 1,000: a q subset
                                      (q = 0, small q, the first and deepest
                                      minima, both sides of a q-block seam, qmax)
  oracle_ellipsoid_sasa_20k.json      20,000 atoms with a hydration weight per
                                      atom (weighted mode), nq = 512: q = 0,
                                      small q, a q-block seam, every minimum of
                                      the atoms profile, qmax

Tolerances: PD_FP64 within 1e-10 and PD_FP32_FP64RED within 1e-5 on every
profile; self profiles relative, cross profiles normalised by
sqrt(self_a·self_b) (conftest.term_errors). Each fixture names the SHA-256 of
its inputs; the CPU test below checks that the seeded generators still
produce them.
"""
import numpy as np
import pytest

from conftest import GOLDEN, load_golden, request_digest, term_errors
from pripps_b200 import workloads
from pripps_b200.debye import solve

TOL = {"fp64": 1e-10, "fp32": 1e-5}
FIXTURES = {
    "sphere_solvent_10k": ("oracle_sphere_solvent_10k.json", workloads.sphere_solvent_10k),
    "ellipsoid_solvent_100k": ("oracle_ellipsoid_solvent_100k.json",
                               workloads.ellipsoid_solvent_100k),
    "ellipsoid_sasa_20k": ("oracle_ellipsoid_sasa_20k.json", workloads.ellipsoid_sasa_20k),
}


def _fixture(name):
    fname, make = FIXTURES[name]
    if not (GOLDEN / fname).exists():
        pytest.skip(f"{fname} not generated (tests/golden/make_oracle_fixtures.py)")
    return load_golden(fname), make


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_fixture_inputs_match_generator(name):
    """CPU: the seeded workload generator reproduces the fixture's inputs."""
    g, make = _fixture(name)
    w = make("fp32")
    assert request_digest(w.request) == g["input_sha256"]
    assert (w.request.n_atoms, w.request.nq) == (g["n_atoms"], g["nq"])
    ref = np.array(g["oracle_terms"])
    assert ref.shape == (6, len(g["q_index"]))
    assert np.all(ref[:3] > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_against_oracle_fixture(gpu_ctx, name, precision):
    g, make = _fixture(name)
    w = make(precision)
    assert request_digest(w.request) == g["input_sha256"], "workload generator changed"
    t = solve(w.request, gpu_ctx)
    qi = np.array(g["q_index"])
    err = term_errors(t[:, qi], np.array(g["oracle_terms"]))
    assert np.all(err < TOL[precision]), dict(zip(g["rows"], err))
