"""Parity of the CUDA backend with the FP64 oracle, through the C ABI.

Tolerances (stated by the target of this backend):
  PD_FP64          every profile within 1e-10 of the oracle
  PD_FP32_FP64RED  every profile within 1e-5 of the oracle
Cross profiles (AC, AB, CB) change sign, so their error is normalised by
sqrt(self_a·self_b) (see conftest.term_errors); self profiles are relative.

The oracle is used in its compensated form (long double accumulators): on
sums of 10^7+ same-sign terms the reference's own sequential FP64
accumulation drifts by up to ~1e-9 (measured: 1.04e-9 at q = 0 for 10,000
atoms, where every sinc is 1 and the exact value is a product of sums), which
is the oracle's rounding, not the kernel's. The reference-order oracle is
checked beside it at 1e-8.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, term_errors
from oracle import oracle as O
from pripps_b200 import _lib, workloads
from pripps_b200.debye import DebyeRequest, solve

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-5}


def _golden_request(g, precision, solvent):
    return DebyeRequest(np.array(g["positions"]), np.array(g["species"]), np.array(g["ff_atoms"]),
                        np.array(g["ff_excluded"]) if solvent else None,
                        np.array(g["hyd_weights"]) if solvent else None,
                        np.array(g["ff_water"]) if solvent else None,
                        g["qmin"], g["qmax"], g["nq"], None, precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_pepsi_golden(gpu_ctx, precision):
    g = load_golden("pepsi_4lzt.json")
    req = _golden_request(g, precision, False)
    t = solve(req, gpu_ctx)
    oracle = np.array(g["oracle_vacuum"])
    assert np.max(np.abs(t[0] - oracle) / oracle) < TOL[precision]
    assert np.all(t[1:] == 0.0)
    pepsi = np.array(g["pepsi_iat"])
    assert np.max(np.abs(t[0] - pepsi) / pepsi) < g["pepsi_rel_tol"]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_solvent_golden(gpu_ctx, precision):
    g = load_golden("solvent_4lzt.json")
    t = solve(_golden_request(g, precision, True), gpu_ctx)
    err = term_errors(t, np.array(g["oracle_terms"]))
    assert np.all(err < TOL[precision]), err


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sphere_vacuum_1k_full(gpu_ctx, precision):
    """1,000 atoms, nq = 500, the whole grid against the oracle."""
    w = workloads.sphere_vacuum_1k(precision)
    t = solve(w.request, gpu_ctx)
    ref = O.terms_for_request(w.request, precise=True)
    err = term_errors(t, ref)
    assert err[0] < TOL[precision], err
    # I(0) = (Σf)² exactly up to FP64 rounding
    f0 = w.request.ff_atoms[w.request.species, 0]
    assert abs(t[0, 0] - f0.sum() ** 2) <= 1e-12 * f0.sum() ** 2


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sphere_solvent_10k_q_subset(gpu_ctx, precision):
    """10,000 atoms with solvent, nq = 500; oracle on a spread of grid points
    (q = 0, the first steps, the middle and the end)."""
    w = workloads.sphere_solvent_10k(precision)
    t = solve(w.request, gpu_ctx)
    qi = np.array([0, 1, 2, 7, 64, 128, 250, 499])
    ref = O.terms_for_request(w.request, q_index=qi, precise=True)
    err = term_errors(t[:, qi], ref)
    assert np.all(err < TOL[precision]), err
    if precision == "fp64":
        ref_order = O.terms_for_request(w.request, q_index=qi)
        assert np.all(term_errors(t[:, qi], ref_order) < 1e-8)


def _random_request(n, nq, solvent, weighted, seed, precision, qmin=0.0, qmax=0.6):
    rng = np.random.default_rng(seed)
    r = max(3.0, 2.0 * n ** (1 / 3))
    xyz = rng.uniform(-r, r, (n, 3))
    sp = rng.integers(0, 3, n)
    ffA = rng.uniform(1, 8, (3, nq))
    ffC = rng.uniform(0.2, 3, (3, nq)) if solvent else None
    if solvent:
        w = rng.uniform(0, 2, n) if weighted else np.where(rng.random(n) < 0.5, 1.25, 0.0)
        fw = rng.uniform(5, 10, nq)
    else:
        w = fw = None
    return DebyeRequest(xyz, sp, ffA, ffC, w, fw, qmin, qmax, nq, None, precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [1, 2, 3, 33, 127, 129, 200])
@pytest.mark.parametrize("nq", [1, 2, 37, 130])
@pytest.mark.parametrize("mode", ["vacuum", "class", "weighted"])
def test_edge_sizes(gpu_ctx, precision, n, nq, mode):
    req = _random_request(n, nq, mode != "vacuum", mode == "weighted", 100 * n + nq, precision,
                          qmin=0.05 if nq == 1 else 0.0)
    t = solve(req, gpu_ctx)
    ref = O.terms_for_request(req, precise=True)
    err = term_errors(t, ref)
    assert np.all(err < TOL[precision]), (err, t[:, :3], ref[:, :3])


@pytest.mark.parametrize("shape", [(32, 4), (64, 2), (64, 4), (96, 2), (128, 2), (128, 4)])
def test_fp32_every_kernel_shape(gpu_ctx, shape):
    """Each instantiated (q block, pairs per thread) shape against the oracle,
    on a grid whose first block sits in the small-q residual form."""
    K, NP = shape
    lib = _lib.lib()
    ctx = _lib.Context(0)
    try:
        w = workloads.small_globule(2500, 17, nq=300, qmax=0.7, precision="fp32")
        _lib.check(lib.pd_set_tuning(ctx.handle, 2500, 300, 0, K, 512, NP), ctx.handle)
        t = solve(w.request, ctx)
        qi = np.array([0, 1, 2, 3, K - 1, K, K + 1, 150, 299])
        ref = O.terms_for_request(w.request, q_index=qi, precise=True)
        assert np.all(term_errors(t[:, qi], ref) < 1e-5)
    finally:
        ctx.close()


@pytest.mark.parametrize("shape", [(32, 2), (64, 2), (64, 4)])
@pytest.mark.parametrize("grid", ["small_q_first_block", "general_step"])
def test_fp32_weighted_every_kernel_shape(tmp_path, shape, grid):
    """Weighted mode (a hydration weight per atom, as SASA areas give: more
    distinct (species, weight) keys than classes) in each instantiated shape
    against the oracle: once on a grid whose first block sits in the small-q
    residual form, once with a step Δq·2R > π/4 (the general step)."""
    K, NP = shape
    if grid == "small_q_first_block":
        w = workloads.small_globule(2500, 23, nq=300, qmax=0.7, precision="fp32")
        qi = np.array([0, 1, 2, 3, K - 1, K, K + 1, 150, 299])
    else:
        w = workloads.small_globule(2500, 29, nq=60, qmax=3.0, precision="fp32")
        qi = np.arange(0, 60, 7)
    rng = np.random.default_rng(K + NP)
    req = w.request
    req.hyd_weights = req.hyd_weights * rng.uniform(0.05, 1.0, req.n_atoms)
    assert len(np.unique(req.hyd_weights)) > 100
    nq_log2 = int(np.log2(req.nq))
    p = tmp_path / "tune.txt"
    p.write_text(f"fp32 weighted single 11 {nq_log2} {K} 512 {NP} 1.0\n")
    ctx = _lib.Context(0)
    try:
        _lib.check(_lib.lib().pd_tuning_load(ctx.handle, str(p).encode()), ctx.handle)
        plan = C.c_void_p()
        r = req.c_struct()
        _lib.check(_lib.lib().pd_plan_create(ctx.handle, C.byref(r), C.byref(plan)), ctx.handle)
        k, tj, np_ = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _lib.check(_lib.lib().pd_plan_info(plan, C.byref(k), C.byref(tj), C.byref(np_), None,
                                           None, None), None)
        _lib.lib().pd_plan_destroy(ctx.handle, plan)
        assert (k.value, np_.value) == (K, NP)
        t = solve(req, ctx)
        ref = O.terms_for_request(req, q_index=qi, precise=True)
        assert np.all(term_errors(t[:, qi], ref) < 1e-5)
    finally:
        ctx.close()


def test_fp32_small_q_bias(gpu_ctx):
    """Many nearly equal terms: 30,000 atoms in a compact ball at q ≤ 0.01,
    where every sin(q r)/r ≈ q. Sequential FP32 sums of such terms round with
    a bias; the residual form must keep every profile within 1e-5."""
    from pripps_b200 import synth
    g = synth.globule(30_000, (42.0, 42.0, 42.0), 23)
    r32 = workloads.globule_request(g, 0.0, 0.01, 50, True, "fp32")
    r64 = workloads.globule_request(g, 0.0, 0.01, 50, True, "fp64")
    err = term_errors(solve(r32, gpu_ctx), solve(r64, gpu_ctx))
    assert np.all(err < 1e-5), err


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_coincident_atoms(gpu_ctx, precision):
    """Two dummies at the same point contribute sinc(0) = 1 at every q."""
    xyz = np.array([[0, 0, 0], [0, 0, 0], [3.0, 0, 0]])
    req = DebyeRequest(xyz, np.zeros(3), np.ones((1, 9)), None, None, None, 0.0, 0.8, 9, None,
                       precision)
    t = solve(req, gpu_ctx)
    ref = O.terms_for_request(req)
    assert np.max(np.abs(t[0] - ref[0]) / ref[0]) < TOL[precision]


def test_fp32_vs_fp64_large_qr(gpu_ctx):
    """Long pairs at high q (q·r up to ~230): FP32 recurrence against the
    FP64 kernel on a 20,000-atom ellipsoid, q ∈ [0, 1.5], nq = 301."""
    from pripps_b200 import synth
    g = synth.globule(20_000, (80.0, 40.0, 40.0), 11)
    r32 = workloads.globule_request(g, 0.0, 1.5, 301, True, "fp32")
    r64 = workloads.globule_request(g, 0.0, 1.5, 301, True, "fp64")
    t32, t64 = solve(r32, gpu_ctx), solve(r64, gpu_ctx)
    err = term_errors(t32, t64)
    assert np.all(err < 1e-5), err


def test_fp32_vs_fp64_full_size_100k(gpu_ctx):
    """The full 100,000-atom ellipsoid solve (nq = 1,000 on [0, 1]) in both
    forms: every profile of the FP32 recurrence within 1e-5 of the plain FP64
    kernel over the whole grid (the FP64 kernel is held to 1e-10 of the oracle
    on the 1,000- and 10,000-atom cases; the CPU oracle needs hours here).
    Size-independent check beside it: at q = 0 every sinc is 1, so each
    self profile is (sum of its weights)^2 and each cross profile the product
    of the two sums."""
    w32 = workloads.ellipsoid_solvent_100k("fp32")
    w64 = workloads.ellipsoid_solvent_100k("fp64")
    t32, t64 = solve(w32.request, gpu_ctx), solve(w64.request, gpu_ctx)
    err = term_errors(t32, t64)
    assert np.all(err < 1e-5), err
    req = w32.request
    a = req.ff_atoms[req.species, 0]
    c = req.ff_excluded[req.species, 0]
    b = req.hyd_weights * req.ff_water[0]
    sums = {"A": np.sum(a, dtype=np.longdouble), "C": np.sum(c, dtype=np.longdouble),
            "B": np.sum(b, dtype=np.longdouble)}
    exact = [sums["A"] ** 2, sums["C"] ** 2, sums["B"] ** 2, sums["A"] * sums["C"],
             sums["A"] * sums["B"], sums["C"] * sums["B"]]
    for t in (t32, t64):
        for r in range(6):
            assert abs(t[r, 0] - float(exact[r])) <= 1e-12 * abs(float(exact[r])), (r, t[r, 0])


def test_fp32_vs_fp64_trajectory_full_size(gpu_ctx):
    """All 256 frames of the 5,000-atom trajectory (nq = 300) in one batched
    solve per form: the frame-weighted mean of the FP32 form within 1e-5 of
    the FP64 form at every q."""
    t32 = solve(workloads.trajectory_5k_256("fp32").request, gpu_ctx)
    t64 = solve(workloads.trajectory_5k_256("fp64").request, gpu_ctx)
    err = term_errors(t32, t64)
    assert err[0] < 1e-5, err


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_deterministic(gpu_ctx, precision):
    w = workloads.small_globule(3000, 5, nq=97, precision=precision)
    a = solve(w.request, gpu_ctx)
    b = solve(w.request, gpu_ctx)
    assert np.array_equal(a, b)


def test_cached_model_matches_one_shot(gpu_ctx):
    """One kernel result feeds both paths, bit for bit
    (src/lib.rs:535-566, :598-633)."""
    from pripps_b200 import ExcludedVolume, Hydration, Pripps, SolventConfig, Structure
    g = load_golden("solvent_4lzt.json")
    from pripps_b200.formfactor import formfactors_from_yaml_str
    pr = Pripps(workloads.foxs(), ctx=gpu_ctx)
    glob = workloads.small_globule(500, 9).globule
    ids = workloads.element_ids()[glob.elements]
    s = Structure(glob.pos, ids)
    weights = np.where(glob.exposed, 1.1, 0.0)
    cfg = SolventConfig(ExcludedVolume.fraser_foxs(1.0), Hydration.sasa(0.03, weights=weights))
    one = pr.intensity(s, 0.0, 0.3, 20, cfg)
    model = pr.debye_model(s, 0.0, 0.3, 20, cfg)
    cached = model.intensity(1.0, 0.03)
    assert np.array_equal(one.total, cached.total)
    assert one.contributions == cached.contributions
    scaled = SolventConfig(ExcludedVolume.fraser_foxs(1.7))
    one17 = pr.intensity(s, 0.0, 0.2, 8, scaled)
    unit = pr.debye_model(s, 0.0, 0.2, 8, SolventConfig(ExcludedVolume.fraser_foxs(1.0)))
    assert np.array_equal(one17.total, unit.intensity(1.7, 0.0).total)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_trajectory_batch(gpu_ctx, precision):
    """All frames in one launch; the weighted mean against the oracle's
    per-frame profiles combined in frame order (src/trajectory.rs:198-248)."""
    from pripps_b200 import synth
    g = synth.globule(400, (9.0, 9.0, 9.0), 21)
    frames, wts = synth.trajectory(g.pos, 6, 0.5, 21)
    req = workloads.globule_request(g, 0.0, 0.5, 31, True, precision, frames, wts)
    t = solve(req, gpu_ctx)
    acc = np.zeros((6, 31))
    for f in range(6):
        rf = workloads.globule_request(g, 0.0, 0.5, 31, True, precision, frames[f], None)
        acc += wts[f] * O.terms_for_request(rf, precise=True)
    ref = acc / wts.sum()
    err = term_errors(t, ref)
    assert np.all(err < TOL[precision]), err


def test_trajectory_stride_and_weights(gpu_ctx):
    """One-hot weights select a frame; uniform weights give the mean; stride
    renormalises by the consumed weight (src/lib.rs:1027-1099)."""
    from pripps_b200 import Pripps, Structure, synth
    pr = Pripps(workloads.foxs(), precision="fp64", ctx=gpu_ctx)
    g = synth.globule(129, (8.0, 8.0, 8.0), 4)
    s = Structure(g.pos, workloads.element_ids()[g.elements])
    frames = np.stack([g.pos, 1.2 * g.pos])
    run = lambda w, stride: pr.intensity(s, 0.05, 0.3, 8, frames=frames, frame_weights=w,
                                         stride=stride).total
    f0 = run([1.0, 0.0], 1)
    f1 = run([0.0, 1.0], 1)
    avg = run(None, 1)
    s2 = run(None, 2)
    close = lambda a, b: np.all(np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), 1.0))
    assert not close(f0, f1)
    assert close(avg, 0.5 * (f0 + f1))
    assert close(s2, f0)


def test_plan_execute_device_pointers(gpu_ctx):
    """pd_plan_execute on device-resident coordinates gives the pd_solve
    result bit for bit."""
    import torch
    w = workloads.small_globule(2500, 13, nq=150)
    ref = solve(w.request, gpu_ctx)
    lib = _lib.lib()
    r = w.request.c_struct()
    plan = C.c_void_p()
    _lib.check(lib.pd_plan_create(gpu_ctx.handle, C.byref(r), C.byref(plan)), gpu_ctx.handle)
    try:
        xyz = torch.from_numpy(w.request.xyz).cuda()
        out = torch.empty((6, w.request.nq), dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):
            _lib.check(lib.pd_plan_execute(gpu_ctx.handle, plan, xyz.data_ptr(), out.data_ptr(),
                                           stream), gpu_ctx.handle)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref)
    finally:
        lib.pd_plan_destroy(gpu_ctx.handle, plan)


def test_serving_alone_equals_mixed(gpu_ctx):
    """Requests submitted together run interleaved on the device; each result
    equals its solo pd_solve bit for bit."""
    from pripps_b200.serving import Server
    reqs = [workloads.small_globule(n, s, nq=nq, solvent=sol).request
            for n, s, nq, sol in [(3000, 1, 211, True), (700, 2, 97, False), (5000, 3, 150, True),
                                  (1500, 4, 64, True), (9000, 5, 120, False), (40, 6, 33, True)]]
    solo = [solve(r, gpu_ctx) for r in reqs]
    srv = Server(gpu_ctx)
    tickets = [srv.submit(r) for r in reqs]
    outs = [srv.wait(t, timeout_s=120) for t in tickets]
    for a, b in zip(outs, solo):
        assert np.array_equal(a, b)
    times = [srv.times(t) for t in tickets]
    assert all(ts[0] <= ts[1] <= ts[2] for ts in times)


def test_serving_express_lanes_beside_a_large_request(gpu_ctx):
    """Small requests (at most 1e10 pair·q of work) submitted while a large
    one runs go to the high-priority express lanes at admission: more of them,
    and of more kernel variants, than there are express lanes (the rest wait
    for a lane, or after 0.25 s take the steps). Every result equals its solo
    solve bit for bit, and most small requests finish before the large one."""
    from pripps_b200.serving import Server
    big = workloads.small_globule(30_000, 11, nq=400).request  # ≈1.8e11 pair·q
    small = [workloads.small_globule(n, 20 + k, nq=nq, solvent=sol, precision=prec).request
             for k, (n, nq, sol, prec) in enumerate(
                 [(4500, 200, True, "fp32"), (1200, 150, False, "fp32"), (800, 40, True, "fp32"),
                  (2000, 300, True, "fp64"), (6000, 160, True, "fp32"), (500, 500, False, "fp32"),
                  (3000, 100, True, "fp32"), (1000, 30, True, "fp32"), (2500, 250, False, "fp64"),
                  (5000, 120, True, "fp32"), (900, 700, True, "fp32"), (1500, 90, False, "fp32")])]
    solo_big = solve(big, gpu_ctx)
    solo = [solve(r, gpu_ctx) for r in small]
    srv = Server(gpu_ctx)
    tb = srv.submit(big)
    ts = [srv.submit(r) for r in small]
    outs = [srv.wait(t, timeout_s=120) for t in ts]
    assert np.array_equal(srv.wait(tb, timeout_s=120), solo_big)
    for a, b in zip(outs, solo):
        assert np.array_equal(a, b)
    done_big = srv.times(tb)[2]
    assert sum(srv.times(t)[2] < done_big for t in ts) >= len(ts) // 2


def test_serving_burst_of_small_requests(gpu_ctx):
    """Eighty small requests of four kernel variants and two large ones
    submitted at once (one admission pass): the small ones queue for the
    express lanes, each lane launch taking every waiting request of its
    variant. Every result equals its solo solve bit for bit, and the small
    requests finish before the large ones."""
    from pripps_b200.serving import Server
    rng = np.random.default_rng(3)
    specs = [(int(rng.integers(300, 2500)), int(rng.integers(30, 400)), bool(k % 3),
              "fp64" if k % 10 == 0 else "fp32") for k in range(80)]
    small = [workloads.small_globule(n, 100 + k, nq=nq, solvent=sol, precision=prec).request
             for k, (n, nq, sol, prec) in enumerate(specs)]
    big = [workloads.small_globule(25_000, 7 + k, nq=300).request for k in range(2)]
    solo = [solve(r, gpu_ctx) for r in small + big]
    srv = Server(gpu_ctx)
    tickets = [srv.submit(r) for r in big + small]
    outs = [srv.wait(t, timeout_s=180) for t in tickets]
    for a, b in zip(outs, solo[-2:] + solo[:-2]):
        assert np.array_equal(a, b)
    done_big = min(srv.times(t)[2] for t in tickets[:2])
    assert sum(srv.times(t)[2] < done_big for t in tickets[2:]) >= 70


def test_serving_budget_admission(gpu_ctx):
    """With a budget that fits about one request, the loop admits them one at
    a time and still completes all; a request that can never fit fails with
    PD_EBUDGET."""
    from pripps_b200.errors import DeviceError
    from pripps_b200.serving import Server
    # each request holds about 1.2 MB of device memory (pd_request_device_bytes)
    reqs = [workloads.small_globule(4000, s, nq=200).request for s in range(3)]
    ctx = _lib.Context(0, mem_budget_bytes=2 << 20)
    try:
        srv = Server(ctx)
        solo = [solve(r, gpu_ctx) for r in reqs]
        ts = [srv.submit(r) for r in reqs]
        for t, ref in zip(ts, solo):
            assert np.array_equal(srv.wait(t, timeout_s=120), ref)
        big = workloads.small_globule(20_000, 1, nq=900).request  # about 11 MB
        t = srv.submit(big)
        with pytest.raises(DeviceError):
            srv.wait(t, timeout_s=120)
    finally:
        ctx.close()


def test_serving_cancel(gpu_ctx):
    from pripps_b200.errors import DeviceError
    from pripps_b200.serving import Server
    srv = Server(gpu_ctx)
    big = workloads.small_globule(30_000, 3, nq=600).request
    t1 = srv.submit(big)
    t2 = srv.submit(workloads.small_globule(500, 4, nq=40).request)
    srv.cancel(t1)
    with pytest.raises(DeviceError) as ei:
        srv.wait(t1, timeout_s=120)
    assert ei.value.code == _lib.PD_ECANCELED
    out = srv.wait(t2, timeout_s=120)
    assert out.shape == (6, 40)


def test_autotune_and_fp32_probe(gpu_ctx):
    lib = _lib.lib()
    assert lib.pd_autotune(gpu_ctx.handle, 3000, 200, 0) == 0
    k, tj, npt = C.c_uint32(), C.c_uint32(), C.c_uint32()
    lib.pd_get_tuning(gpu_ctx.handle, 3000, 200, 0, C.byref(k), C.byref(tj), C.byref(npt))
    assert k.value in (32, 64, 96, 128) and tj.value % 32 == 0 and npt.value in (1, 2, 4)
    w = workloads.small_globule(3000, 7, nq=200)
    t = solve(w.request, gpu_ctx)
    ref = O.terms_for_request(w.request, q_index=np.array([0, 1, 50, 199]), precise=True)
    assert np.all(term_errors(t[:, [0, 1, 50, 199]], ref) < 1e-5)
    a, b = C.c_double(), C.c_double()
    assert lib.pd_measure_fp32_peak(gpu_ctx.handle, C.byref(a), C.byref(b)) == 0
    assert 10.0 < a.value < 200.0


def test_serving_more_kernel_variants_than_lanes(gpu_ctx):
    """Requests of six kernel variants in flight together (FP32 class K = 128
    and K = 64, FP32 weighted, FP64 class, FP64 weighted, grid solvent with
    lattice sets): a step runs at most four variants, the others wait for the
    next step; every result still equals its solo solve bit for bit."""
    from pripps_b200.serving import Server
    rng = np.random.default_rng(3)
    reqs = [
        workloads.small_globule(6000, 1, nq=300, precision="fp32").request,   # K = 128
        workloads.small_globule(2000, 2, nq=90, precision="fp32").request,    # K = 64
        workloads.small_globule(3000, 3, nq=120, precision="fp64").request,   # FP64 class
    ]
    w = workloads.small_globule(1500, 4, nq=70, precision="fp32").request
    w.hyd_weights = rng.uniform(0.0, 3.0, w.n_atoms)                      # > 48 weights
    reqs.append(w)
    w64 = workloads.small_globule(1200, 5, nq=50, precision="fp64").request
    w64.hyd_weights = rng.uniform(0.0, 3.0, w64.n_atoms)
    reqs.append(w64)
    g = workloads.small_globule(400, 6).globule
    reqs.append(workloads.grid_solvent_request(g, 0.0, 0.5, 60, "fp32", 1.4))
    solo = [solve(r, gpu_ctx) for r in reqs]
    srv = Server(gpu_ctx)
    for _ in range(2):  # twice, so the second round finds the graphs built
        tickets = [srv.submit(r) for r in reqs]
        outs = [srv.wait(t, timeout_s=300) for t in tickets]
        for a, b in zip(outs, solo):
            assert np.array_equal(a, b)
