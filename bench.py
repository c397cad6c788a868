"""Debye pair·q throughput on B200: FP32-recurrence kernel vs plain FP64, with
the reference's CPU Debye (its FP64 restatement) timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ellipsoid_solvent_100k] [--precision fp32]

One step = one full six-profile Debye solve of the workload (100,000 atoms in
an 80×40×40 Å ellipsoid, FoXS excluded volume + surface hydration, nq = 1,000
on [0, 1] Å⁻¹ by default). `value` is pair·q/s with the coordinates resident
in HBM (pd_plan_execute), `e2e` the same metric through the blocking C-ABI
call with host buffers (pd_solve: plan, upload, kernels, download). Work unit:
one unordered atom pair at one q, P = N(N-1)/2·nq per solve.

With --gpus N (torchrun) the ranks split one solve: rank r runs every N-th
tile in cost order (pd_plan_set_shard) and one NCCL all-reduce of the 6·nq
partial profiles completes the step ("scaling": "strong"; the step time is
the max over ranks). Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Debye pair·q evals/s (FP32 recurrence, FP64 reduction)"
UNIT = "pair·q/s"
# FP32 flops of one pair·q in the inner loop. Class mode: the d-step (FFMA,
# 2) and the v-step (FADD, 1) of the recurrence, and the accumulation — an add
# of terms whose weight 1/r the recurrence state already carries (FADD, 1) when
# Δq·(largest pair distance) <= π/4, else an FFMA with the weight (2).
# Weighted mode (a weight per atom): the same step and a second accumulator
# of the terms times w_j (FFMA, 2); with the general step both accumulations
# are FFMAs with the weight.
FLOPS_PER_PAIRQ = {"class": 4, "class_general_step": 5, "weighted": 6,
                   "weighted_general_step": 7}
# FP32 pipe slots (lane operations) of one pair·q: three with one
# accumulator, four with two.
SLOTS_PER_PAIRQ = {"class": 3, "class_general_step": 3, "weighted": 4,
                   "weighted_general_step": 4}
PROFILES = ("atoms", "excluded", "hydration", "atom_excluded", "atom_hydration",
            "excluded_hydration")


def profile_errors(got, ref):
    """Per-profile max error of [6, m] tables: relative for the three self
    profiles (>= 0); the cross profiles, which change sign, normalised by
    sqrt(self_a·self_b) (the Cauchy-Schwarz bound of a cross term). Rows that
    are zero in both (no solvent) give 0."""
    err = []
    pairs = {3: (0, 1), 4: (0, 2), 5: (1, 2)}
    for r in range(6):
        d = np.abs(got[r] - ref[r])
        scale = np.abs(ref[r]) if r < 3 else np.sqrt(np.abs(ref[pairs[r][0]] * ref[pairs[r][1]]))
        m = scale > 0
        e = float(np.max(d[m] / scale[m])) if m.any() else 0.0
        if np.any(d[~m] > 0):
            e = float("inf")
        err.append(e)
    return err


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
                power.append(float(p[3]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_median": statistics.median(power) if power else None}


def cpu_sample(w, n_sample=6000, n_q=0, threads=0):
    """Time the FP64 oracle (the reference's Debye code restated, q-parallel
    on host threads) on a bounded sample of the workload: the first
    `n_sample` atoms and `n_q` grid points spread over the q range (n_q <= 0:
    two per host core, so that every core has work). Returns (rate, pair·q,
    seconds, description, threads used)."""
    from oracle import oracle as O
    req = w.request
    n = min(n_sample, req.n_atoms)
    cores = os.cpu_count() or 1
    if n_q <= 0:
        n_q = max(16, 2 * cores)
    qi = np.unique(np.linspace(0, req.nq - 1, n_q).astype(np.int64)).astype(np.uint32)
    xyz = (req.xyz[0] if req.xyz.ndim == 3 else req.xyz)[:n]
    t0 = time.perf_counter()
    if w.name == "sphere_grid_solvent_10k":
        # The reference sums the three sets apart (3 self + 3 cross sums, the
        # union's pairs once): sample the same fraction of each set.
        from pripps_b200.workloads import grid_solvent_sets
        a_xyz, a_sp, ffA, c_xyz, c_kind, ffC, b_xyz, b_w, ffW = grid_solvent_sets(
            req, w.globule.pos.shape[0])
        f = n / req.n_atoms
        na, nc, nb = (max(1, int(round(f * len(x)))) for x in (a_xyz, c_xyz, b_xyz))
        n = na + nc + nb
        O.build_model_sets(a_xyz[:na], a_sp[:na], ffA, c_xyz[:nc], c_kind[:nc], ffC,
                           b_xyz[:nb], b_w[:nb], ffW, req.qmin, req.qmax, req.nq, qi, threads)
    elif req.ff_excluded is None and req.hyd_weights is None:
        O.vacuum(xyz, req.species[:n], req.ff_atoms, req.qmin, req.qmax, req.nq, qi, threads)
    else:
        O.build_model(xyz, req.species[:n], req.ff_atoms, req.ff_excluded,
                      None if req.hyd_weights is None else req.hyd_weights[:n], req.ff_water,
                      req.qmin, req.qmax, req.nq, qi, threads)
    dt = time.perf_counter() - t0
    pq = n * (n - 1) // 2 * len(qi)
    return (pq / dt, pq, dt, f"first {n} of {req.n_atoms} atoms × {len(qi)} of {req.nq} q points",
            min(cores, len(qi)))


def run_reference(args, ws, rank):
    """The reference arm: the FP64 CPU restatement of the reference's Debye
    path on all host cores, each step a bounded sample of the workload."""
    if rank != 0:
        return
    from pripps_b200 import workloads
    w = workloads.WORKLOADS[args.workload](args.precision)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(w, args.cpu_atoms, args.cpu_q)
    rates, times = [], []
    sample = None
    for _ in range(args.steps):
        rate, pq, dt, sample, cores = cpu_sample(w, args.cpu_atoms, args.cpu_q)
        rates.append(rate)
        times.append(dt)
    pq_total = pq * len(times)
    value = pq_total / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(args, w),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict(args, w):
    req = w.request
    solvent = "vacuum"
    if req.ff_excluded is not None:
        solvent = "foxs_fraser_excluded" + ("+surface_hydration" if req.hyd_weights is not None else "")
    return {"workload": w.name, "n_atoms": req.n_atoms, "nq": req.nq,
            "q_range": [req.qmin, req.qmax], "n_frames": req.n_frames, "solvent": solvent,
            "precision_form": args.precision, "pairs_per_solve": w.pairs,
            "pair_q_per_step": w.pair_q,
            "l2": "flushed between timed steps (256 MiB write outside the timed events)"}


def load_traffic(workload):
    """DRAM bytes per pair-kernel launch from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get(workload, {}).get("dram_bytes_per_launch")
    except (ValueError, OSError):
        return None


def run_ours(args, ws, rank, local):
    import torch

    from pripps_b200 import _lib, workloads
    from pripps_b200.debye import solve

    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    w = workloads.WORKLOADS[args.workload](args.precision)
    req = w.request
    ctx = _lib.Context(local)
    lib = _lib.lib()

    # FP32 issue peak: best of three probe runs (a single short probe reads a
    # few % low when the power state is still settling)
    peak_ffma, peak_ffma2 = C.c_double(0.0), C.c_double(0.0)
    for _ in range(3):
        a, b = C.c_double(), C.c_double()
        _lib.check(lib.pd_measure_fp32_peak(ctx.handle, C.byref(a), C.byref(b)), ctx.handle)
        peak_ffma.value = max(peak_ffma.value, a.value)
        peak_ffma2.value = max(peak_ffma2.value, b.value)

    # ---- device-resident path
    r = req.c_struct()
    plan = C.c_void_p()
    _lib.check(lib.pd_plan_create(ctx.handle, C.byref(r), C.byref(plan)), ctx.handle)
    if ws > 1:
        _lib.check(lib.pd_plan_set_shard(ctx.handle, plan, rank, ws), ctx.handle)
    kb, tj, npt, ntile, dbytes, ubytes = (C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64(),
                                          C.c_uint64(), C.c_uint64())
    lib.pd_plan_info(plan, C.byref(kb), C.byref(tj), C.byref(npt), C.byref(ntile), C.byref(dbytes),
                     C.byref(ubytes))
    from_table = C.c_int(0)
    lib.pd_tuning_lookup(ctx.handle, C.byref(r), None, None, None, C.byref(from_table))
    xyz = torch.from_numpy(req.xyz).to(f"cuda:{local}")
    out = torch.empty((6, req.nq), dtype=torch.float64, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def execute():
        _lib.check(lib.pd_plan_execute(ctx.handle, plan, xyz.data_ptr(), out.data_ptr(), sp),
                   ctx.handle)
        if ws > 1:
            torch.distributed.all_reduce(out, op=torch.distributed.ReduceOp.SUM)

    for _ in range(args.warmup):
        execute()
        flush.zero_()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    lib.pd_plan_set_profiling(ctx.handle, plan, 1)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = ctx.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for i in range(args.steps):
        starts[i].record(stream)
        execute()
        ends[i].record(stream)
        flush.zero_()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    launches = ctx.launch_count() - launches0
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    pair_ms, n_pair = C.c_double(), C.c_uint64()
    _lib.check(lib.pd_plan_pair_kernel_ms(ctx.handle, plan, C.byref(pair_ms), C.byref(n_pair)),
               ctx.handle)
    lib.pd_plan_set_profiling(ctx.handle, plan, 0)
    if ws > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = w.pair_q / (ms_per_step * 1e-3)
    result_dev = out.cpu().numpy()

    # ---- plain FP64 kernel on the same structure (bounded q grid)
    fp64 = None
    parity = None
    if rank == 0 and not args.no_fp64:
        r64 = w.with_grid(args.fp64_nq, "fp64")
        p64 = C.c_void_p()
        c64 = r64.c_struct()
        _lib.check(lib.pd_plan_create(ctx.handle, C.byref(c64), C.byref(p64)), ctx.handle)
        out64 = torch.empty((6, r64.nq), dtype=torch.float64, device=f"cuda:{local}")
        _lib.check(lib.pd_plan_execute(ctx.handle, p64, xyz.data_ptr(), out64.data_ptr(), sp),
                   ctx.handle)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(lib.pd_plan_execute(ctx.handle, p64, xyz.data_ptr(), out64.data_ptr(), sp),
                   ctx.handle)
        e1.record(stream)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1)
        pq64 = w.pairs * r64.nq * r64.n_frames
        lib.pd_plan_destroy(ctx.handle, p64)
        # accuracy of the timed FP32 result against the FP64 kernel: on a
        # grid whose points are every d-th point of the timed grid (d divides
        # nq - 1), else on a separate grid solved by both forms
        steps = [d for d in range(1, req.nq) if (req.nq - 1) % d == 0 and
                 8 <= (req.nq - 1) // d <= 63]
        if steps:
            d = min(steps)
            rp = w.with_grid((req.nq - 1) // d + 1, "fp64")
            ours, how = result_dev[:, ::d], f"every {d}th point of the timed grid"
        else:
            rp, ours, how = r64, None, f"a {r64.nq}-point grid solved by both forms"
        pp = C.c_void_p()
        cp = rp.c_struct()
        _lib.check(lib.pd_plan_create(ctx.handle, C.byref(cp), C.byref(pp)), ctx.handle)
        outp = torch.empty((6, rp.nq), dtype=torch.float64, device=f"cuda:{local}")
        _lib.check(lib.pd_plan_execute(ctx.handle, pp, xyz.data_ptr(), outp.data_ptr(), sp),
                   ctx.handle)
        torch.cuda.synchronize()
        lib.pd_plan_destroy(ctx.handle, pp)
        ref64 = outp.cpu().numpy()
        if ours is None:
            r32 = w.with_grid(r64.nq, args.precision)
            p32 = C.c_void_p()
            c32 = r32.c_struct()
            _lib.check(lib.pd_plan_create(ctx.handle, C.byref(c32), C.byref(p32)), ctx.handle)
            _lib.check(lib.pd_plan_execute(ctx.handle, p32, xyz.data_ptr(), outp.data_ptr(), sp),
                       ctx.handle)
            torch.cuda.synchronize()
            lib.pd_plan_destroy(ctx.handle, p32)
            ours = outp.cpu().numpy()
        parity = {"max_err_vs_fp64_kernel": dict(zip(PROFILES, profile_errors(ours, ref64))),
                  "q_points": int(rp.nq), "grid": how, "tolerance": 1e-5,
                  "normalisation": "self profiles relative; cross profiles by "
                                   "sqrt(self_a·self_b)"}
        fp64 = {"value": pq64 / (ms64 * 1e-3), "unit": UNIT, "nq": r64.nq, "ms": ms64,
                "fp32_over_fp64": (w.pair_q / (ms_per_step * 1e-3)) / (pq64 / (ms64 * 1e-3))}

    # ---- end to end through the C ABI with host buffers: every step plans
    # the request on the host, uploads it and downloads the result (N = 1:
    # the blocking pd_solve; N > 1: a plan of this rank's tiles, the
    # coordinates from pinned memory, the all-reduce and the download)
    e2e_times = []
    res_host = None
    xyz_pinned = torch.from_numpy(req.xyz).pin_memory() if ws > 1 else None
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        if ws > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        if ws == 1:
            res_host = solve(req, ctx)  # pd_solve: plan, upload, kernels, download
        else:
            pe = C.c_void_p()
            _lib.check(lib.pd_plan_create(ctx.handle, C.byref(r), C.byref(pe)), ctx.handle)
            _lib.check(lib.pd_plan_set_shard(ctx.handle, pe, rank, ws), ctx.handle)
            xyz.copy_(xyz_pinned, non_blocking=True)
            _lib.check(lib.pd_plan_execute(ctx.handle, pe, xyz.data_ptr(), out.data_ptr(), sp),
                       ctx.handle)
            torch.distributed.all_reduce(out, op=torch.distributed.ReduceOp.SUM)
            res_host = out.cpu().numpy()
            lib.pd_plan_destroy(ctx.handle, pe)
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_times.append(dt)
    e2e_ms = 1e3 * sum(e2e_times) / len(e2e_times) if e2e_times else float("nan")
    if ws > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    same = bool(np.array_equal(res_host, result_dev)) if res_host is not None else None
    lib.pd_plan_destroy(ctx.handle, plan)
    secondary = None
    if rank == 0 and ws == 1 and not args.no_secondary:
        secondary = run_secondary(ctx, args, local)

    if rank == 0:
        mode = kernel_mode(req)
        flops = FLOPS_PER_PAIRQ[mode]
        slots = SLOTS_PER_PAIRQ[mode]
        launch_ms = pair_ms.value / max(n_pair.value, 1)
        # Pairs of a lattice set with itself are counted, not summed by the
        # pair kernel (see pd_lattice): the roofline counts the kernel's pairs.
        lat_pairs = 0
        for lat in (req.lattices or []):
            m = int(np.count_nonzero(req.species == lat[0]))
            lat_pairs += m * (m - 1) // 2
        kernel_pair_q = (w.pairs - lat_pairs) * req.nq * req.n_frames
        achieved = flops * kernel_pair_q / (launch_ms * 1e-3) / 1e12
        peak = peak_ffma.value
        theoretical = 2 * 128 * 148 * (clk["sm_max_mhz"] or 1965.0) * 1e-6
        # The fixed accounting constants of an angle-addition recurrence with
        # one accumulator (vacuum, 8 FLOP) or four (six colocated profiles,
        # 14 FLOP) per pair·q; this kernel executes `flops` per pair·q.
        solvent = req.ff_excluded is not None or req.hyd_weights is not None
        fixed = 14 if solvent else 8
        fixed_achieved = fixed * kernel_pair_q / (launch_ms * 1e-3) / 1e12
        cpu = None
        if not args.no_cpu and ws == 1:  # the host-core baseline is an N = 1 figure
            rate, pq, dt, sample, used = cpu_sample(w, args.cpu_atoms, args.cpu_q)
            cpu = {"value": rate, "unit": UNIT, "cores": used, "kind": "port",
                   "sample": sample, "seconds": dt}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config_dict(args, w),
            "e2e": {"value": w.pair_q / (e2e_ms * 1e-3), "unit": UNIT,
                    "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(ubytes.value) if ws == 1 else int(req.xyz.nbytes),
                    "d2h_bytes_per_step": 6 * req.nq * 8,
                    "same_result_as_device_path": same},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": load_traffic(w.name),
                         "kernel": "pd_pairs_fp32", "flops_per_pair_q": flops,
                         "fp32_pipe": {
                             "lane_ops_per_pair_q": slots,
                             "achieved_tops": slots * kernel_pair_q / (launch_ms * 1e-3) / 1e12,
                             "peak_tops": peak / 2.0,
                             "frac": slots * kernel_pair_q / (launch_ms * 1e-3) / 1e12 /
                                     (peak / 2.0),
                             "note": "the kernel is bound by FP32 pipe slots: each pair·q "
                                     f"takes {slots} FP32 lane operations ({mode} mode) "
                                     f"for {flops} FLOP; an FADD fills a slot for 1 FLOP, "
                                     "so the FLOP fraction tops out at "
                                     f"{flops}/{2 * slots} of the FFMA peak and the slot "
                                     "fraction at 1"},
                         "kernel_pair_q_per_launch": kernel_pair_q,
                         "kernel_ms_per_launch": launch_ms,
                         "peak_source": "measured FFMA probe (pd_measure_fp32_peak), best of "
                                        "3 in this run",
                         "peak_ffma2_tflops": peak_ffma2.value,
                         "theoretical_peak_tflops_at_max_clock": theoretical,
                         "frac_of_theoretical": achieved / theoretical,
                         "fixed_accounting": {
                             "flops_per_pair_q": fixed, "achieved": fixed_achieved,
                             "frac_of_measured": fixed_achieved / peak,
                             "note": "recurrence-equivalent FLOP rate: a kernel doing the "
                                     "textbook angle-addition step plus one accumulator per "
                                     "profile term would need this rate; this kernel executes "
                                     f"{flops} FLOP per pair·q (species-class factoring, "
                                     "Reinsch form, weights carried in the recurrence), so "
                                     "the figure exceeds the FP32 peak"}},
            "fp64_kernel": fp64,
            "parity": parity,
            "cpu_baseline": cpu,
            "clocks": clk,
            "parallelism": f"tile-sharded solve over {ws} GPUs + NCCL all-reduce" if ws > 1
                           else "1 GPU",
            "tiles": {"q_block": kb.value, "j_chunk": tj.value, "pairs_per_thread": npt.value,
                      "tiles_per_solve": ntile.value, "device_bytes": dbytes.value,
                      "shape_source": "autotuned table entry for the request's bucket"
                                      if from_table.value else "default shape (no table entry)"},
        }
        if secondary:
            line["secondary"] = secondary
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def kernel_mode(req):
    """The pair kernel's mode for a request, as the planner picks it: class
    mode while at most 48 (species, hydration weight) keys exist, else
    weighted; "_general_step" where Δq·2·(largest distance from the
    centroid) > 0.78."""
    mode = "class"
    if req.hyd_weights is not None:
        keys = set(zip(req.species.tolist(), req.hyd_weights.tolist()))
        mode = "weighted" if len(keys) > 48 else "class"
    xyz = req.xyz.reshape(-1, req.n_atoms, 3)
    radius = max(float(np.sqrt(((f - f.mean(axis=0)) ** 2).sum(axis=1)).max()) for f in xyz)
    dq = (req.qmax - req.qmin) / max(req.nq - 1, 1)
    if dq * 2.0 * radius > 0.78:
        mode += "_general_step"
    return mode


def timed_workload(ctx, w, local, min_seconds=2.0):
    """Device-resident executions of one workload, repeated until the timed
    region lasts at least `min_seconds` (so the clock sampler sees it), L2
    flushed before each; returns pair·q/s, ms per solve, repeats, clocks."""
    import torch

    from pripps_b200 import _lib
    lib = _lib.lib()
    req = w.request
    r = req.c_struct()
    plan = C.c_void_p()
    _lib.check(lib.pd_plan_create(ctx.handle, C.byref(r), C.byref(plan)), ctx.handle)
    xyz = torch.from_numpy(req.xyz).to(f"cuda:{local}")
    out = torch.empty((6, req.nq), dtype=torch.float64, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def execute():
        _lib.check(lib.pd_plan_execute(ctx.handle, plan, xyz.data_ptr(), out.data_ptr(), sp),
                   ctx.handle)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        execute()
        flush.zero_()
    e0.record(stream)
    execute()
    e1.record(stream)
    torch.cuda.synchronize()
    reps = max(3, int(np.ceil(min_seconds / max(e0.elapsed_time(e1) * 1e-3, 1e-6))))
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)  # the sampler's first reading falls inside the timed region
    for i in range(reps):
        starts[i].record(stream)
        execute()
        ends[i].record(stream)
        flush.zero_()
    torch.cuda.synchronize()
    clk = clocks.stop()
    lib.pd_plan_destroy(ctx.handle, plan)
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / reps
    return {"value": w.pair_q / (ms * 1e-3), "unit": UNIT, "ms_per_solve": ms, "repeats": reps,
            "n_atoms": req.n_atoms, "nq": req.nq, "n_frames": req.n_frames, "clocks": clk}


def serving_burst(ctx, local, n_requests=400, precision="fp32"):
    """n_requests requests of the serving stream's distribution submitted at
    once to the request loop, after the same burst once untimed: p50/p99
    latency and aggregate pair·q/s."""
    from pripps_b200 import synth, workloads
    from pripps_b200.serving import Server
    stream = synth.request_stream(n_requests, 1e9, seed=4)
    pool = workloads.GlobulePool()
    reqs = [workloads.stream_request_pooled(sr, pool, precision) for sr in stream]
    srv = Server(ctx)
    # warm the loop (lanes and captured graphs of the kernel variants the
    # burst uses, the device pool and the pinned staging blocks grown to the
    # burst's concurrency): the same burst once, untimed
    for t in [srv.submit(w.request) for w in reqs]:
        srv.wait(t)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    t0 = time.perf_counter()
    tickets = [srv.submit(w.request) for w in reqs]
    for t in tickets:
        srv.wait(t)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    lat = np.array([d - s for s, a, d in (srv.times(t) for t in tickets)])
    pq = sum(w.pair_q for w in reqs)
    return {"requests": n_requests, "arrival": "all at once", "value": pq / wall, "unit": UNIT,
            "wall_s": wall, "latency_ms": {"p50": float(np.percentile(lat, 50) * 1e3),
                                           "p99": float(np.percentile(lat, 99) * 1e3)},
            "clocks": clk}


def run_secondary(ctx, args, local):
    """The other workloads, each timed for at least 2 s with its own clock
    record, and a 400-request serving burst."""
    from pripps_b200 import workloads
    out = {}
    for name in ("sphere_solvent_10k", "trajectory_5k_256", "ellipsoid_sasa_20k"):
        if name != args.workload:
            w = workloads.WORKLOADS[name](args.precision)
            out[name] = timed_workload(ctx, w, local)
            out[name]["kernel_mode"] = kernel_mode(w.request)
    out["serving_burst_400"] = serving_burst(ctx, local, 400, args.precision)
    return out


def run_serve(args, ws, rank, local):
    """Serving stream: Poisson-arriving globules (N log-uniform 500–50,000,
    nq 100–1000, qmax 0.3–1.0, 70 % with solvent) submitted at their arrival
    times to the continuous-batching loop (pd_submit); reports p50/p99
    latency (arrival → result), aggregate pair·q/s over the stream, and
    whether a sample of results equals its solo solve bit for bit."""
    import torch

    from pripps_b200 import _lib, synth, workloads
    from pripps_b200.debye import solve
    from pripps_b200.serving import Server

    torch.cuda.set_device(local)
    stream = synth.request_stream(args.requests, args.rate, seed=4 + rank)
    if args.requests > 500:
        # long streams: compact sub-globules of a pool instead of one RSA run
        # per request (same density and size distribution)
        pool = workloads.GlobulePool()
        reqs = [workloads.stream_request_pooled(sr, pool, args.precision) for sr in stream]
    else:
        reqs = [workloads.stream_request(sr, args.precision) for sr in stream]
    ctx = _lib.Context(local, mem_budget_bytes=int(args.budget_gb * (1 << 30)))
    srv = Server(ctx)
    # warm the kernels and graphs on a few requests
    for w in reqs[:3]:
        srv.wait(srv.submit(w.request))
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = ctx.launch_count()
    t0 = time.perf_counter()
    tickets = []
    for sr, w in zip(stream, reqs):
        delay = sr.arrival - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        tickets.append(srv.submit(w.request))
    outs = [srv.wait(t) for t in tickets]
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    launches = ctx.launch_count() - launches0
    times = [srv.times(t) for t in tickets]
    lat = np.array([d - s for s, a, d in times])
    qwait = np.array([a - s for s, a, d in times])
    if args.latency_log:
        np.save(args.latency_log, np.array(
            [(sr.arrival, a - s, d - s, w.request.n_atoms, w.request.nq)
             for (s, a, d), sr, w in zip(times, stream, reqs)]))
    pq = sum(w.pair_q for w in reqs)
    check_idx = list(range(0, len(reqs), max(1, len(reqs) // 8)))
    same = all(np.array_equal(outs[i], solve(reqs[i].request, ctx)) for i in check_idx)
    if rank == 0:
        line = {
            "metric": "Debye serving stream: p50/p99 latency and pair·q/s",
            "value": pq / wall, "unit": UNIT, "n_gpus": ws, "steps": len(reqs),
            "warmup": 3, "ms_per_step": 1e3 * wall / len(reqs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "stream", "requests": len(reqs), "rate_hz": args.rate,
                       "structures": "pooled compact sub-globules" if args.requests > 500
                                     else "one RSA globule per request",
                       "n_atoms": "log-uniform 500-50000", "nq": "uniform 100-1000",
                       "qmax": "uniform 0.3-1.0", "solvent_fraction": 0.7,
                       "budget_gb": args.budget_gb, "precision_form": args.precision},
            "latency_ms": {"p50": float(np.percentile(lat, 50) * 1e3),
                           "p99": float(np.percentile(lat, 99) * 1e3),
                           "mean": float(lat.mean() * 1e3),
                           "admission_wait_p50": float(np.percentile(qwait, 50) * 1e3)},
            "pair_q_total": pq, "wall_s": wall, "gpu_launches": int(launches),
            "alone_equals_mixed": bool(same), "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def run_direct(args, ws, rank, local):
    """Direct transform of a periodic box (pd_direct_lattice, with pd_direct
    beside it): 64 copies of a 2,000-atom globule on a 4×4×4 grid in a 320 Å
    box, Miller vectors with p_max = args.p_max, per-molecule self terms.
    Unit: (q-vector, point) amplitude terms per second; the oracle's rows on a
    sample beside it."""
    import torch
    from oracle import oracle as O
    from pripps_b200 import _lib, synth, workloads
    from pripps_b200.direct import amplitudes, miller_indices, q_vectors
    torch.cuda.set_device(local)
    ctx = _lib.Context(local)
    g = synth.globule(2000, (25.0, 25.0, 25.0), 9)
    L = 320.0
    offs = [(i, j, k) for i in range(4) for j in range(4) for k in range(4)]
    xyz = np.concatenate([g.pos + 80.0 * np.array(o) + 40.0 for o in offs])
    ids = workloads.element_ids()[np.tile(g.elements, len(offs))]
    used = np.unique(ids)
    kind = np.searchsorted(used, ids)
    hkl = miller_indices(args.p_max)
    qv = q_vectors(hkl, [L] * 3)
    qn = np.sqrt((qv * qv).sum(axis=1))
    ff = workloads.foxs().table(used, qn)

    def run(lattice):
        if lattice:  # pd_direct_lattice: per-point phase tables (the path DirectTransform takes)
            return amplitudes(xyz, kind, ff, None, len(offs), None, ctx, hkl=hkl, box=[L] * 3)
        return amplitudes(xyz, kind, ff, qv, len(offs), None, ctx)  # pd_direct: one sincos per term

    def timed(lattice):
        for _ in range(args.warmup):
            run(lattice)
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r = run(lattice)
            ts.append(time.perf_counter() - t0)
        return 1e3 * sum(ts) / len(ts), r

    ms, rows = timed(True)
    ms_sincos, rows_sincos = timed(False)
    work = len(qv) * len(xyz)
    # oracle on a sample: the first 8 molecules (16,000 points), 39 vectors
    nsamp = 16000
    t0 = time.perf_counter()
    O.direct_rows(xyz[:nsamp], kind[:nsamp], ff[:, :39], qv[:39], 8)
    dt = time.perf_counter() - t0
    if rank == 0:
        print(json.dumps({
            "metric": "Direct transform (q-vector, point) terms/s", "value": work / (ms * 1e-3),
            "unit": "vector·point/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "direct_box_64x2000", "points": len(xyz), "molecules": 64,
                       "box": L, "p_max": args.p_max, "vectors": len(qv),
                       "timed": "blocking pd_direct_lattice with host buffers (upload, "
                                "phase tables + amplitude kernel, reduction, download)"},
            "sincos_path": {"value": work / (ms_sincos * 1e-3), "ms_per_step": ms_sincos,
                            "entry": "pd_direct (one FP64 sincos per term)",
                            "max_rel_diff_self_term": float(np.max(
                                np.abs(rows[:, 3] - rows_sincos[:, 3]) /
                                np.abs(rows_sincos[:, 3]).max()))},
            "cpu_baseline": {"value": nsamp * 39 / dt, "unit": "vector·point/s", "cores": 1,
                             "kind": "port", "sample": "16,000 points x 39 vectors",
                             "seconds": dt},
            "checksum_selfterm": float(rows[:, 3].sum())}), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="ellipsoid_solvent_100k")
    ap.add_argument("--precision", default="fp32", choices=("fp32", "fp64"))
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--fp64-nq", type=int, default=64)
    ap.add_argument("--cpu-atoms", type=int, default=6000)
    ap.add_argument("--cpu-q", type=int, default=0,
                    help="q points of the CPU baseline sample (0: two per host core)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the other workloads and the serving burst")
    ap.add_argument("--serve", action="store_true", help="serving-stream benchmark")
    ap.add_argument("--direct", action="store_true", help="direct-transform benchmark")
    ap.add_argument("--p-max", type=int, default=100)
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=20.0, help="Poisson arrival rate (1/s)")
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--latency-log", default=None,
                    help="serving: save per-request (arrival s, admission wait s, latency s, "
                         "n_atoms, nq) to this .npy")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    elif args.serve:
        run_serve(args, ws, rank, local)
    elif args.direct:
        run_direct(args, ws, rank, local)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
