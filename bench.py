"""Benchmark of the batched convergent Born series solve on B200.

Workload (one "step"): the batching configuration -- 128x128x64 grid at 50 nm, water background
(eps_bg = 1.33^2), a seeded phantom of 12 non-overlapping beads (radius U[4,12] px, index U[1.36,1.60]),
64 right-hand sides per GPU (32 illumination angles in an NA 1.2 cone snapped to the lattice x 2 polarisations),
500 nm, periodic x,y and absorbing z (padded grid 128^3), tolerance 1e-6, GMRES as the reference runs it
(no restart, maxiters = max(2*Bornmax, 100), warm start b); complex64 fields in HBM, FFT / Green /
potential arithmetic in FP64 registers, FP64 dots; the Krylov basis is built by block (s-step) GMRES with
s = 8 (``--ortho cgs`` for classical Gram-Schmidt; ``--precision float32`` runs the arithmetic in FP32 too).
With N GPUs the job has 32N angles x 2 polarisations and each rank solves its own 64 (weak scaling).

value : solves/s of that step with the potential resident in HBM and the fields left in HBM
        (device time from CUDA events on the library's stream, max over ranks).
e2e   : solves/s through the public API (fmcuda.solve_batch) from host permittivity to host E, H.
Also reported: the plain FP64 GPU method (same algorithm with Krylov.jl's MGS, one RHS), timed the same two ways,
and the relative L2 distance of the batched FP32 fields to it; the CPU oracle's complete FP64 solve of RHS 0
(the CPU baseline, and ``vs_oracle``: both GPU forms against it); the roofline of the dominant kernel class from
live CUDA-event timing.

`--impl reference` times the CPU restatement of the reference path (the reference is Julia, which this
image does not have) on the same workload and prints its own line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
import warnings

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "frequencymaxwell.jl_b200"))

GRID = (128, 128, 64)
RES = (50e-9, 50e-9, 50e-9)
WL = 500e-9
EPS_BG = 1.33 ** 2
SEED = 20261203
NA = 1.2
METRIC = "solves/s at rel-L2<=1e-5 vs FP64: batched FP32 vs plain FP64; p50/p99 latency"


def batching_sources(n_angles=32, seed=SEED):
    """``n_angles`` (kx, ky) uniform in the NA 1.2 disk (sin(theta) <= NA/n_bg), snapped to the lattice
    2*pi*m/(N*dx); polarisations s and p (two unit vectors orthogonal to k).  The first 32 angles do not depend
    on ``n_angles``."""
    import fmcuda as F
    return [(s.k_vector, s.polarization.real) for s in
            F.illumination_cone(GRID, RES, WL, EPS_BG, n_angles, NA, seed)]


def make_inputs(n_angles=32):
    import fmcuda as F
    med = F.phantom_random_beads(GRID, 12, (4, 12), (1.36, 1.60), EPS_BG, SEED)
    bc_z = F.AbsorbingBoundaryCondition(thickness=GRID[2] * RES[2], attenuation_thickness=GRID[2] * RES[2],
                                        sharpness=1.0, profile=F.TanhProfile)
    bcs = (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(), bc_z)
    srcs = [F.PlaneWaveSource(wavelength=WL, polarization=p, k_vector=k) for k, p in batching_sources(n_angles)]
    return med, bcs, srcs


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def rel_l2(a, b):
    """||a - b||_2 / ||b||_2 in FP64."""
    a = np.asarray(a, dtype=np.complex128).ravel()
    b = np.asarray(b, dtype=np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def oracle_rhs0(callback=None):
    """The CPU oracle (numpy/scipy FP64 restatement of the reference path, all host cores) on right-hand side 0
    of the workload: potential set-up, incident field, source term, b = G S, the complete GMRES solve as the
    reference runs it (MGS, no restart, warm start b, maxiters = max(2 Bornmax, 100)), curl and crop.
    ``callback(k)`` is called after GMRES iteration k.  Returns (result, start time, seconds)."""
    from oracle import cbs_oracle as O
    med, _, srcs = make_inputs()
    t_pad = GRID[2] * RES[2]
    cfg = O.SolverConfig(RES, GRID, (O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(t_pad, t_pad, 1.0)))
    s = srcs[0]
    src = O.PlaneWave(WL, s.polarization, s.k_vector)
    t0 = time.perf_counter()
    r = O.solve(cfg, src, med.permittivity, EPS_BG, callback=callback)
    return r, t0, time.perf_counter() - t0


def cpu_baseline():
    """One complete oracle solve of right-hand side 0, timed on the host cores (see oracle_rhs0)."""
    r, _, T = oracle_rhs0()
    sample = (f"right-hand side 0 of the workload, one complete FP64 solve: set-up, RHS, {r.iterations} GMRES "
              f"iterations (MGS), curl, crop; {T:.1f} s")
    cb = {"value": 1.0 / T, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port", "sample": sample,
          "seconds_per_solve": T, "iterations": r.iterations}
    return cb, r


def run_reference(args):
    """The reference arm: the oracle (the CPU restatement of the reference's path; the reference itself is Julia,
    which this image does not have) with all host cores.  Its steps are consecutive slices of complete solves of
    right-hand side 0: step i is GMRES iterations (i*c, (i+1)*c] with c = ceil(maxiters / (warmup + steps)); the
    first step of a solve also carries its set-up and the last its curl and crop.  ``value`` is one over the
    duration of the complete solve(s); ``ms_per_step`` is the mean of the timed (non-warm-up) steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n_steps = args.warmup + args.steps
    step_times = []        # duration of every step, over consecutive solves
    solve_secs = []
    iters_done = []
    while len(step_times) < n_steps:
        marks = []
        r, t_start, T = oracle_rhs0(callback=lambda k: marks.append((k, time.perf_counter())))
        c = max(1, math.ceil(r.iterations / n_steps))
        ends = [t for k, t in marks if k % c == 0 and k < r.iterations] + [t_start + T]
        starts = [t_start] + ends[:-1]
        step_times += [e - b for b, e in zip(starts, ends)]
        solve_secs.append(T)
        iters_done.append(r.iterations)
    timed = step_times[args.warmup:n_steps]
    T = statistics.mean(solve_secs)
    v = 1.0 / T
    cb = {"value": v, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
          "sample": f"right-hand side 0 of the workload, {len(solve_secs)} complete FP64 solve(s) of "
                    f"{iters_done[0]} GMRES iterations split into {n_steps} steps; {T:.1f} s per solve",
          "seconds_per_solve": T}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.mean(timed),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "batching: 128x128x64 (padded 128^3), 12 seeded beads, 64 RHS (32 NA-1.2 "
                                   "angles x 2 pol), GMRES-100; sample: complete solves of RHS 0",
                       "grid": list(GRID), "padded": [128, 128, 128], "rhs": 64, "solver": "gmres-100 (MGS)"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run(args):
    import torch
    import fmcuda as F
    from fmcuda.replicas import max_over_ranks, shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)

    # The job: nrhs right-hand sides per GPU.  With N GPUs it has N*nrhs/2 angles x 2 polarisations, and every
    # rank solves its own share of them (round-robin shard, weak scaling, no collective on the data path).
    med, bcs, srcs_all = make_inputs(n_angles=world * args.nrhs // 2)
    mine = shard(len(srcs_all), world, rank)
    srcs = [srcs_all[i] for i in mine]
    lists = [[s] for s in srcs]
    nrhs = len(lists)
    solver = F.ConvergentBornSolver(resolution=RES, grid_size=GRID, boundary_conditions=bcs, tolerance=1e-6,
                                    precision=args.precision,
                                    linear_solver=F.KrylovJL_GMRES(ortho=args.ortho, block_size=args.block,
                                                                   block_vectors=args.block_store),
                                    max_rhs=nrhs, device_index=dev)
    tuning = None
    if args.autotune:
        from fmcuda import autotune as AT
        tuning = AT.autotune(solver, lists, med)
        AT.configure(solver, tuning)
    if args.block_dot >= 0:
        from fmcuda import autotune as AT
        AT.apply(solver.plan(), {"block_dot": args.block_dot})
    plan = solver.plan()
    info = plan.build_potential(med.permittivity, med.permittivity_bg, WL, solver.attenuation_filters(), -1)
    opts = solver.solve_options(int(info.bornmax))
    stream = torch.cuda.ExternalStream(plan.stream(), device=torch.device("cuda", dev))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def step():
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            _, _, infos, st = plan.solve_plane_waves(lists, EPS_BG, opts, keep_on_device=True)
        return infos

    for _ in range(args.warmup):
        step()
    barrier()
    times = []
    plan.set_profiling(True)
    launches0 = plan.launch_count()
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            barrier()
            ev0.record(stream)
            infos = step()
            ev1.record(stream)
            ev1.synchronize()
            times.append(ev0.elapsed_time(ev1) / 1000.0)
            barrier()
    launches = plan.launch_count() - launches0
    kstats = plan.kernel_stats()
    plan.set_profiling(False)
    t_med = max_over_ranks(statistics.median(times))  # the slowest rank sets the job time
    value = world * nrhs / t_med
    n_pad = float(np.prod(solver.padded_size()))
    iters = [i.iterations for i in infos]

    # end to end through the public API (host permittivity in, host E/H out)
    e2e_times = []
    outs = None
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        for _ in range(args.e2e_steps):
            barrier()
            t0 = time.perf_counter()
            outs = F.solve_batch(solver, lists, med)
            barrier()
            e2e_times.append(time.perf_counter() - t0)
    e2e_t = max_over_ranks(statistics.median(e2e_times)) if e2e_times else float("nan")
    g = int(np.prod(GRID))
    h2d = g * 16 + sum(GRID[d] + 2 * solver.padding()[d] for d in range(3)) * 8
    d2h = 2 * nrhs * 3 * g * 16

    solver.release()  # the batched plan's device memory is not needed past this point
    # The plain FP64 GPU method (the reference algorithm: GMRES with MGS, one RHS at a time), timed the same way
    # as the batched form (CUDA events on the library stream, potential and fields resident in HBM), and end to
    # end through F.solve (host permittivity in, host E/H out).
    fp64 = F.ConvergentBornSolver(resolution=RES, grid_size=GRID, boundary_conditions=bcs, tolerance=1e-6,
                                  precision="float64", linear_solver=F.KrylovJL_GMRES(ortho="mgs"), max_rhs=1,
                                  device_index=dev)
    t64_dev, t64_e2e = [], []
    ref = None
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        if args.fp64_steps > 0:
            ref = F.solve(fp64, srcs[0], med)  # untimed: plan creation and first-touch allocations
            p64 = fp64.plan()
            o64 = fp64.solve_options(fp64.Bornmax)
            s64 = torch.cuda.ExternalStream(p64.stream(), device=torch.device("cuda", dev))
        for _ in range(args.fp64_steps):
            barrier()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(s64)
            p64.solve_plane_waves(lists[:1], EPS_BG, o64, keep_on_device=True)
            ev1.record(s64)
            ev1.synchronize()
            t64_dev.append(ev0.elapsed_time(ev1) / 1000.0)
        for _ in range(args.fp64_steps):
            barrier()
            t0 = time.perf_counter()
            ref = F.solve(fp64, srcs[0], med)
            barrier()
            t64_e2e.append(time.perf_counter() - t0)
    fp64_sps = 1.0 / max_over_ranks(statistics.median(t64_dev)) if t64_dev else float("nan")
    fp64_e2e_sps = 1.0 / max_over_ranks(statistics.median(t64_e2e)) if t64_e2e else float("nan")
    fp64_iters = fp64.iteration_count
    # accuracy of the batched form against the plain FP64 method on the first accuracy_rhs right-hand sides
    errs_e, errs_h = [], []
    if ref is not None and outs:
        errs_e.append(rel_l2(outs[0].E, ref.E))
        errs_h.append(rel_l2(outs[0].H, ref.H))
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            for i in range(1, min(args.accuracy_rhs, len(outs))):
                r = F.solve(fp64, srcs[i], med)
                errs_e.append(rel_l2(outs[i].E, r.E))
                errs_h.append(rel_l2(outs[i].H, r.H))
    err_e = max(errs_e) if errs_e else None
    err_h = max(errs_h) if errs_h else None
    fp64.release()

    # roofline of the dominant kernel class (live CUDA-event timing over the timed steps)
    peak, peak_kind = load_peaks()
    dom = max(kstats.items(), key=lambda kv: kv[1]["ms"])
    dname, ds = dom
    achieved = ds["bytes"] / (ds["ms"] / 1000.0) / 1e9 if ds["ms"] > 0 else 0.0
    total_ms = sum(v["ms"] for v in kstats.values())
    traffic = None
    try:  # DRAM / algorithmic bytes of this kernel class from its ncu capture (profiles/traffic.txt)
        with open(os.path.join(ROOT, "profiles", "traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if parts and not line.startswith("#") and parts[0] == dname:
                    traffic = float(parts[1]) * ds["bytes"] / max(1, ds["launches"])
    except OSError:
        pass
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": dname, "peak_kind": peak_kind,
            "share": ds["ms"] / total_ms if total_ms > 0 else None,
            "bytes_per_launch": ds["bytes"] / max(1, ds["launches"]),
            "ms_per_launch": ds["ms"] / max(1, ds["launches"])}
    all_bytes = sum(v["bytes"] for v in kstats.values())
    classes = {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                   "GBps": round(v["bytes"] / (v["ms"] / 1000) / 1e9, 1) if v["ms"] > 0 else None}
               for k, v in kstats.items() if v["launches"]}

    serving = None
    if rank == 0 and world == 1 and args.serving_requests > 0:
        serving = run_serving(args)
    large = None
    if rank == 0 and world == 1 and args.large:
        large = run_large(args)
    cb = None
    oracle_acc = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # the CPU oracle's complete FP64 solve of right-hand side 0: the CPU baseline, and the reference result
        # both GPU forms are measured against
        cb, orc = cpu_baseline()
        oracle_acc = {"rhs": 0, "oracle_iterations": orc.iterations}
        if outs:
            oracle_acc.update(rel_l2_E_batched=rel_l2(outs[0].E, orc.E), rel_l2_H_batched=rel_l2(outs[0].H, orc.H))
        if ref is not None:
            oracle_acc.update(rel_l2_E_fp64=rel_l2(ref.E, orc.E), rel_l2_H_fp64=rel_l2(ref.H, orc.H),
                              fp64_iterations=fp64_iters)
    clocks = clk.summary()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_med * 1000.0, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128" if args.precision == "float32-math64" else "c64",
                "data": "synthetic",
                "config": {"workload": "batching: 128x128x64 (padded 128^3), 12 seeded beads, "
                                       f"{nrhs} RHS per GPU ({nrhs // 2} NA-1.2 angles x 2 pol), "
                                       f"GMRES-{opts.maxiters}",
                           "grid": list(GRID), "padded": list(solver.padded_size()), "rhs_per_gpu": nrhs,
                           "rhs_total": world * nrhs,
                           "precision": f"{args.precision}: complex64 fields in HBM, FP64 dots"
                                        + (", FP64 FFT/Green/V arithmetic" if args.precision != "float32" else ""),
                           "ortho": args.ortho + (f"-{args.block}-{args.block_store}" if args.ortho == "block" else ""),
                           "parallelism": f"replicas{world}: right-hand sides sharded round-robin over ranks",
                           "l2": "inputs larger than L2 (Krylov basis of 50 MB vectors)", "seed": SEED,
                           "tuning": tuning},
                "latency_s": {"p50": statistics.median(times), "p99": float(np.percentile(times, 99)),
                              "unit": "batched step"},
                "iterations": {"min": min(iters), "max": max(iters)},
                "born_iterations_per_s": world * sum(iters) / t_med,
                "padded_voxel_iterations_per_s": world * sum(iters) / t_med * n_pad,
                "flops_model": {"per_iteration": 12 * 5 * n_pad * math.log2(n_pad),
                                "achieved_GFLOPs": world * sum(iters) / t_med * 12 * 5 * n_pad * math.log2(n_pad) / 1e9,
                                "model": "12 x 5 N log2 N per Born iteration (2 branches x fwd+inv x 3 components)"},
                "fp64_plain": {"solves_per_s": fp64_sps, "timing": "CUDA events, potential and fields in HBM",
                               "e2e_solves_per_s": fp64_e2e_sps, "iterations": fp64_iters,
                               "rel_l2_E_fp32_vs_fp64": err_e, "rel_l2_H_fp32_vs_fp64": err_h,
                               "rel_l2_over_rhs": len(errs_e), "bar": 1e-5,
                               "ratio_fp32_batched_over_fp64": value / world / fp64_sps,
                               "ratio_e2e": (world * nrhs / e2e_t) / world / fp64_e2e_sps},
                "vs_oracle": oracle_acc,
                "e2e": {"value": world * nrhs / e2e_t, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "roofline": roof, "kernel_classes": classes,
                "algorithmic_GBps_all_kernels": all_bytes / (total_ms / 1000) / 1e9 if total_ms else None,
                "serving": serving, "large": large, "cpu_baseline": cb, "clocks": clocks, "gpu_launches": launches}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_serving(args):
    """Continuous batching of a seeded Poisson request stream (bounded sample of the serving workload):
    grids drawn uniformly from {64x64x32, 96x96x64, 128x128x64, 256x256x128}, 1-32 angles each, 12-bead
    phantoms, complex64 fields with FP64 dots, tolerance 1e-5, slots sized from a 150 GB device budget.  With
    the default ortho "block", the slots run s-step block GMRES (one block of 8 iterations per engine step),
    restarted every basis iterations when their limit exceeds the basis."""
    from fmcuda import serving as SV
    reqs = SV.serving_requests(args.serving_requests, rate=args.serving_rate, seed=SEED)
    srv = SV.Server(SV.SERVING_SHAPES, budget_bytes=args.serving_budget_gb * 1e9, basis=args.serving_basis,
                    precision=args.precision, ortho=args.serving_ortho)
    try:
        srv.start()
        rep = SV.run_stream(srv, reqs, timeout=1800)
    finally:
        srv.stop()
    rep.update({"budget_GB": args.serving_budget_gb, "basis": args.serving_basis, "ortho": args.serving_ortho,
                "tolerance": 1e-5,
                "rate_req_per_s": args.serving_rate, "shapes": ["x".join(map(str, s)) for s in SV.SERVING_SHAPES],
                "latency": "request arrival to its last right-hand side's fields on the host",
                "iterations": {"min": min(i["iterations"] for r in reqs for i in r.infos.values()),
                               "max": max(i["iterations"] for r in reqs for i in r.infos.values())}})
    return rep


def run_large(args):
    """The large single configuration: 512x512x256 at 50 nm (padded z 512, the two shifted z branches as two
    z passes), 40 seeded beads (radius U[6,24] px, index U[1.4,2.0]) in water, 500 nm x-pol +z, GMRES(20) on
    the CBS-preconditioned operator with FP32 fields and FP64 dots, tolerance 1e-6.  One solve is timed on the
    device (2-iteration warm-up for the plan and tables)."""
    import torch
    import fmcuda as F
    grid = (512, 512, 256)
    med = F.phantom_random_beads(grid, 40, (6, 24), (1.4, 2.0), EPS_BG, SEED + 4)
    bc_z = F.AbsorbingBoundaryCondition(thickness=grid[2] * RES[2], attenuation_thickness=grid[2] * RES[2],
                                        sharpness=1.0, profile=F.TanhProfile)
    bcs = (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(), bc_z)
    src = F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1])
    solver = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=bcs, tolerance=1e-6,
                                    precision=args.precision, max_rhs=1,
                                    linear_solver=F.KrylovJL_GMRES(ortho="cgs", gmres_restart=20))
    plan = solver.plan()
    info = plan.build_potential(med.permittivity, med.permittivity_bg, WL, solver.attenuation_filters(), -1)
    opts = solver.solve_options(int(info.bornmax))
    stream = torch.cuda.ExternalStream(plan.stream(), device=torch.device("cuda", 0))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        warm = solver.solve_options(int(info.bornmax))
        warm.maxiters = 2
        plan.solve_plane_waves([[src]], EPS_BG, warm, keep_on_device=True)
        plan.set_profiling(True)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        _, _, infos, st = plan.solve_plane_waves([[src]], EPS_BG, opts, keep_on_device=True)
        ev1.record(stream)
        ev1.synchronize()
    t = ev0.elapsed_time(ev1) / 1000.0
    ks = plan.kernel_stats()
    plan.set_profiling(False)
    tot = sum(v["ms"] for v in ks.values())
    out = {"workload": "large single: 512x512x256 (padded 512^3), 40 beads n 1.4-2.0, GMRES(20), tol 1e-6",
           "precision": args.precision, "bornmax": int(info.bornmax), "maxiters": int(opts.maxiters),
           "iterations": int(infos[0].iterations), "solved": bool(infos[0].solved),
           "relative_residual": float(infos[0].residual / infos[0].residual0), "seconds_per_solve": t,
           "born_iterations_per_s": infos[0].iterations / t,
           "kernel_classes": {k: {"ms": round(v["ms"], 1), "GBps": round(v["bytes"] / (v["ms"] / 1000) / 1e9, 1)}
                              for k, v in ks.items() if v["launches"] and v["ms"] > 0},
           "share_top": max(((k, v["ms"] / tot) for k, v in ks.items()), key=lambda kv: kv[1]) if tot else None}
    solver.release()
    if args.large_check:
        out["fp32_vs_fp64_check"] = large_check(args)
    return out


def large_check(args):
    """The large configuration's accuracy check at reduced lateral size: 128x128x256 (the same padded z of 512,
    two shifted z passes), 10 beads with the large configuration's statistics (radius U[6,24] px, index
    U[1.4,2.0]), x-pol +z, GMRES(20).  The FP32-field form against the plain FP64 GPU method (MGS), both full
    solves; the full 512^3 FP64 solve needs ~182 GB and does not fit one GPU."""
    import fmcuda as F
    grid = (128, 128, 256)
    med = F.phantom_random_beads(grid, 10, (6, 24), (1.4, 2.0), EPS_BG, SEED + 5)
    bc_z = F.AbsorbingBoundaryCondition(thickness=grid[2] * RES[2], attenuation_thickness=grid[2] * RES[2],
                                        sharpness=1.0, profile=F.TanhProfile)
    bcs = (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(), bc_z)
    src = F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1])
    res = {}
    for prec, ortho in ((args.precision, "cgs"), ("float64", "mgs")):
        sv = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=bcs, tolerance=1e-6,
                                    precision=prec, max_rhs=1, linear_solver=F.KrylovJL_GMRES(ortho=ortho,
                                                                                            gmres_restart=20))
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            t0 = time.perf_counter()
            f = F.solve(sv, src, med)
            dt = time.perf_counter() - t0
        res[prec] = (f, sv.iteration_count, sv.residual_history[-1], dt)
        sv.release()
    f32, it32, r32, t32 = res[args.precision]
    f64, it64, r64, t64 = res["float64"]
    return {"grid": list(grid), "padded_z": 512, "iterations": [it32, it64], "seconds": [t32, t64],
            "rel_l2_E": rel_l2(f32.E, f64.E), "rel_l2_H": rel_l2(f32.H, f64.H),
            "residual_ratio": r32 / r64 if r64 else None}


def run_two_beam_example(args):
    """The reference's examples/two_beam_interference.jl homogeneous case: 201x201x191 at 50 nm (odd axes, the
    general passes), periodic x/y, 300 nm Tanh absorbing z, water, two coherent x-polarised 532 nm waves at the
    +-3rd order, BiCGStab, tolerance 1e-6.  Each precision's solve is timed from host arrays to host fields
    (wall clock, after one untimed solve for the plan and tables), with the example's fringe contrast."""
    import fmcuda as F
    grid, res = (201, 201, 191), (50e-9,) * 3
    bc_z = F.AbsorbingBoundaryCondition(thickness=300e-9, attenuation_thickness=300e-9, sharpness=1.0,
                                        profile=F.TanhProfile)
    bcs = (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(), bc_z)
    eps_bg, wl = 1.333 ** 2, 532e-9
    ky = 2 * math.pi * 3 / (grid[1] * res[1])
    a = math.asin(ky / (2 * math.pi * math.sqrt(eps_bg) / wl))
    srcs = [F.PlaneWaveSource(wavelength=wl, polarization=[1.0, 0.0, 0.0], k_vector=[0.0, sg * math.sin(a),
                                                                                   math.cos(a)]) for sg in (1, -1)]
    med = F.Medium(np.full(grid, eps_bg, dtype=np.complex128), eps_bg)
    out = {"grid": list(grid), "solver": "bicgstab", "tolerance": 1e-6}
    for prec in ("float64", args.precision):
        sv = F.ConvergentBornSolver(resolution=res, grid_size=grid, boundary_conditions=bcs, tolerance=1e-6,
                                    precision=prec, linear_solver=F.KrylovJL_BICGSTAB())
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            F.solve(sv, srcs, med)
            t0 = time.perf_counter()
            f = F.solve(sv, srcs, med)
            dt = time.perf_counter() - t0
        it = np.sum(np.abs(f.E) ** 2, axis=3)[grid[0] // 2, :, grid[2] // 2]
        out[prec] = {"seconds_per_solve": dt, "iterations": sv.iteration_count,
                     "padded": list(sv.padded_size()),
                     "contrast": float((it.max() - it.min()) / (it.max() + it.min()))}
        sv.release()
    return out


def run_basic_example(args):
    """The reference's examples/basic_scattering.jl: 128x128x64 at 50 nm, periodic x/y, 3 um Tanh absorbing z
    (padded z 124, the general passes), a SiO2 bead (n = 1.46, radius 10 px) in water, an x-polarised 532 nm
    plane wave along +z, GMRES, tolerance 1e-2.  Each precision's solve is timed from host arrays to host fields
    (wall clock, after one untimed solve for the plan and tables), the bead painted on the device."""
    import fmcuda as F
    grid, res, eps_bg = (128, 128, 64), (50e-9,) * 3, 1.333 ** 2
    bc_z = F.AbsorbingBoundaryCondition(thickness=3e-6, attenuation_thickness=3e-6, sharpness=1.0,
                                        profile=F.TanhProfile)
    bcs = (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(), bc_z)
    src = F.PlaneWaveSource(wavelength=532e-9, polarization=[1.0, 0.0, 0.0], k_vector=[0.0, 0.0, 1.0])
    med = F.phantom_bead(grid, [1.46 ** 2], 10.0, permittivity_bg=eps_bg, on_device=True)
    out = {"grid": list(grid), "solver": "gmres", "tolerance": 1e-2}
    for prec in ("float64", args.precision):
        sv = F.ConvergentBornSolver(resolution=res, grid_size=grid, boundary_conditions=bcs, tolerance=1e-2,
                                    precision=prec, linear_solver=F.KrylovJL_GMRES())
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            F.solve(sv, src, med)
            t0 = time.perf_counter()
            f = F.solve(sv, src, med)
            dt = time.perf_counter() - t0
        out[prec] = {"seconds_per_solve": dt, "iterations": sv.iteration_count, "padded": list(sv.padded_size()),
                     "max_abs_E": float(np.abs(f.E).max())}
        sv.release()
    return out


def run_operator_case(args):
    """Small case for profilers: `reps` applications of the CBS operator on `nrhs` seeded random fields
    on the bench grid (no solve)."""
    import fmcuda as F
    med, bcs, _ = make_inputs()
    rng = np.random.default_rng(0)
    shp = (128, 128, 128, 3, args.nrhs)
    x = np.asfortranarray(rng.standard_normal(shp) + 1j * rng.standard_normal(shp))
    s = F.ConvergentBornSolver(resolution=RES, grid_size=GRID, boundary_conditions=bcs, precision=args.precision,
                               max_rhs=args.nrhs)
    p = s.plan()
    p.build_potential(med.permittivity, EPS_BG, WL, s.attenuation_filters(), -1)
    t0 = time.perf_counter()
    for _ in range(args.reps):
        y = p.apply_operator(x)
    print(json.dumps({"operator_case": args.precision, "nrhs": args.nrhs, "reps": args.reps,
                      "s_per_rep_host": (time.perf_counter() - t0) / args.reps, "mean_abs": float(np.abs(y).mean())}))
    s.release()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fmcuda", choices=["fmcuda", "reference"])
    ap.add_argument("--nrhs", type=int, default=64)
    ap.add_argument("--ortho", default="block", choices=["mgs", "cgs", "cgs2", "block"])
    ap.add_argument("--block", type=int, default=8, help="vectors per block for --ortho block")
    ap.add_argument("--block-store", default="fp64-ortho", choices=["fp64", "storage", "fp64-ortho"],
                    help="raw block vectors in complex FP64 or in the plan's storage type")
    ap.add_argument("--accuracy-rhs", type=int, default=8, help="right-hand sides checked against plain FP64")
    ap.add_argument("--autotune", type=int, default=1, help="1: pick launch shapes and block size with fmcuda.autotune")
    ap.add_argument("--block-dot", type=int, default=-1,
                    help="block dot of block GMRES: 1 bulk-copy pipeline, 0 register-staged, -1 the plan's default")
    ap.add_argument("--precision", default="float32-math64", choices=["float32", "float32-math64"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--operator-case", action="store_true", help="profiling case: operator applications only")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--serving-requests", type=int, default=8, help="requests in the serving sample (0: skip)")
    ap.add_argument("--serving-rate", type=float, default=200.0)
    ap.add_argument("--serving-budget-gb", type=float, default=150.0)
    ap.add_argument("--serving-basis", type=int, default=112, help="Krylov basis per slot (block slots run full "
                    "GMRES when maxiters + 8 <= basis, else restart when the basis is full)")
    ap.add_argument("--serving-ortho", default="block", choices=["cgs", "cgs2", "block"])
    ap.add_argument("--serving-only", action="store_true", help="run the serving sample alone and print it")
    ap.add_argument("--large-only", action="store_true", help="run the large single configuration and print it")
    ap.add_argument("--large-check", type=int, default=1, help="with the large configuration: FP32 vs FP64 check at 128x128x256")
    ap.add_argument("--large", type=int, default=1, help="1: also run the large single configuration (N = 1 only)")
    ap.add_argument("--example-two-beam", action="store_true",
                    help="time the reference's examples/two_beam_interference.jl solve (201x201x191, BiCGStab)")
    ap.add_argument("--example-basic", action="store_true",
                    help="time the reference's examples/basic_scattering.jl solve (128x128x64 bead, GMRES)")
    args = ap.parse_args()
    if args.example_basic:
        print(json.dumps({"basic_scattering_example": run_basic_example(args)}))
        return 0
    if args.example_two_beam:
        print(json.dumps({"two_beam_example": run_two_beam_example(args)}))
        return 0
    if args.operator_case:
        return run_operator_case(args)
    if args.serving_only:
        print(json.dumps({"serving": run_serving(args)}))
        return 0
    if args.large_only:
        print(json.dumps({"large": run_large(args)}))
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run(args)


if __name__ == "__main__":
    sys.exit(main())
