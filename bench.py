"""Benchmark of the smoke step: ms/step and PCG iterations of the 128^3 plume to relative residual 1e-5.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--n 128]

One JSON line on rank 0. "value" is the device time of one step of the headline form (FP32 stencils, multigrid-
preconditioned FCG with FP64 dot products and an FP64 true-residual refinement, to 1e-5) with every input resident
in HBM and L2 flushed between timed steps; "e2e" is the same step driven through the C ABI with the step's host
input copied in from pinned memory and its result (total density) read back, per step. The Jacobi-PCG and plain-
FP32 forms run on the same states and are reported beside it. `--impl reference` runs the reference's own CUDA
library (compiled from its sources into oracle/_ref) on the same scene through the same ABI, with the fixed CG
iteration count that reaches its FP32 residual floor on this scene. Several GPUs run independent replicas (the
step does not shard); timing is the max over ranks. `--profile` runs a profiling workload instead (no JSON line).
The line's "other_configs" holds short runs of the other configurations (64^3 plain method, 256x384x256 scene, 48-
scene batch) taken after the headline; `--no-other-configs` skips them.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "visual-simulation-of-smoke_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

import smoke_abi as abi  # noqa: E402

METRIC = "ms/step and PCG iters at 128³ to rel-res 1e-5: learned+mixed vs plain FP32"
REF_LIBRARY = os.path.join(ROOT, "oracle", "_ref", "libvisual-simulation-of-smoke.so")
# Fixed CG iteration count of the reference on the 128^3 plume: its FP32 CG stalls near relative residual 2.5e-5
# (it never reaches 1e-5), and 900 is the smallest count that reaches that floor on every step after the spin-up
# (measured on a B200 with `bench.py --calibrate-reference`).
REFERENCE_CG_ITERATIONS = 900
SPINUP_STEPS = 30
# Kernels of one step outside the pressure solve: vorticity, cell force, face force, velocity pad, advect velocity,
# rhs, project, scalar prep, velocity pad, scalar pad, advect scalars, density fill (the velocity views' kernel,
# timed with the step, is counted beside it).
STEP_KERNELS = 12


def mg_grid_levels(n):
    """Levels of the multigrid hierarchy of an n^3 grid and how many run grid-wide (mirrors context.cpp)."""
    dims, (x, y, z) = [], (n, n, n)
    dims.append((x, y, z))
    while (x > 1 or y > 1 or z > 1) and len(dims) < 12:
        x, y, z = (x + 1) // 2, (y + 1) // 2, (z + 1) // 2
        dims.append((x, y, z))
    cells = [a * b * c for a, b, c in dims]
    grid, words = len(dims) - 1, 0
    for l in range(len(dims) - 1, 0, -1):
        words += 3 * cells[l] + (cells[l] + 2) // 2
        if cells[l] > 512 or words * 4 > 16 * 1024:
            break
        grid = l
    return len(dims), grid


# Kernels one network evaluation launches inside a learned solve: input packing, 8 convolutions, 3 pools, 3 up-adds.
NET_FORWARD_KERNELS = 15


def solver_launches(n, iterations, refinement, learned=False, net_iterations=0):
    """Kernels the multigrid solve graph launches: set-up and write-back, per refinement pass the first update, the
    accumulation and the FP64 residual, and per iteration the loop body (restriction and the fused prolongation +
    smoothing of every grid level below 0, the block-level cycle, level-0 prolongation, smoothing, p/q and update).
    The learned form adds per pass the gate of its second loop, and per iteration with the network (the first
    `net_iterations`, 0: all) the residual after the V-cycle and its restriction, the network on level 1, the
    prolongation of its output and the correction."""
    _, g = mg_grid_levels(n)
    # coarse grid levels of at most 64^3 cells fuse prolongation and smoothing (mg_up_kernel)
    per_iteration = sum(2 if -(-n // (1 << l)) ** 3 <= 64 ** 3 else 3 for l in range(1, g)) + 5
    total = 2 + 3 * (refinement + 1) + per_iteration * iterations
    if learned:
        with_net = iterations if net_iterations == 0 else min(net_iterations, iterations)
        total += (refinement + 1) + (4 + NET_FORWARD_KERNELS) * with_net
    return total


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def peak_tflops():
    """Measured dense BF16 tensor throughput (burst) of this pool's B200s, else the fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(value: float, world: int) -> float:
    """The largest of the ranks' values (every rank takes part; NCCL on GPUs, gloo on host-only test ranks)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


class L2Flush:
    def __init__(self):
        import torch

        self.buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def __call__(self):
        self.buf.fill_(1)


def run_steps(sim, driver, first_step, count, flush, timed=True, status=False):
    """Per-step device time of sim.step() plus the velocity views the next step's inputs read (events on the
    simulation stream; the reference computes its views inside its step), driver inputs untimed."""
    import torch

    times, iters, resid = [], [], []
    for k in range(count):
        driver.apply(first_step + k)
        if flush is not None:
            with torch.cuda.stream(sim.stream):
                flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(sim.stream)
        sim.step()
        sim.view_raw(abi.VIEW_FLOW_VELOCITY, sim.stream)  # the lazily computed centred-velocity group, inside the timed region
        e1.record(sim.stream)
        driver.read_result()
        sim.stream.synchronize()
        times.append(e0.elapsed_time(e1))
        if status:
            st = sim.solver_status()
            iters.append(st.iterations)
            if st.true_relative_residual >= 0:
                resid.append(st.true_relative_residual)
            else:  # no FP64 residual from the solver: measure it on the views (closed box, no solids)
                import plume_scene

                with torch.cuda.stream(sim.stream):
                    r = plume_scene.closed_box_residual(sim.view(abi.VIEW_FLOW_PRESSURE).double(), sim.view(abi.VIEW_FLOW_PRESSURE_RHS).double())
                    resid.append(float(r))
    return times, iters, resid


def run_e2e(sim, driver, first_step, count):
    """Wall time per step through the ABI: host input -> H2D, step, result D2H, host read."""
    t0 = time.perf_counter()
    total = 0.0
    for k in range(count):
        host = driver.inputs_for(first_step + k)
        driver.apply(first_step + k, host)
        sim.step()
        res = driver.read_result()
        sim.stream.synchronize()
        total += float(res[0])
    return (time.perf_counter() - t0) * 1e3 / count, total


def save_state(sim):
    import torch

    with torch.cuda.stream(sim.stream):
        u, v, w = (t.clone() for t in sim.face_velocity(0))
        d = sim.view(abi.VIEW_DENSITY).clone()
        t_ = sim.view(abi.VIEW_TEMPERATURE).clone()
    sim.stream.synchronize()
    return u, v, w, d, t_


def restore_state(sim, state):
    import torch

    u, v, w, d, t_ = state
    with torch.cuda.stream(sim.stream):
        sim.set_face_velocity(u, v, w)
        sim.update_density(d)
        sim.update_temperature(t_)
    sim.stream.synchronize()


# Algorithmic bytes per cell and iteration of the solver kernels (each operand counted once per kernel):
#  - Jacobi/CG (pcg_kernel): reads p, x, r, s, w (4 B each) + code (2 B); writes p, x, r, s, w -> 42 B;
#  - multigrid FCG graph, level 0: update reads r, q, p, e, code, writes r', zp, e (30 B); prolongation reads code,
#    zp, writes zp (10 B); smoothing reads code, zp, r, q, writes z (18 B); p/q reads code, z, p, r, writes p', q
#    (22 B) -> 80 B; the coarser levels add 1/8 + 1/64 + ... of their 34 B (restriction 10, prolongation 10,
#    smoothing 14) plus the restricted right-hand sides -> 85 B per fine cell and iteration.
JACOBI_BYTES_PER_CELL_ITERATION = 42.0
MG_BYTES_PER_CELL_ITERATION = 85.0
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum over every kernel) of one multigrid FCG solve from zero
# on the 128^3 plume after the spin-up, 12 iterations, 1 pass: the kernels of the graph launched one by one
# (bench.py --profile solve, ncu --cache-control none so that L2 carries over between kernels as in the graph);
# 63.8 MB read + 447.9 MB written, per grid size. Scaled by iterations when a solve takes another count.
MG_SOLVE_DRAM_BYTES = {128: (511.7e6, 12)}


def solver_kernel_roofline(sim, n_cells, peak_gbs, peak_kind, repeats=5, bytes_per_iteration=JACOBI_BYTES_PER_CELL_ITERATION, kernel="pcg_kernel", traffic_table=None):
    """Times the pressure solve alone (smoke_b200_solve_pressure_cuda on the step's right-hand side: one graph launch
    on the context stream) with CUDA events on that stream; algorithmic bytes = cells x (bytes per iteration x
    iterations + set-up 24 B + 46 B per refinement pass)."""
    import torch

    flush = L2Flush()
    durs, iters = [], []
    passes = 1
    for _ in range(repeats):
        with torch.cuda.stream(sim.stream):
            flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(sim.stream)
        sim.solve_pressure()
        e1.record(sim.stream)
        sim.stream.synchronize()
        durs.append(e0.elapsed_time(e1))
        st = sim.solver_status()
        iters.append(st.iterations)
        passes = st.passes
    ms = statistics.median(durs)
    it = statistics.median(iters)
    algo_bytes = n_cells * (bytes_per_iteration * it + 24.0 + 46.0 * passes)
    achieved = algo_bytes / (ms * 1e-3) / 1e9
    n = round(n_cells ** (1.0 / 3.0))
    traffic = None
    if traffic_table and n in traffic_table:
        measured, measured_its = traffic_table[n]
        traffic = round(measured * it / measured_its)
    return {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1), "peak": peak_gbs, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": round(achieved / peak_gbs, 3), "traffic": traffic, "traffic_over_algorithmic": round(traffic / algo_bytes, 3) if traffic else None,
            "algorithmic_bytes_per_launch": algo_bytes, "launch_ms": round(ms, 4), "iterations": it,
            "bytes_per_cell_iteration": bytes_per_iteration,
            "note": ("traffic: DRAM bytes of one solve from an ncu capture of its kernels (cache control off, so L2 carries over as in the graph); "
                     "the working set (~90 MB at 128^3) stays mostly in the 126 MB L2, so the solve is bound by latency, not by HBM") if n_cells * 43 < 126e6 else
                    "the solve's arrays (about 43 B per cell) are far larger than L2, so the level-0 passes stream from HBM; no ncu traffic capture at this size"}


def divergence_norms(cfg, u, v, w):
    """(L2 / sqrt(cells), L-infinity) of the discrete divergence of face velocities (no solids), on the scale
    max|u| / h."""
    u, v, w = (np.asarray(a, np.float64) for a in (u, v, w))
    d = (u[:, :, 1:] - u[:, :, :-1] + v[:, 1:, :] - v[:, :-1, :] + w[1:, :, :] - w[:-1, :, :]) / cfg.cell_size
    scale = max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max()) / cfg.cell_size
    d = d / scale if scale > 0 else d
    return float(np.sqrt(np.mean(d * d))), float(np.abs(d).max())


def cpu_baseline(sim, driver, cfg, first_step, steps=2):
    """The oracle (C restatement, OpenMP on all host cores) on the GPU's states, and the GPU steps' errors against an
    FP64 oracle of the same steps.

    For each of `steps` consecutive steps from the GPU's current state S: the GPU takes the step (the form set on
    `sim`); the FP64 oracle takes the same step from S with the pressure solved to 1e-10 (the truth), and the density
    error (max-norm and L2, relative, and the cells whose error exceeds 1e-4 of the largest density) and the
    post-projection divergence (L2 and L-infinity, on the scale max|u| / h) of both are recorded. The timed CPU sample is the FP64 oracle taking the same steps from S with Jacobi-PCG to the GPU's
    tolerance, 1e-5."""
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    errors, cpu_ms, cpu_its = [], [], []
    for k in range(steps):
        driver.apply(first_step + k)
        u, v, w = sim.face_velocity_host(0)
        snap = sim.snapshot([abi.VIEW_DENSITY, abi.VIEW_TEMPERATURE, abi.VIEW_DENSITY_SOURCE, abi.VIEW_TEMPERATURE_SOURCE, abi.VIEW_FORCE])
        states = []
        for _ in range(2):
            st = O.OracleState(cfg, 64)
            st.set("u", u)
            st.set("v", v)
            st.set("w", w)
            for name in ("density", "temperature", "density_source", "temperature_source"):
                st.set(name, snap[name])
            for ax in "xyz":
                st.set(f"force_{ax}", snap[f"force_{ax}"])
            states.append(st)
        sim.step()
        gu, gv, gw = sim.face_velocity_host(0)
        gd = sim.snapshot([abi.VIEW_DENSITY])["density"]
        gst = sim.solver_status()
        torch.cuda.synchronize()
        truth = states[0].step(0, 5, mode=1, max_iterations=8000, tolerance=1e-10)
        t0 = time.perf_counter()
        timed = states[1].step(0, 5, mode=1, max_iterations=3000, tolerance=1e-5)
        cpu_ms.append((time.perf_counter() - t0) * 1e3)
        cpu_its.append(timed.iterations)
        t = states[0]
        d_gpu = divergence_norms(cfg, gu, gv, gw)
        d_64 = divergence_norms(cfg, t["u"], t["v"], t["w"])
        dd = np.abs(gd - t["density"])
        dmax = np.abs(t["density"]).max()
        errors.append({"density_rel_err": float(dd.max() / dmax),
                       "density_rel_err_l2": float(np.linalg.norm(gd - t["density"]) / np.linalg.norm(t["density"])),
                       "density_cells_above_1e-4": int((dd > 1e-4 * dmax).sum()),
                       "divergence_l2_gpu": d_gpu[0], "divergence_linf_gpu": d_gpu[1], "divergence_l2_fp64": d_64[0], "divergence_linf_fp64": d_64[1],
                       "gpu_iterations": gst.iterations, "gpu_true_rel_residual": gst.true_relative_residual, "fp64_oracle_rel_residual": truth.relative_residual})
    cpu = {"value": round(statistics.mean(cpu_ms), 1), "unit": "ms/step", "cores": os.cpu_count(), "kind": "port",
           "sample": f"{steps} full steps of the 128^3 plume from the GPU's states (FP64 oracle, Jacobi-PCG to rel-res 1e-5, {cpu_its} iterations)"}
    accuracy = {"vs": "FP64 oracle of the same step from the same state, pressure solved to rel-res 1e-10", "steps": errors}
    return cpu, accuracy


def build_sim(lib, cfg, stream):
    import smoke_b200

    return smoke_b200.Simulation(lib, cfg, stream)


# Solver forms measured on the same plume states. The headline ("value") is the first one: multigrid FCG that starts
# each step's solve from the previous step's FP64 pressure (warm start) and stops on the same test as a cold start,
# ||b - A x|| <= 1e-5 ||b||; the cold form is measured beside it. One FP32 pass reaches 1e-5 on these scenes; a
# second (refinement = 1) is the margin, and the graph carries no further unrolled passes that would launch as no-ops.
FORMS = {
    "multigrid_fp64": dict(mode=abi.SOLVER_MG_FCG, reduction=abi.REDUCTION_FP64, max_iterations=500, tolerance=1e-5, refinement=1, warm_start=True),
    "multigrid_fp64_cold": dict(mode=abi.SOLVER_MG_FCG, reduction=abi.REDUCTION_FP64, max_iterations=500, tolerance=1e-5, refinement=1),
    "jacobi_fp64": dict(mode=abi.SOLVER_JACOBI_PCG, reduction=abi.REDUCTION_FP64, max_iterations=3000, tolerance=1e-5, refinement=3),
    "plain_fp32": dict(mode=abi.SOLVER_JACOBI_PCG, reduction=abi.REDUCTION_FP32, max_iterations=1500, tolerance=1e-5, refinement=0),
}
HEADLINE = "multigrid_fp64"
# The learned+mixed form the metric names: the same FCG with the V-cycle's result corrected by the tcgen05 U-Net on the
# multigrid level 1 (z = V(r) + P N(R(r - A V(r)))), FP64 dots and refinement, warm start; measured when the package's
# trained weights exist, and from zero beside the multigrid form from zero.
LEARNED_NAME = "learned_fp64"
LEARNED_FORM = dict(mode=abi.SOLVER_LEARNED_FCG, reduction=abi.REDUCTION_FP64, max_iterations=500, tolerance=1e-5, refinement=1, warm_start=True)
# Schedules of the learned form, measured before the forms: the network in the first k iterations of each pass only
# (0: in every iteration); the fastest one that meets the tolerance is the learned form's schedule.
LEARNED_SCHEDULES = (1, 2, 4, 0)


def bench_b200(args, rank, world, local):
    import torch

    import plume_scene
    import smoke_b200

    n = args.n
    lib = smoke_b200.SmokeLibrary()
    stream = torch.cuda.Stream()
    cfg = plume_scene.plume_config(n, abi.MONOTONIC_CUBIC)
    sim = smoke_b200.Simulation(lib, cfg, stream)
    driver = plume_scene.PlumeDriver(sim, n, seed=1 + rank)
    net = learned_net(lib)
    forms = dict(FORMS)
    headline = HEADLINE
    if net is not None:  # the learned+mixed form leads: it is the form the metric names
        sim.set_preconditioner_net(net)
        forms = {LEARNED_NAME: LEARNED_FORM, **FORMS, LEARNED_NAME + "_cold": dict(LEARNED_FORM, warm_start=False)}
        headline = LEARNED_NAME
    sim.set_solver(**FORMS[HEADLINE])
    flush = L2Flush()
    # spin-up (untimed): the plume develops from rest
    run_steps(sim, driver, 0, SPINUP_STEPS, None)
    state = save_state(sim)
    step0 = SPINUP_STEPS
    results = {}
    tunes = {}
    clocks = None
    schedules = {}
    schedule = 0
    if net is not None:  # the learned form's schedule: the fastest that meets the tolerance
        for k in LEARNED_SCHEDULES:
            restore_state(sim, state)
            sim.set_solver(**LEARNED_FORM)
            sim.set_learned_iterations(k)
            run_steps(sim, driver, step0, args.warmup, flush)
            barrier(world)
            t, its, res = run_steps(sim, driver, step0 + args.warmup, args.steps, flush, status=True)
            schedules[k] = (max_over_ranks(statistics.mean(t), world), statistics.mean(its), max(res))
        ok = [k for k, v in schedules.items() if v[2] <= LEARNED_FORM["tolerance"]] or list(schedules)
        schedule = min(ok, key=lambda k: schedules[k][0])
        sim.set_learned_iterations(schedule)
    for name, form in forms.items():
        restore_state(sim, state)
        sim.set_solver(**form)
        if args.tune:  # launch shapes for this solver form (the tuner restores the state it timed on)
            tunes[name] = sim.autotune()
        run_steps(sim, driver, step0, args.warmup, flush)
        barrier(world)
        torch.cuda.synchronize()
        if name == headline:
            with ClockSampler(local) as clocks:
                t, its, res = run_steps(sim, driver, step0 + args.warmup, args.steps, flush, status=True)
        else:
            t, its, res = run_steps(sim, driver, step0 + args.warmup, args.steps, flush, status=True)
        torch.cuda.synchronize()
        barrier(world)
        flags = sim.solver_status().flags
        results[name] = (max_over_ranks(statistics.mean(t), world), statistics.mean(its), max(res), flags)
    learned = bench_learned(sim, net, n, results.get(LEARNED_NAME), results) if net is not None else {"unavailable": "no trained weights in the package"}
    if schedules:
        learned["schedule"] = schedule_name(schedule)
        learned["schedules"] = {schedule_name(k): {"ms_per_step": round(v[0], 4), "pcg_iterations": round(v[1], 1), "true_rel_residual_max": v[2]}
                                for k, v in schedules.items()}
    # e2e through the ABI (headline form), same state
    restore_state(sim, state)
    sim.set_solver(**forms[headline])
    if args.tune:
        sim.autotune()  # cached: the headline form's shapes
    run_e2e(sim, driver, step0, args.warmup)
    barrier(world)
    e2e_ms, _ = run_e2e(sim, driver, step0 + args.warmup, args.steps)
    barrier(world)
    e2e_ms = max_over_ranks(e2e_ms, world)
    # the oracle on the host cores, and the headline form's per-step error against the FP64 oracle of the same step
    cpu, accuracy = cpu_baseline(sim, driver, cfg, step0 + args.warmup + args.steps) if (rank == 0 and world == 1 and not args.no_cpu_baseline) else (None, None)
    # the solve alone, cold (a warm start would begin each repeat from the converged answer of the previous one)
    sim.set_solver(**FORMS["multigrid_fp64_cold"])
    roof = solver_kernel_roofline(sim, n ** 3, *load_peaks(), bytes_per_iteration=MG_BYTES_PER_CELL_ITERATION, kernel="multigrid-preconditioned FCG solve from zero (one graph launch of the mg_* kernels)", traffic_table=MG_SOLVE_DRAM_BYTES)
    sim.close()
    if net is not None:
        net.close()
    if rank != 0:
        return None
    cells = n ** 3
    ms, its, res, _ = results[headline]
    line = {
        "metric": METRIC, "value": round(ms, 4), "unit": "ms/step", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (fp64 reductions)", "data": "synthetic (seeded plume scene)",
        "config": {"workload": f"plume {n}^3 monotone-cubic; pressure to rel-res 1e-5: " + (
                       "learned+mixed: flexible CG preconditioned by a multigrid V-cycle corrected by the tcgen05 BF16 U-Net (4 levels, 16/32/64/128 channels) run on the multigrid level 1, FP32 stencils, FP64 dots and refinement, warm start"
                       if headline == LEARNED_NAME else "multigrid-preconditioned FCG, FP64 dots, FP64 refinement, warm start from the previous step's pressure"), "grid": [n, n, n], "dt": 0.01,
                   "source_box": "16x8x16 at x,z in [56,72), y in [0,8)" if n == 128 else "n/8 x n/16 x n/8", "spinup_steps": SPINUP_STEPS,
                   "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "learned_preconditioner": f"headline form, {schedule_name(schedule)}" if headline == LEARNED_NAME else "not used (no trained weights)"},
        "pcg_iterations": round(its, 1), "true_rel_residual_max": res,
        "cells_per_s": round(cells * world / (ms * 1e-3), 1),
        "forms": {k: {"ms_per_step": round(v[0], 4), "pcg_iterations": round(v[1], 1), "rel_residual_max": v[2]} for k, v in results.items()},
        "headline_form": headline,
        "speedup_vs_plain_fp32": round(results["plain_fp32"][0] / ms, 2),
        "roofline": roof,
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms/step", "h2d_bytes_per_step": driver.h2d_bytes, "d2h_bytes_per_step": driver.d2h_bytes,
                "includes": "per-step box inputs H2D, velocity/density/temperature views, source/force updates, step, total-density D2H, host sync"},
        "gpu_launches": round(args.steps * (STEP_KERNELS + 1 + solver_launches(n, its, forms[headline]["refinement"], learned=headline == LEARNED_NAME, net_iterations=schedule))),
        "clocks": clocks.summary() if clocks is not None else None,
        "launch_tune": {k: tune_summary(v) for k, v in tunes.items()} if tunes else "defaults (--no-tune)",
        "learned": learned,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
        line["accuracy"] = accuracy
    return line



# (cin, cout, level) of the network's convolutions (unet.h: 4 levels, 16/32/64/128 channels)
NET_LAYERS = [(2, 16, 0), (16, 32, 1), (32, 64, 2), (64, 128, 3), (128, 64, 3), (64, 32, 2), (32, 16, 1), (16, 1, 0)]


def schedule_name(k):
    return "network in every iteration" if k == 0 else f"network in the first {k} iteration{'s' if k > 1 else ''} of a pass"


def net_flops(nx, ny, nz, executed=False):
    """FLOPs of one network evaluation: 2 * 27 * cin * cout per cell of each layer's level, with the real channel
    counts (dense), or with the channels the tensor cores run (executed: inputs of at most 8 channels padded to 8,
    outputs to a multiple of 16)."""
    dims = [(nx, ny, nz)]
    for _ in range(3):
        dims.append(tuple((v + 1) // 2 for v in dims[-1]))
    total = 0
    for ci, co, l in NET_LAYERS:
        if executed:
            ci, co = (8 if ci <= 8 else ci), -(-co // 16) * 16
        total += 2 * 27 * ci * co * dims[l][0] * dims[l][1] * dims[l][2]
    return total


def learned_net(lib):
    """The network with the package's trained weights, or None when the package has none."""
    import smoke_b200
    import train_preconditioner

    if not os.path.exists(train_preconditioner.DEFAULT_WEIGHTS):
        return None
    net = smoke_b200.Net(lib, seed=0)
    train_preconditioner.load(net)
    return net


def bench_learned(sim, net, n, learned, results):
    """The learned form's figures beside the plain FP32 form (the metric's comparison), and the network evaluation
    alone: ms per apply on the multigrid level 1 of the step's right-hand side (the volume the solve runs it on), and
    on the full n^3 grid with its tensor FLOP rate against the measured BF16 peak."""
    import torch

    import train_preconditioner

    with torch.cuda.stream(sim.stream):
        rhs = sim.view(abi.VIEW_FLOW_PRESSURE_RHS).clone()
        occ = torch.zeros(rhs.shape, dtype=torch.uint8, device="cuda")
        rhs1 = train_preconditioner._children(rhs).sum(-1).contiguous()  # the solve's restriction onto level 1
        occ1 = torch.zeros(rhs1.shape, dtype=torch.uint8, device="cuda")
    sim.stream.synchronize()

    def time_apply(x, o, reps=20):
        net.apply(x, o)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            net.apply(x, o)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    apply1_ms, apply_ms = time_apply(rhs1, occ1), time_apply(rhs, occ)
    n1 = (n + 1) // 2
    flops, executed = net_flops(n, n, n), net_flops(n, n, n, executed=True)
    tflops, tflops_exec = flops / (apply_ms * 1e-3) / 1e12, executed / (apply_ms * 1e-3) / 1e12
    bf16_peak = peak_tflops()
    ms, its, res, flags = learned
    plain = results["plain_fp32"][0]
    return {"form": "FCG, z = V(r) + P N(R(r - A V(r))): multigrid V(1,1) cycle corrected by the tcgen05 BF16 U-Net (4 levels, 16/32/64/128 channels, 582257 parameters) run on the multigrid level 1 "
                    f"({n1}^3; R: child sums, P: the V-cycle's trilinear prolongation), FP32 stencils, FP64 dots + refinement, warm start, to 1e-5",
            "ms_per_step": round(ms, 4), "pcg_iterations": round(its, 1), "true_rel_residual_max": res, "network_dropped": bool(flags & 1),
            "speedup_vs_plain_fp32": round(plain / ms, 2), "target": "learned+mixed >= 3x faster per step than plain FP32 PCG", "target_met": bool(plain / ms >= 3.0),
            "vs_multigrid_alone": round(results["multigrid_fp64"][0] / ms, 3),
            "net_apply_ms": round(apply1_ms, 4), "net_apply_grid": [n1, n1, n1], "net_dense_gflop_per_apply": round(net_flops(n1, n1, n1) / 1e9, 2),
            "net_apply_full_grid_ms": round(apply_ms, 4), "net_full_grid_dense_gflop": round(flops / 1e9, 2), "net_full_grid_executed_gflop": round(executed / 1e9, 2),
            "tensor_roofline": {"bound": "tensor", "achieved": round(tflops, 2), "achieved_executed": round(tflops_exec, 2), "peak": bf16_peak, "unit": "TFLOP/s", "frac": round(tflops / bf16_peak, 5),
                                "note": f"one network evaluation (input packing, 8 convolutions, 3 pools, 3 up-adds) on the full {n}^3 right-hand side; dense FLOPs of the real channels, and the FLOPs the tensor cores execute with the padded channels"}}


def tune_summary(rep):
    """The autotuner's choice in words, with the step times it measured for the default and chosen shapes."""
    c = rep["chosen"]
    out = {"advect_tile": abi.ADVECT_TILE_NAMES[c["advect_tile"]], "mg_wave": abi.MG_WAVE_NAMES[c["mg_wave"]], "pcg_grid": abi.PCG_GRID_NAMES[c["pcg_grid"]],
           "pcg_regs": abi.PCG_REGS_NAMES[c["pcg_regs"]]}
    if not rep["from_cache"]:
        out.update(default_ms=round(rep["default_ms"], 4), chosen_ms=round(rep["chosen_ms"], 4), candidates=len(rep["records"]))
    return out


def _line(metric, ms, args, world, config, **extra):
    line = {"metric": metric, "value": round(ms, 4), "unit": "ms/step", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (fp64 reductions)", "data": "synthetic (seeded plume scenes)", "config": config}
    line.update(extra)
    return line


def bench_plume64(args, rank, world, local):
    """Config 1: the plain method at 64^3 (trilinear advection, Jacobi-PCG to 1e-5, at most 500 iterations), with the
    multigrid form on the same states beside it."""
    import torch

    import plume_scene
    import smoke_b200

    n = 64
    lib = smoke_b200.SmokeLibrary()
    stream = torch.cuda.Stream()
    cfg = plume_scene.plume_config(n, abi.LINEAR)
    sim = smoke_b200.Simulation(lib, cfg, stream)
    driver = plume_scene.PlumeDriver(sim, n, seed=1 + rank)
    forms = {"plain_fp32_jacobi": dict(mode=abi.SOLVER_JACOBI_PCG, reduction=abi.REDUCTION_FP32, max_iterations=500, tolerance=1e-5, refinement=0),
             "multigrid_fp64": FORMS["multigrid_fp64"]}
    sim.set_solver(**forms["plain_fp32_jacobi"])
    run_steps(sim, driver, 0, SPINUP_STEPS, None)
    state = save_state(sim)
    flush = L2Flush()
    results, clocks, tunes = {}, None, {}
    for name, form in forms.items():
        restore_state(sim, state)
        sim.set_solver(**form)
        if args.tune:
            tunes[name] = tune_summary(sim.autotune())
        run_steps(sim, driver, SPINUP_STEPS, args.warmup, flush)
        barrier(world)
        with ClockSampler(local) as c:
            t, its, res = run_steps(sim, driver, SPINUP_STEPS + args.warmup, args.steps, flush, status=True)
        clocks = clocks or c
        results[name] = (max_over_ranks(statistics.mean(t), world), statistics.mean(its), max(res))
    sim.close()
    if rank != 0:
        return None
    ms, its, res = results["plain_fp32_jacobi"]
    return _line("ms/step and PCG iterations at 64^3 to rel-res 1e-5 (plain method)", ms, args, world,
                 {"workload": "plume 64^3, trilinear, closed walls, source 8x4x8 at the bottom centre; Jacobi-PCG FP32 to 1e-5 (max 500)", "grid": [n, n, n],
                  "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas x{world}"},
                 dtype="f32", pcg_iterations=round(its, 1), rel_residual_max=res, cells_per_s=round(n ** 3 * world / (ms * 1e-3), 1),
                 forms={k: {"ms_per_step": round(v[0], 4), "pcg_iterations": round(v[1], 1), "rel_residual_max": v[2]} for k, v in results.items()},
                 clocks=clocks.summary() if clocks else None, launch_tune=tunes or "defaults (--no-tune)")


def bench_large(args, rank, world, local):
    """Config 3: 256 x 384 x 256 with a solid sphere and two plume sources, multigrid FCG to 1e-5."""
    import torch

    import plume_scene
    import smoke_b200

    cfg, occ, boxes = plume_scene.large_scene(seed=1 + rank)
    lib = smoke_b200.SmokeLibrary()
    stream = torch.cuda.Stream()
    sim = smoke_b200.Simulation(lib, cfg, stream)
    with torch.cuda.stream(stream):
        occ_dev = torch.from_numpy(occ).cuda()
        sim.update_occupancy(occ_dev)
    stream.synchronize()
    sim.set_solver(**FORMS[HEADLINE])
    driver = plume_scene.SceneDriver(sim, boxes, seed=1 + rank)
    flush = L2Flush()
    spin = 10
    run_steps(sim, driver, 0, spin, flush)
    tune = tune_summary(sim.autotune()) if args.tune else "defaults (--no-tune)"
    run_steps(sim, driver, spin, args.warmup, flush)
    barrier(world)
    with ClockSampler(local) as clocks:
        t, its, res = run_steps(sim, driver, spin + args.warmup, args.steps, flush, status=True)
    cells = cfg.nx * cfg.ny * cfg.nz
    sim.set_solver(**FORMS["multigrid_fp64_cold"])  # the solve alone, from zero
    roof = solver_kernel_roofline(sim, cells, *load_peaks(), repeats=3, bytes_per_iteration=MG_BYTES_PER_CELL_ITERATION, kernel="multigrid-preconditioned FCG solve from zero (one graph launch of the mg_* kernels)", traffic_table=MG_SOLVE_DRAM_BYTES)
    sim.close()
    ms = max_over_ranks(statistics.mean(t), world)
    if rank != 0:
        return None
    return _line("ms/step and PCG iterations, 256x384x256 scene with a solid sphere, to rel-res 1e-5", ms, args, world,
                 {"workload": "256x384x256, h=1/256, sphere r=40 cells at (128, 153.6, 128), two 32x8x32 floor sources, monotone cubic; multigrid FCG, FP64 dots + refinement, warm start",
                  "grid": [cfg.nx, cfg.ny, cfg.nz], "spinup_steps": spin, "l2": "inputs (25.2 M cells) larger than L2; also flushed", "parallelism": f"replicas x{world}"},
                 pcg_iterations=round(statistics.mean(its), 1), true_rel_residual_max=max(res), cells_per_s=round(cells * world / (ms * 1e-3), 1), roofline=roof,
                 clocks=clocks.summary(), launch_tune=tune)


def bench_batched(args, rank, world, local):
    """Config 5: 48 independent plumes of uneven sizes and obstacles advanced together by one graph launch per
    step (smoke_b200_batch_step_cuda); each scene also stepped alone for the per-scene latency distribution."""
    import torch

    import plume_scene
    import smoke_b200

    scenes_ = plume_scene.batched_scenes(48, seed=1 + rank)
    lib = smoke_b200.SmokeLibrary()
    sims, drivers, keep = [], [], []
    for cfg, occ, boxes in scenes_:
        stream = torch.cuda.Stream()
        sim = smoke_b200.Simulation(lib, cfg, stream)
        with torch.cuda.stream(stream):
            o = torch.from_numpy(occ).cuda()
            sim.update_occupancy(o)
        keep.append(o)
        sim.set_solver(**FORMS[HEADLINE])
        sims.append(sim)
        drivers.append(plume_scene.SceneDriver(sim, boxes, seed=1 + rank))
    torch.cuda.synchronize()
    cells = sum(s.config.nx * s.config.ny * s.config.nz for s in sims)
    flush = L2Flush()
    # solo: one step per scene alone (after a short spin-up), for the per-scene latency distribution
    solo = []
    tuned = 0
    for k, (sim, drv) in enumerate(zip(sims, drivers)):
        run_steps(sim, drv, 0, 3, None)
        if args.tune:
            tuned += 0 if sim.autotune(steps=2)["from_cache"] else 1
        t, _, _ = run_steps(sim, drv, 3, 2, flush)
        solo.append(min(t))
    batch_stream = torch.cuda.Stream()
    batch = smoke_b200.Batch(sims, batch_stream)

    inside = []  # per-scene latency inside the batch: batch start to the end of the scene's branch (graph events)

    def batch_steps(first, count, timed):
        times = []
        for k in range(count):
            for sim, drv in zip(sims, drivers):
                drv.apply(first + k)
            with torch.cuda.stream(batch_stream):
                flush()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(batch_stream)
            batch.step()
            e1.record(batch_stream)
            batch_stream.synchronize()
            times.append(e0.elapsed_time(e1))
            if timed:
                inside.extend(batch.member_times().tolist())
        return times

    batch_steps(5, args.warmup, False)
    barrier(world)
    with ClockSampler(local) as clocks:
        bt = batch_steps(5 + args.warmup, args.steps, True)
    iters = [s.solver_status().iterations for s in sims]
    batch.close()
    # the same batch with the learned+mixed form (the network corrects the V-cycle in the first iteration of each
    # pass, the schedule the 128^3 plume measures fastest), one graph launch per batched step again
    learned = None
    net = learned_net(lib)
    if net is not None:
        for sim in sims:
            sim.set_preconditioner_net(net)
            sim.set_solver(**LEARNED_FORM)
            sim.set_learned_iterations(1)
        batch = smoke_b200.Batch(sims, batch_stream)
        inside_mg, inside = inside, []
        batch_steps(5 + args.warmup + args.steps, args.warmup, False)
        lt = batch_steps(5 + 2 * args.warmup + args.steps, args.steps, True)
        lits = [s.solver_status().iterations for s in sims]
        dropped = sum(1 for s in sims if s.solver_status().flags & 1)
        batch.close()
        lms = max_over_ranks(statistics.mean(lt), world)
        learned = {"ms_per_batched_step": round(lms, 4), "cells_per_s": round(cells * world / (lms * 1e-3), 1),
                   "scene_latency_in_batch_ms": {"p50": round(float(np.percentile(inside, 50)), 4), "p99": round(float(np.percentile(inside, 99)), 4), "max": round(max(inside), 4)},
                   "pcg_iterations": {"min": min(lits), "max": max(lits), "mean": round(statistics.mean(lits), 1)}, "network_dropped_scenes": dropped,
                   "form": "learned FCG (V-cycle corrected by the tcgen05 U-Net in the first iteration of each pass), FP64 dots and refinement, warm start, to 1e-5"}
        inside = inside_mg
        net.close()
    for s in sims:
        s.close()
    ms = max_over_ranks(statistics.mean(bt), world)
    if rank != 0:
        return None
    solo_sorted = sorted(solo)
    return _line("ms per batched step of 48 uneven plumes (aggregate cells/s, per-scene latency)", ms, args, world,
                 {"workload": "48 plumes, extents drawn in [32,128]x[32,192]x[32,128], one floor source and 0-3 spheres each, monotone cubic, multigrid FCG to 1e-5 with warm start; one graph launch per batched step",
                  "scenes": len(sims), "cells": cells, "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas x{world}"},
                 cells_per_s=round(cells * world / (ms * 1e-3), 1),
                 scene_latency_in_batch_ms={"p50": round(float(np.percentile(inside, 50)), 4), "p99": round(float(np.percentile(inside, 99)), 4), "max": round(max(inside), 4),
                                            "note": "from the start of the batch graph to the end of the scene's step inside it, every scene of every timed batch step"},
                 solo_step_ms={"p50": round(statistics.median(solo), 4), "p99": round(solo_sorted[min(len(solo) - 1, int(0.99 * len(solo)))], 4), "sum": round(sum(solo), 3)},
                 batch_speedup_vs_sequential=round(sum(solo) / ms, 2), pcg_iterations={"min": min(iters), "max": max(iters), "mean": round(statistics.mean(iters), 1)},
                 clocks=clocks.summary(), launch_tune=f"each scene autotuned alone before the batch ({tuned} timed, {len(sims) - tuned} from the cache)" if args.tune else "defaults (--no-tune)",
                 learned=learned if learned is not None else {"unavailable": "no trained weights in the package"})


def other_configs(args, rank, world, local):
    """Short runs of the other benchmark configurations after the headline (5 timed steps after 3 warm-up steps
    each; the full runs are `--workload plume64 | large | batched`): the 64^3 plain method (C1), the 256x384x256 scene
    with a sphere (C3) and the 48-scene batch (C5), each line as its own workload prints it. Every rank runs them."""
    import copy

    import torch

    sub = copy.copy(args)
    sub.steps, sub.warmup = min(args.steps, 5), 3
    out = {}
    for name, fn in (("C1_plume64_plain", bench_plume64), ("C3_large_256x384x256", bench_large), ("C5_batched_48", bench_batched)):
        t0 = time.perf_counter()
        res = fn(sub, rank, world, local)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        if res is not None:
            res["wall_s"] = round(time.perf_counter() - t0, 1)
            out[name] = res
    return out


def bench_reference(args, rank, world, local):
    import torch

    import plume_scene
    import smoke_b200

    if rank != 0:
        return None
    if not os.path.exists(REF_LIBRARY):
        return {"impl": "reference", "unavailable": f"reference library not built ({REF_LIBRARY}); oracle/build_oracle.py builds it from the reference sources"}
    n = args.n
    lib = smoke_b200.SmokeLibrary(REF_LIBRARY, extensions=False)
    stream = torch.cuda.Stream()
    cfg = plume_scene.plume_config(n, abi.MONOTONIC_CUBIC, pressure_iterations=REFERENCE_CG_ITERATIONS)
    sim = smoke_b200.Simulation(lib, cfg, stream)
    driver = plume_scene.PlumeDriver(sim, n, seed=1)
    flush = L2Flush()
    run_steps(sim, driver, 0, SPINUP_STEPS + args.warmup, flush)
    with ClockSampler(local) as clocks:
        t, _, _ = run_steps(sim, driver, SPINUP_STEPS + args.warmup, args.steps, flush)
    e2e_ms, _ = run_e2e(sim, driver, SPINUP_STEPS + args.warmup + args.steps, args.steps)
    sim.close()
    ms = statistics.mean(t)
    sample = f"{args.steps} steps of the {n}^3 plume after {SPINUP_STEPS + args.warmup} untimed steps, reference CUDA/cuSPARSE build, {REFERENCE_CG_ITERATIONS} fixed CG iterations"
    return {
        "metric": METRIC, "impl": "reference", "value": round(ms, 4), "unit": "ms/step", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plume scene)",
        "config": {"workload": f"plume {n}^3 monotone-cubic, reference fixed CG x{REFERENCE_CG_ITERATIONS} (smallest count reaching its FP32 floor, rel-res ~2.5e-5)", "grid": [n, n, n],
                   "l2": "flushed between timed steps (256 MiB write)"},
        "pcg_iterations": REFERENCE_CG_ITERATIONS,
        "cpu_baseline": {"value": round(ms, 4), "unit": "ms/step", "cores": 1, "kind": "reference", "sample": sample,
                         "where": "the reference has no CPU implementation; its own CUDA build runs on the same B200, driven by one host thread"},
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms/step", "h2d_bytes_per_step": driver.h2d_bytes, "d2h_bytes_per_step": driver.d2h_bytes},
        "clocks": clocks.summary(),
    }


def profile_workload(args):
    """Profiling workloads (for ncu; prints one status line, no benchmark JSON): the 128^3 plume after the spin-up,
    then --profile-count repetitions of: `solve` an eager multigrid solve (every kernel a plain launch), `learned-solve`
    an eager learned solve (packaged weights), `solve-graph`
    the multigrid solve graph, `step` an eager step (stage kernels launched one by one, the solve as its graph), `net`
    the learned preconditioner's network on the step's right-hand side (packaged weights)."""
    import torch

    import plume_scene
    import smoke_b200

    n = args.n
    lib = smoke_b200.SmokeLibrary()
    stream = torch.cuda.Stream()
    sim = smoke_b200.Simulation(lib, plume_scene.plume_config(n, abi.MONOTONIC_CUBIC), stream)
    driver = plume_scene.PlumeDriver(sim, n, seed=1)
    sim.set_solver(**FORMS["multigrid_fp64_cold"])  # profiled solves start from zero
    if args.shapes:  # explicit launch shapes (the autotuner's timing launches stay out of the profile)
        a, w, g = (int(v) for v in args.shapes.split(","))
        sim.set_launch_tune(advect_tile=a, mg_wave=w, pcg_grid=g)
    run_steps(sim, driver, 0, SPINUP_STEPS, None)
    if args.profile == "learned-solve":  # the learned form's solve from zero, every kernel a plain launch
        net = learned_net(lib)
        sim.set_preconditioner_net(net)
        sim.set_solver(**dict(LEARNED_FORM, warm_start=False))
    if args.profile == "net":  # the learned preconditioner's network on the step's right-hand side
        import train_preconditioner

        net = smoke_b200.Net(lib, seed=0)
        train_preconditioner.load(net)
        with torch.cuda.stream(stream):
            rhs = sim.view(abi.VIEW_FLOW_PRESSURE_RHS).clone()
            occ = torch.zeros(rhs.shape, dtype=torch.uint8, device="cuda")
        stream.synchronize()
        torch.cuda.cudart().cudaProfilerStart()  # ncu --profile-from-start off captures from here
        for k in range(args.profile_count):
            out = net.apply(rhs, occ)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
        print(json.dumps({"profile": "net", "count": args.profile_count, "out_norm": float(out.norm())}), flush=True)
        net.close()
        sim.close()
        return
    stream.synchronize()
    torch.cuda.cudart().cudaProfilerStart()  # ncu --profile-from-start off captures from here
    for k in range(args.profile_count):
        if args.profile == "step":
            driver.apply(SPINUP_STEPS + k)
            sim.step_stages(abi.STAGE_SCALARS)
        else:
            sim.solve_pressure(eager=args.profile in ("solve", "learned-solve"))
    stream.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    st = sim.solver_status()
    print(json.dumps({"profile": args.profile, "count": args.profile_count, "iterations": st.iterations, "passes": st.passes, "status": st.status,
                      "true_rel_residual": st.true_relative_residual}), flush=True)
    sim.close()


def calibrate_reference(args):
    """Fixed CG counts vs achieved relative residual ||b - A p|| / ||b|| of the reference on the plume scene."""
    import torch

    import plume_scene
    import smoke_b200

    lib = smoke_b200.SmokeLibrary(REF_LIBRARY, extensions=False)
    out = {}
    for iters in args.calibrate_counts:
        stream = torch.cuda.Stream()
        cfg = plume_scene.plume_config(args.n, abi.MONOTONIC_CUBIC, pressure_iterations=iters)
        sim = smoke_b200.Simulation(lib, cfg, stream)
        driver = plume_scene.PlumeDriver(sim, args.n, seed=1)
        run_steps(sim, driver, 0, SPINUP_STEPS, None)
        worst = 0.0
        for k in range(10):
            run_steps(sim, driver, SPINUP_STEPS + k, 1, None)
            with torch.cuda.stream(stream):
                p = sim.view(abi.VIEW_FLOW_PRESSURE).double()
                b = sim.view(abi.VIEW_FLOW_PRESSURE_RHS).double()
                worst = max(worst, float(plume_scene.closed_box_residual(p, b)))
        sim.close()
        out[iters] = worst
        print(json.dumps({"reference_cg_iterations": iters, "max_rel_residual": worst}), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--calibrate-reference", action="store_true")
    ap.add_argument("--calibrate-counts", type=int, nargs="*", default=[200, 300, 400, 500, 600, 800, 1000])
    ap.add_argument("--profile", choices=["solve", "solve-graph", "step", "net", "learned-solve"], help="run a profiling workload instead of the benchmark")
    ap.add_argument("--workload", default="plume128", choices=["plume128", "plume64", "large", "batched"],
                    help="plume128: the headline (default); plume64, large, batched: the other benchmark configurations")
    ap.add_argument("--profile-count", type=int, default=1)
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="keep the default launch shapes (skip the autotuner)")
    ap.add_argument("--no-other-configs", dest="other_configs", action="store_false",
                    help="plume128 only: skip the short runs of the other configurations (64^3 plain, 256x384x256, 48-scene batch) that the line carries")
    ap.add_argument("--shapes", default="", help="--profile only: launch shapes 'advect_tile,mg_wave,pcg_grid' (default: the defaults)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_setup(args.gpus)
    if args.calibrate_reference:
        calibrate_reference(args)
        return
    if args.profile:
        profile_workload(args)
        return
    if args.impl == "reference":
        line = bench_reference(args, rank, world, local)
    else:
        line = {"plume128": bench_b200, "plume64": bench_plume64, "large": bench_large, "batched": bench_batched}[args.workload](args, rank, world, local)
        if args.workload == "plume128" and args.other_configs:
            others = other_configs(args, rank, world, local)
            if line is not None:
                line["other_configs"] = others
    barrier(world) if args.impl == "b200" else None
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
