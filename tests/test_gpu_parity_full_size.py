"""Parity at the benchmark sizes, against the FP64 oracle and the reference's own library.

1. One step from an identical seeded state (the bar: per field, normwise max|gpu - fp64| / max|fp64| <= 1e-5):
   the 64^3 plume (closed walls, trilinear advection) and the 128^3 plume (monotone cubic advection) are spun up on
   the GPU; their state (face velocities, density, temperature, the step's sources and forces) is loaded into the
   FP64 oracle; both take one step with the pressure solved far below the tolerance (GPU: multigrid FCG with FP64
   refinement to 1e-9 from zero; oracle: FP64 Jacobi-PCG to 1e-10). Also recorded: the post-projection divergence
   (L2 and L-infinity on the scale max|u| / h) of both.
2. A deep solid: a sphere of radius 9 cells in a 32^3 box, so the density fill of solid cells walks several
   Chebyshev shells (backend-cuda.cu:1243-1290), one step against the FP32 and FP64 oracles.
3. The reference library (backend-cuda.cu built from its sources) and this one, from rest through the same ABI
   calls with the same per-step plume inputs, against the FP64 oracle stepped with the same inputs. The reference
   runs its fixed-count FP32 CG (500 iterations at 64^3, 900 at 128^3: its FP32 floor), this library the
   multigrid FCG with FP64 reductions and refinement to 1e-7. The reference's own distance to the FP64 oracle is its
   floor; this library must be within max(1e-5, that floor) of the oracle on every field.
"""
import json
import os

import numpy as np
import pytest
import torch

import oracle as O
import plume_scene
import scenes
import smoke_abi as abi
import smoke_b200

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIBRARY = os.path.join(ROOT, "oracle", "_ref", "libvisual-simulation-of-smoke.so")
REPORT = os.environ.get("SMOKE_PARITY_REPORT")
BAR = 1e-5  # per-field normwise relative error of one step from an identical state

SIZES = {"plume64_linear": (64, abi.LINEAR, 12), "plume128_cubic": (128, abi.MONOTONIC_CUBIC, 12)}


def report(name, value):
    if REPORT:
        with open(REPORT, "a") as f:
            f.write(json.dumps({"check": name, "value": value}) + "\n")


def face_arrays(sim, which=0):
    with torch.cuda.stream(sim.stream):
        t = [x.clone() for x in sim.face_velocity(which)]
    sim.stream.synchronize()
    return [x.cpu().numpy() for x in t]


def divergence_norms(cfg, u, v, w, occ):
    """(L2 / sqrt(fluid cells), L-infinity) of the discrete divergence over fluid cells, on the scale max|u| / h."""
    u, v, w = (np.asarray(a, np.float64) for a in (u, v, w))
    d = (u[:, :, 1:] - u[:, :, :-1] + v[:, 1:, :] - v[:, :-1, :] + w[1:, :, :] - w[:-1, :, :]) / cfg.cell_size
    fluid = occ == 0
    scale = max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max()) / cfg.cell_size
    d = d[fluid] / scale
    return float(np.sqrt(np.mean(d * d))), float(np.abs(d).max())


@pytest.mark.parametrize("name", list(SIZES))
def test_one_step_from_identical_state_at_benchmark_size(smoke_lib, cuda_stream, name):
    n, mode, spin = SIZES[name]
    cfg = plume_scene.plume_config(n, mode=mode)
    sim = smoke_b200.Simulation(smoke_lib, cfg, cuda_stream)
    sim.set_solver(abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, max_iterations=200, tolerance=1e-5, refinement=1, warm_start=True)
    driver = plume_scene.PlumeDriver(sim, n, seed=1)
    for k in range(spin):
        driver.apply(k)
        with torch.cuda.stream(cuda_stream):
            sim.step()
    driver.apply(spin)  # the parity step's sources and forces
    with torch.cuda.stream(cuda_stream):
        state = {"density": sim.view(abi.VIEW_DENSITY).clone(), "temperature": sim.view(abi.VIEW_TEMPERATURE).clone(), "force_y": driver.force_y.clone(),
                 "density_source": driver.density_source.clone(), "temperature_source": driver.temperature_source.clone()}
    cuda_stream.synchronize()
    state = {k: t.cpu().numpy() for k, t in state.items()}
    u0, v0, w0 = face_arrays(sim)
    sim.set_solver(abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, max_iterations=400, tolerance=1e-9, refinement=6, warm_start=False)
    with torch.cuda.stream(cuda_stream):
        sim.step()
    status = sim.solver_status()
    gu, gv, gw = face_arrays(sim)
    snap = sim.snapshot([abi.VIEW_DENSITY, abi.VIEW_TEMPERATURE, abi.VIEW_FLOW_PRESSURE])
    sim.close()

    st = O.OracleState(cfg, 64)
    for k, val in (("u", u0), ("v", v0), ("w", w0), ("density", state["density"]), ("temperature", state["temperature"]), ("force_y", state["force_y"]),
                   ("density_source", state["density_source"]), ("temperature_source", state["temperature_source"])):
        st.set(k, val)
    solved = st.step(0, 5, mode=1, max_iterations=8000, tolerance=1e-10)
    occ = np.zeros(abi.cell_shape(cfg), np.uint8)
    errs = {"u": scenes.rel_err(gu, st["u"]), "v": scenes.rel_err(gv, st["v"]), "w": scenes.rel_err(gw, st["w"]), "density": scenes.rel_err(snap["density"], st["density"]),
            "temperature": scenes.rel_err(snap["temperature"], st["temperature"]), "pressure": scenes.rel_err(snap["pressure"], st["pressure"])}
    div_gpu = divergence_norms(cfg, gu, gv, gw, occ)
    div_oracle = divergence_norms(cfg, st["u"], st["v"], st["w"], occ)
    report(f"full_size/{name}", {"err_vs_fp64": errs, "divergence_l2_linf_gpu": div_gpu, "divergence_l2_linf_fp64": div_oracle, "gpu_iterations": status.iterations,
                                 "gpu_true_residual": status.true_relative_residual, "oracle_iterations": solved.iterations, "oracle_residual": solved.relative_residual})
    assert status.status == abi.SOLVE_CONVERGED and status.true_relative_residual <= 1e-9
    assert solved.relative_residual <= 1e-10
    for k, e in errs.items():
        assert e <= BAR, (k, e, errs)
    assert div_gpu[1] <= 1e-5, div_gpu


def test_deep_solid_density_fill(smoke_lib, cuda_stream):
    """A sphere of radius 9 cells in a 32^3 closed box with random density, temperature and velocity: one full step
    (monotone cubic) against the FP32 and FP64 oracles. Solid cells up to 9 cells deep take the density of their
    nearest fluid cells (backend-cuda.cu:1243-1290); the fill map (built once per occupancy) must reproduce it."""
    cfg = scenes.make_config(32, 32, 32, boundary="closed", mode=abi.MONOTONIC_CUBIC)
    inp = scenes.random_inputs(cfg, seed=21, solids=False)
    inp["occupancy"] = plume_scene.sphere_occupancy((32, 32, 32), (16.0, 16.0, 16.0), 9.0)
    occ = inp["occupancy"] != 0
    sim = smoke_b200.Simulation(smoke_lib, cfg, cuda_stream)
    keep = scenes.load_gpu(sim, inp)
    sim.set_solver(abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, max_iterations=400, tolerance=1e-9, refinement=6)
    with torch.cuda.stream(cuda_stream):
        sim.step()
    snap = sim.snapshot([abi.VIEW_DENSITY, abi.VIEW_TEMPERATURE])
    sim.close()
    del keep
    out = {}
    for bits in (32, 64):
        st = O.OracleState(cfg, bits)
        scenes.load_oracle(st, inp)
        st.step(0, 5, mode=1, max_iterations=8000, tolerance=1e-10 if bits == 64 else 1e-7)
        out[bits] = st
    depth = int(occ.sum())
    e_solid = scenes.rel_err(np.where(occ, snap["density"], 0), np.where(occ, out[64]["density"], 0))
    e_density, flips = scenes.rel_err_either(snap["density"], out[32]["density"], out[64]["density"], BAR)
    e_temp = scenes.rel_err(snap["temperature"], out[64]["temperature"])
    report("full_size/deep_solid32", {"solid_cells": depth, "density_in_solid": e_solid, "density": e_density, "cells_matching_only_fp64": flips, "temperature": e_temp})
    assert depth > 2500  # 4/3 pi 9^3 ~ 3054 cells
    assert e_solid <= BAR and e_density <= BAR and e_temp <= BAR, (e_solid, e_density, e_temp)
    assert flips <= 32, flips


# ---------------------------------------------------------------------------------------------- reference library
def oracle_plume_inputs(st, box, xi, dt):
    """The plume driver's per-step inputs computed from the oracle's own state (plume_scene.SceneDriver.apply)."""
    zs, ys, xs = box
    for name in ("force_y", "density_source", "temperature_source"):
        st[name][...] = 0.0
    st["force_y"][zs, ys, xs] = (1.0 + xi - st["centered_y"][zs, ys, xs]) / dt
    st["density_source"][zs, ys, xs] = (1.0 - st["density"][zs, ys, xs]) / dt
    st["temperature_source"][zs, ys, xs] = (1.0 - st["temperature"][zs, ys, xs]) / dt


REFERENCE_SIZES = {"plume64_linear": (64, abi.LINEAR, 500, 3), "plume128_cubic": (128, abi.MONOTONIC_CUBIC, 900, 2)}


@pytest.mark.parametrize("name", list(REFERENCE_SIZES))
def test_reference_library_at_benchmark_size(smoke_lib, cuda_stream, name):
    n, mode, ref_iterations, steps = REFERENCE_SIZES[name]
    if not os.path.exists(REF_LIBRARY):
        pytest.fail(f"reference library missing: {REF_LIBRARY} (oracle/build_oracle.py builds it)")
    ref_lib = smoke_b200.SmokeLibrary(REF_LIBRARY, extensions=False)
    cfg = plume_scene.plume_config(n, mode=mode, pressure_iterations=ref_iterations)
    s_ref = torch.cuda.Stream()
    ref = smoke_b200.Simulation(ref_lib, cfg, s_ref)
    mine = smoke_b200.Simulation(smoke_lib, cfg, cuda_stream)
    mine.set_solver(abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, max_iterations=200, tolerance=1e-7, refinement=3)
    d_ref = plume_scene.PlumeDriver(ref, n, seed=1)
    d_mine = plume_scene.PlumeDriver(mine, n, seed=1)
    st = O.OracleState(cfg, 64)
    box = plume_scene.source_box(n)
    size = tuple(s.stop - s.start for s in box)
    fields = {"density": ("density", abi.VIEW_DENSITY), "temperature": ("temperature", abi.VIEW_TEMPERATURE), "pressure": ("pressure", abi.VIEW_FLOW_PRESSURE)}
    worst = {"reference": {}, "b200": {}, "b200_vs_reference": {}}
    for k in range(steps):
        xi = d_ref.inputs_for(k).numpy().copy()
        d_ref.apply(k, d_ref.inputs_for(k))
        d_mine.apply(k, d_mine.inputs_for(k))
        oracle_plume_inputs(st, box, xi.reshape(size).astype(np.float64), cfg.dt)
        with torch.cuda.stream(s_ref):
            ref.step()
        with torch.cuda.stream(cuda_stream):
            mine.step()
        st.step(0, 5, mode=1, max_iterations=8000, tolerance=1e-10)
        a = ref.snapshot([abi.VIEW_DENSITY, abi.VIEW_TEMPERATURE, abi.VIEW_FLOW_PRESSURE, abi.VIEW_FLOW_VELOCITY])
        b = mine.snapshot([abi.VIEW_DENSITY, abi.VIEW_TEMPERATURE, abi.VIEW_FLOW_PRESSURE, abi.VIEW_FLOW_VELOCITY])
        pairs = dict(fields)
        for ax in "xyz":
            pairs[f"velocity_{ax}"] = (f"centered_{ax}", None)
        for key, (okey, _) in pairs.items():
            for who, snap in (("reference", a), ("b200", b)):
                worst[who][key] = max(worst[who].get(key, 0.0), scenes.rel_err(snap[key], st[okey]))
            worst["b200_vs_reference"][key] = max(worst["b200_vs_reference"].get(key, 0.0), scenes.rel_err(b[key], a[key]))
    ref.close()
    mine.close()
    report(f"reference_full_size/{name}", worst)
    for key, e in worst["b200"].items():
        floor = max(BAR, worst["reference"][key])
        assert e <= floor, (key, e, floor, worst)
