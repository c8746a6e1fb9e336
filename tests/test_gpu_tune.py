"""Launch shapes and the autotuner (smoke_b200_set_launch_tune_cuda, smoke_b200_autotune_cuda).

Every advection shape computes each face and cell with the same arithmetic, so the advected velocity is bit for
bit the flat launch's; the multigrid solver grids change how the FP64 dot products are split over blocks, so a
converged solve lands on the same answer within the solve's tolerance. The autotuner must leave the simulation state as it found it."""
import numpy as np
import pytest
import torch

import scenes
import smoke_abi as abi
import smoke_b200

pytestmark = pytest.mark.gpu

SHAPES = [
    dict(shape=(37, 29, 21), boundary="closed", mode=abi.MONOTONIC_CUBIC, seed=11),
    dict(shape=(24, 40, 18), boundary="mixed", mode=abi.LINEAR, seed=12),
]
KINDS = [abi.VIEW_DENSITY, abi.VIEW_TEMPERATURE, abi.VIEW_FLOW_VELOCITY, abi.VIEW_FLOW_PRESSURE]
MG = (abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, 500, 1e-7, 2)
JACOBI = (abi.SOLVER_JACOBI_PCG, abi.REDUCTION_FP64, 6000, 1e-8, 3)


def make(lib, m, solver=MG):
    cfg = scenes.make_config(*m["shape"], boundary=m["boundary"], mode=m["mode"])
    inp = scenes.random_inputs(cfg, seed=m["seed"], solids=True, cfl=0.8)
    sim = smoke_b200.Simulation(lib, cfg, torch.cuda.Stream())
    keep = scenes.load_gpu(sim, inp)
    sim.set_solver(*solver)
    return sim, keep


@pytest.mark.parametrize("m", SHAPES, ids=["closed_cubic", "mixed_linear"])
def test_advection_shapes_are_bit_exact(smoke_lib, m):
    flat, keep = make(smoke_lib, m)
    flat.step_stages(abi.STAGE_ADVECT_VELOCITY)
    want = flat.face_velocity_host(1)
    for tile in range(1, len(abi.ADVECT_TILE_NAMES)):
        sim, keep2 = make(smoke_lib, m)
        sim.set_launch_tune(advect_tile=tile)
        assert sim.launch_tune()["advect_tile"] == tile
        sim.step_stages(abi.STAGE_ADVECT_VELOCITY)
        got = sim.face_velocity_host(1)
        for a, b in zip(got, want):
            assert np.array_equal(a, b), abi.ADVECT_TILE_NAMES[tile]
        sim.close()
    flat.close()


@pytest.mark.parametrize("m", SHAPES, ids=["closed_cubic", "mixed_linear"])
def test_advection_shapes_full_step(smoke_lib, m):
    """Scalar advection runs in the chosen shape too; two steps agree with the flat launch bit for bit (the
    advection is bit-exact in every shape and the multigrid solve's sums run in a fixed order)."""
    flat, keep = make(smoke_lib, m)
    for _ in range(2):
        flat.step()
    want = flat.snapshot(KINDS)
    for tile in (1, 3):
        sim, keep2 = make(smoke_lib, m)
        sim.set_launch_tune(advect_tile=tile)
        for _ in range(2):
            sim.step()
        got = sim.snapshot(KINDS)
        for key in want:
            assert np.array_equal(got[key], want[key]), (tile, key)
        sim.close()
    flat.close()


@pytest.mark.parametrize("m", SHAPES, ids=["closed_cubic", "mixed_linear"])
def test_multigrid_solve_is_deterministic(smoke_lib, m):
    """Two simulations of the same inputs step to bit-identical fields: every dot product of the multigrid FCG is
    summed in a fixed order (per-block partials added in block order), whatever order the blocks finish in."""
    runs = []
    for _ in range(2):
        sim, keep = make(smoke_lib, m)
        statuses = []
        for _ in range(2):
            sim.step()
            st = sim.solver_status()
            statuses.append((st.iterations, st.passes, st.true_relative_residual))
        runs.append((sim.snapshot(KINDS), statuses))
        sim.close()
    assert runs[0][1] == runs[1][1]
    for key in runs[0][0]:
        assert np.array_equal(runs[0][0][key], runs[1][0][key]), key


@pytest.mark.parametrize("solver,field,count", [(MG, "mg_wave", len(abi.MG_WAVE_NAMES)), (JACOBI, "pcg_grid", len(abi.PCG_GRID_NAMES)), (JACOBI, "pcg_regs", len(abi.PCG_REGS_NAMES))],
                         ids=["multigrid", "jacobi_grid", "jacobi_regs"])
def test_solver_grids_reach_the_same_answer(smoke_lib, solver, field, count):
    m = SHAPES[0]
    ref, keep = make(smoke_lib, m, solver)
    ref.step()
    want = ref.snapshot(KINDS)
    assert ref.solver_status().status == abi.SOLVE_CONVERGED
    want_it = ref.solver_status().iterations
    for code in range(count):
        sim, keep2 = make(smoke_lib, m, solver)
        sim.set_launch_tune(**{field: code})
        sim.step()
        st = sim.solver_status()
        assert st.status == abi.SOLVE_CONVERGED, (field, code)
        if field == "mg_wave":  # the multigrid solve's count is stable; the Jacobi solve's refinement restarts are not
            assert abs(st.iterations - want_it) <= 2, (field, code)
        got = sim.snapshot(KINDS)
        for key in want:  # the solves stop at rel-res 1e-7 / 1e-8: their answers differ at that level
            assert scenes.rel_err(got[key], want[key]) < 1e-4, (field, code, key)
        sim.close()
    ref.close()


def test_unknown_codes_are_rejected(smoke_lib):
    sim, keep = make(smoke_lib, SHAPES[1])
    for bad in (dict(advect_tile=len(abi.ADVECT_TILE_NAMES)), dict(mg_wave=len(abi.MG_WAVE_NAMES)), dict(pcg_grid=len(abi.PCG_GRID_NAMES)), dict(pcg_regs=len(abi.PCG_REGS_NAMES))):
        with pytest.raises(smoke_b200.SmokeError):
            sim.set_launch_tune(**bad)
    assert sim.launch_tune() == {"advect_tile": 0, "mg_wave": 1, "pcg_grid": 0, "pcg_regs": 0}
    sim.close()


def test_autotune_restores_state_and_caches(smoke_lib):
    m = dict(shape=(33, 47, 26), boundary="plume", mode=abi.MONOTONIC_CUBIC, seed=13)
    sim, keep = make(smoke_lib, m)
    twin, keep2 = make(smoke_lib, m)
    sim.step()
    twin.step()
    before = sim.snapshot(KINDS)
    rep = sim.autotune(steps=2, force=True)
    after = sim.snapshot(KINDS)
    for key in before:
        assert np.array_equal(after[key], before[key]), key
    assert not rep["from_cache"]
    # the start shapes, every other advection shape, every other multigrid depth
    assert len(rep["records"]) == 1 + (len(abi.ADVECT_TILE_NAMES) - 1) + (len(abi.MG_WAVE_NAMES) - 1)
    assert rep["records"][0]["ms_per_step"] == pytest.approx(rep["default_ms"])
    assert all(r["ms_per_step"] > 0 for r in rep["records"])
    assert rep["chosen"] == sim.launch_tune()
    assert rep["chosen_ms"] <= rep["default_ms"]
    assert any(dict(advect_tile=r["advect_tile"], mg_wave=r["mg_wave"], pcg_grid=r["pcg_grid"], pcg_regs=r["pcg_regs"]) == rep["chosen"] for r in rep["records"])
    # the tuned context keeps stepping like its untuned twin
    sim.step()
    twin.step()
    a, b = sim.snapshot(KINDS), twin.snapshot(KINDS)
    for key in a:
        assert scenes.rel_err(a[key], b[key]) < 1e-5, key
    # a context with the same grid and solver takes the cached shapes without timing
    third, keep3 = make(smoke_lib, m)
    rep3 = third.autotune()
    assert rep3["from_cache"] and rep3["chosen"] == rep["chosen"] and third.launch_tune() == rep["chosen"]
    for s in (sim, twin, third):
        s.close()
