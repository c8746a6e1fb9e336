"""The pressure solve that allocates nothing (smoke_b200_solve_pressure_noalloc_cuda), called through the C ABI.

It exists for callers that cannot call cudaMalloc while they run -- an engine that reserves its GPU memory up
front and forbids allocations in its frame loop, or a plug-in inside another application's memory budget -- and
keeps its scratch in one device array inside the library. These tests check that it returns the pressure of the
context's own solve (smoke_b200_solve_pressure_cuda) for the same right-hand side on two calls in a row, that the
second call leaves the device's free memory unchanged, and that grids above its limit are refused with a reason.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import scenes
import smoke_abi as abi
import smoke_b200

pytestmark = pytest.mark.gpu


def _bind(raw):
    fn = raw.smoke_b200_solve_pressure_noalloc_cuda
    fn.argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(abi.SolverDesc), C.c_void_p, C.POINTER(abi.SolverStatus)]
    fn.restype = C.c_int
    raw.smoke_b200_last_error.restype = C.c_char_p
    raw.smoke_b200_noalloc_max_cells.restype = C.c_ulonglong
    return fn


SOLVERS = {
    "fixed_cg": abi.SolverDesc(abi.SOLVER_FIXED_CG, abi.REDUCTION_FP32, 500, 1e-5, 0, 0),
    "jacobi_fp64_refined": abi.SolverDesc(abi.SOLVER_JACOBI_PCG, abi.REDUCTION_FP64, 3000, 1e-6, 3, 0),
}


@pytest.mark.parametrize("solids", [True, False])
@pytest.mark.parametrize("solver", list(SOLVERS))
def test_no_alloc_solve_matches_context_solve(solver, solids):
    lib = smoke_b200.SmokeLibrary()
    solve = _bind(lib.lib)
    stream = torch.cuda.Stream()
    cfg = scenes.make_config(24, 20, 16, boundary="mixed", mode=abi.LINEAR, pressure_iterations=60)
    inp = scenes.random_inputs(cfg, seed=9, solids=solids)
    desc = SOLVERS[solver]
    sim = smoke_b200.Simulation(lib, cfg, stream)
    keep = scenes.load_gpu(sim, inp)
    sim.set_solver(desc.mode, desc.reduction, desc.max_iterations, desc.tolerance, desc.refinement)
    with torch.cuda.stream(stream):
        sim.step_stages(abi.STAGE_PRESSURE)  # right-hand side of the advected velocity
        sim.solve_pressure()                 # the context's standalone solve of that right-hand side
        rhs = sim.view(abi.VIEW_FLOW_PRESSURE_RHS).clone()
        expected = sim.view(abi.VIEW_FLOW_PRESSURE).clone()
    ref_status = sim.solver_status()
    occ = torch.from_numpy(inp["occupancy"]).cuda() if solids else None
    torch.cuda.synchronize()
    results = []
    for call in range(2):
        out = torch.full_like(rhs, float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = abi.SolverStatus()
        rc = solve(C.byref(cfg), C.c_void_p(occ.data_ptr()) if occ is not None else None, C.c_void_p(rhs.data_ptr()), C.c_void_p(out.data_ptr()), C.byref(desc),
                   C.c_void_p(stream.cuda_stream), C.byref(st))
        assert rc == abi.RESULT_OK, lib.lib.smoke_b200_last_error()
        stream.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            assert free_after == free_before, (free_before, free_after)
        assert st.iterations == ref_status.iterations and st.status == ref_status.status, (st.iterations, ref_status.iterations, st.status, ref_status.status)
        results.append(out.cpu().numpy())
    sim.close()
    del keep
    e = expected.cpu().numpy()
    for r in results:
        assert np.isfinite(r).all()
        assert scenes.rel_err(r, e) <= 1e-6, scenes.rel_err(r, e)


def test_no_alloc_refuses_grids_above_its_limit():
    lib = smoke_b200.SmokeLibrary()
    solve = _bind(lib.lib)
    limit = lib.lib.smoke_b200_noalloc_max_cells()
    assert limit == 64 ** 3
    cfg = scenes.make_config(65, 64, 64)
    dummy = torch.zeros(4, device="cuda")
    rc = solve(C.byref(cfg), None, C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), None, None, None)
    assert rc == abi.RESULT_BACKEND_FAILURE
    assert b"exceeds the no-allocation limit" in lib.lib.smoke_b200_last_error()
