"""The pressure solve that allocates nothing (smoke_b200_solve_pressure_noalloc_cuda), called through the C ABI.

It exists for callers that cannot call cudaMalloc while they run -- an engine that reserves its GPU memory up
front and forbids allocations in its frame loop, or a plug-in inside another application's memory budget -- and
keeps its scratch in one device array inside the library. These tests check that it returns the pressure of the
context's own solve (smoke_b200_solve_pressure_cuda) for the same right-hand side on two calls in a row, that the
second call leaves the device's free memory unchanged, that nothing of one call's problem carries over to the next
through the shared array (a grid with solids, then a larger one without, asynchronously), that the 64^3 limit itself
works, and that grids above its limit are refused with a reason.
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


def _context_solve(lib, cfg, inp, desc, stream):
    """(rhs, pressure, status) of a context's own standalone solve of the step's pressure system."""
    sim = smoke_b200.Simulation(lib, cfg, stream)
    keep = scenes.load_gpu(sim, inp)
    sim.set_solver(desc.mode, desc.reduction, desc.max_iterations, desc.tolerance, desc.refinement)
    with torch.cuda.stream(stream):
        sim.step_stages(abi.STAGE_PRESSURE)  # right-hand side of the advected velocity
        sim.solve_pressure()                 # the context's standalone solve of that right-hand side
        rhs = sim.view(abi.VIEW_FLOW_PRESSURE_RHS).clone()
        expected = sim.view(abi.VIEW_FLOW_PRESSURE).clone()
    status = sim.solver_status()
    stream.synchronize()
    sim.close()
    del keep
    return rhs, expected, status


@pytest.mark.parametrize("solids", [True, False])
@pytest.mark.parametrize("solver", list(SOLVERS))
def test_no_alloc_solve_matches_context_solve(solver, solids):
    lib = smoke_b200.SmokeLibrary()
    solve = _bind(lib.lib)
    stream = torch.cuda.Stream()
    cfg = scenes.make_config(24, 20, 16, boundary="mixed", mode=abi.LINEAR, pressure_iterations=60)
    inp = scenes.random_inputs(cfg, seed=9, solids=solids)
    desc = SOLVERS[solver]
    rhs, expected, ref_status = _context_solve(lib, cfg, inp, desc, stream)
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


def test_no_alloc_calls_share_nothing_but_the_array():
    """A 24x20x16 grid with solids, then a 40x36x32 grid without, both asynchronous (no status, one stream
    synchronisation after the second call): the second result must equal its context solve, so no operator code,
    anchor, control word or FP64 accumulator of the first problem leaks into the second."""
    lib = smoke_b200.SmokeLibrary()
    solve = _bind(lib.lib)
    stream = torch.cuda.Stream()
    desc = SOLVERS["jacobi_fp64_refined"]
    cfg1 = scenes.make_config(24, 20, 16, boundary="mixed", mode=abi.LINEAR, pressure_iterations=60)
    inp1 = scenes.random_inputs(cfg1, seed=5, solids=True)
    cfg2 = scenes.make_config(40, 36, 32, boundary="plume", mode=abi.LINEAR, pressure_iterations=60)
    inp2 = scenes.random_inputs(cfg2, seed=6, solids=False)
    rhs1, _, _ = _context_solve(lib, cfg1, inp1, desc, stream)
    rhs2, expected2, _ = _context_solve(lib, cfg2, inp2, desc, stream)
    occ1 = torch.from_numpy(inp1["occupancy"]).cuda()
    out1 = torch.full_like(rhs1, float("nan"))
    out2 = torch.full_like(rhs2, float("nan"))
    torch.cuda.synchronize()
    rc = solve(C.byref(cfg1), C.c_void_p(occ1.data_ptr()), C.c_void_p(rhs1.data_ptr()), C.c_void_p(out1.data_ptr()), C.byref(desc), C.c_void_p(stream.cuda_stream), None)
    assert rc == abi.RESULT_OK, lib.lib.smoke_b200_last_error()
    rc = solve(C.byref(cfg2), None, C.c_void_p(rhs2.data_ptr()), C.c_void_p(out2.data_ptr()), C.byref(desc), C.c_void_p(stream.cuda_stream), None)
    assert rc == abi.RESULT_OK, lib.lib.smoke_b200_last_error()
    stream.synchronize()
    r2 = out2.cpu().numpy()
    assert np.isfinite(r2).all() and np.isfinite(out1.cpu().numpy()).all()
    assert scenes.rel_err(r2, expected2.cpu().numpy()) <= 1e-6, scenes.rel_err(r2, expected2.cpu().numpy())


def test_no_alloc_at_its_limit():
    """Exactly 64^3 cells, the largest offsets of the scratch layout, with solids."""
    lib = smoke_b200.SmokeLibrary()
    solve = _bind(lib.lib)
    stream = torch.cuda.Stream()
    desc = SOLVERS["jacobi_fp64_refined"]
    cfg = scenes.make_config(64, 64, 64, boundary="closed", mode=abi.LINEAR, pressure_iterations=60)
    inp = scenes.random_inputs(cfg, seed=11, solids=True)
    rhs, expected, ref_status = _context_solve(lib, cfg, inp, desc, stream)
    occ = torch.from_numpy(inp["occupancy"]).cuda()
    for _ in range(2):
        out = torch.full_like(rhs, float("nan"))
        st = abi.SolverStatus()
        rc = solve(C.byref(cfg), C.c_void_p(occ.data_ptr()), C.c_void_p(rhs.data_ptr()), C.c_void_p(out.data_ptr()), C.byref(desc), C.c_void_p(stream.cuda_stream), C.byref(st))
        assert rc == abi.RESULT_OK, lib.lib.smoke_b200_last_error()
        assert st.status == ref_status.status == abi.SOLVE_CONVERGED
        r = out.cpu().numpy()
        assert np.isfinite(r).all()
        assert scenes.rel_err(r, expected.cpu().numpy()) <= 1e-6
