"""The device-side waits give up instead of hanging, and the context stays usable afterwards.

The persistent CG kernel's grid barrier waits a bounded time for every block (globaltimer, plus a poll cap). The
test hook smoke_b200_test_barrier_timeout_cuda tells one block of the cooperative grid to leave before its first
barrier, so nothing ever completes that barrier: the other blocks' waits must run out after the given limit, abort
the solve and report SMOKE_B200_SOLVE_BARRIER_TIMEOUT, with no trap and no fault. A normal solve on the same
context then converges as before.

The tensor-core convolution's waits (TMA arrival, MMA completion, accumulator drain) are bounded in clock cycles. The
test hook smoke_b200_test_conv_wait_timeout_cuda expects every TMA load but issues none, so each block's first wait
runs out: the block raises the error word, frees its tensor memory and leaves; the convolution then runs normally.

(The reference has no device-side waits: its CG is a graph of library calls whose errors map to BACKEND_FAILURE,
backend-cuda.cu:1611-1614, 2063-2071.)
"""
import ctypes as C
import time

import numpy as np
import pytest
import torch

import scenes
import smoke_abi as abi
import smoke_b200

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [abi.SOLVER_FIXED_CG, abi.SOLVER_JACOBI_PCG], ids=["fixed_cg", "jacobi"])
def test_grid_barrier_wait_runs_out_and_the_context_recovers(smoke_lib, cuda_stream, mode):
    cfg = scenes.make_config(48, 40, 32, boundary="mixed", mode=abi.LINEAR, pressure_iterations=80)
    inp = scenes.random_inputs(cfg, seed=4, solids=True)
    sim = smoke_b200.Simulation(smoke_lib, cfg, cuda_stream)
    keep = scenes.load_gpu(sim, inp)
    sim.set_solver(mode, abi.REDUCTION_FP64, max_iterations=3000, tolerance=1e-6, refinement=2)
    with torch.cuda.stream(cuda_stream):
        sim.step_stages(abi.STAGE_PRESSURE)
    good = sim.solver_status()
    with torch.cuda.stream(cuda_stream):
        p_good = sim.view(abi.VIEW_FLOW_PRESSURE).clone()
    cuda_stream.synchronize()

    st = abi.SolverStatus()
    t0 = time.perf_counter()
    rc = smoke_lib.lib.smoke_b200_test_barrier_timeout_cuda(sim.handle, 1, 100, C.byref(st))
    waited = time.perf_counter() - t0
    assert rc == abi.RESULT_OK
    assert st.status == abi.SOLVE_BARRIER_TIMEOUT, st.status
    assert 0.05 < waited < 5.0, waited  # the 100 ms limit ran out once; nothing waited for the 2 s default

    # the context still works: the same solve again, to the same answer
    with torch.cuda.stream(cuda_stream):
        sim.solve_pressure()
    again = sim.solver_status()
    with torch.cuda.stream(cuda_stream):
        p_again = sim.view(abi.VIEW_FLOW_PRESSURE).clone()
    cuda_stream.synchronize()
    assert again.status == good.status and abs(again.iterations - good.iterations) <= 1
    assert scenes.rel_err(p_again.cpu().numpy(), p_good.cpu().numpy()) < 1e-6
    sim.close()
    del keep


def test_barrier_hook_refuses_what_it_cannot_run(smoke_lib, cuda_stream):
    cfg = scenes.make_config(16, 16, 16)
    sim = smoke_b200.Simulation(smoke_lib, cfg, cuda_stream)
    st = abi.SolverStatus()
    fn = smoke_lib.lib.smoke_b200_test_barrier_timeout_cuda
    assert fn(sim.handle, 0, 100, C.byref(st)) == abi.RESULT_BACKEND_FAILURE     # block 0 writes the status
    assert fn(sim.handle, 1, 0, C.byref(st)) == abi.RESULT_BACKEND_FAILURE       # no limit
    sim.set_solver(abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, max_iterations=100, tolerance=1e-5, refinement=1)
    assert fn(sim.handle, 1, 100, C.byref(st)) == abi.RESULT_BACKEND_FAILURE     # the multigrid graph has no barrier
    sim.close()


def test_tensor_core_wait_runs_out_and_the_convolution_recovers(smoke_lib):
    fn = smoke_lib.lib.smoke_b200_test_conv_wait_timeout_cuda
    fn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(C.c_uint), C.c_void_p]
    fn.restype = C.c_int
    err = C.c_uint(0)
    t0 = time.perf_counter()
    rc = fn(40, 32, 6, 20_000_000, C.byref(err), None)  # 2e7 cycles: about 10 ms per wait
    waited = time.perf_counter() - t0
    assert rc == abi.RESULT_OK
    assert err.value & 1, err.value
    assert waited < 5.0, waited
    # a normal convolution afterwards, checked against float64
    rng = np.random.default_rng(1)
    nz, ny, nx = 6, 32, 40
    x = rng.standard_normal((nz, ny, nx, 16)).astype(np.float32)
    w = (rng.standard_normal((27, 16, 16)) / 20.0).astype(np.float32)
    xb = torch.from_numpy(x).to(torch.bfloat16)
    wb = torch.from_numpy(w).to(torch.bfloat16).float().numpy().astype(np.float64)
    x_dev, w_dev = xb.cuda().contiguous(), torch.from_numpy(w).cuda()
    out0 = torch.zeros((nz, ny, nx), dtype=torch.float32, device="cuda")
    conv = smoke_lib.lib.smoke_b200_conv3d_cuda
    rc = conv(nx, ny, nz, 16, 16, C.c_void_p(x_dev.data_ptr()), C.c_void_p(w_dev.data_ptr()), None, 0, None, C.c_void_p(out0.data_ptr()), None)
    assert rc == abi.RESULT_OK
    xp = np.zeros((nz + 2, ny + 2, nx + 2, 16))
    xp[1:-1, 1:-1, 1:-1] = xb.float().numpy()
    ref = np.zeros((nz, ny, nx))
    for tap in range(27):
        dx, dy, dz = tap % 3 - 1, (tap // 3) % 3 - 1, tap // 9 - 1
        ref += xp[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx] @ wb[tap][:, 0]
    assert np.abs(out0.cpu().numpy() - ref).max() <= 2e-6 * np.abs(ref).max()
