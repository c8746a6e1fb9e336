"""Warm starts (smoke_b200_set_solver_cuda with warm_start = 1): each step's solve starts from the previous step's
FP64 pressure instead of 0 and stops on the same test, ||b - A x|| <= tol ||b||, so the answer meets the tolerance
of a cold start, in fewer iterations once the flow has developed."""
import numpy as np
import pytest
import torch

import plume_scene
import smoke_abi as abi
import smoke_b200

pytestmark = pytest.mark.gpu

STEPS = 12


def run(lib, stream, mode, warm, n=32):
    cfg = plume_scene.plume_config(n, abi.MONOTONIC_CUBIC)
    sim = smoke_b200.Simulation(lib, cfg, stream)
    driver = plume_scene.PlumeDriver(sim, n, seed=3)
    sim.set_solver(mode, abi.REDUCTION_FP64, max_iterations=3000, tolerance=1e-5, refinement=3, warm_start=warm)
    its, res = [], []
    for k in range(STEPS):
        driver.apply(k)
        sim.step()
        stream.synchronize()
        st = sim.solver_status()
        assert st.status == abi.SOLVE_CONVERGED, (k, st.status)
        its.append(st.iterations)
        res.append(st.true_relative_residual)
    with torch.cuda.stream(stream):
        d = sim.view(abi.VIEW_DENSITY).clone()
    stream.synchronize()
    sim.close()
    return its, res, d.double().cpu().numpy()


@pytest.mark.parametrize("mode", [abi.SOLVER_MG_FCG, abi.SOLVER_JACOBI_PCG], ids=["multigrid", "jacobi"])
def test_warm_start_meets_the_tolerance_in_fewer_iterations(smoke_lib, cuda_stream, mode):
    its_c, res_c, d_c = run(smoke_lib, cuda_stream, mode, False)
    its_w, res_w, d_w = run(smoke_lib, cuda_stream, mode, True)
    assert max(res_w) <= 1e-5 and max(res_c) <= 1e-5, (res_w, res_c)
    assert sum(its_w[2:]) < sum(its_c[2:]), (its_w, its_c)
    # both runs solve every step to 1e-5, so the flows stay close
    assert np.abs(d_w - d_c).max() <= 1e-3 * max(np.abs(d_c).max(), 1e-30)


def test_warm_start_after_an_occupancy_change_keeps_solid_pressure_zero(smoke_lib, cuda_stream):
    n = 32
    cfg = plume_scene.plume_config(n, abi.MONOTONIC_CUBIC)
    sim = smoke_b200.Simulation(smoke_lib, cfg, cuda_stream)
    driver = plume_scene.PlumeDriver(sim, n, seed=5)
    sim.set_solver(abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, max_iterations=500, tolerance=1e-5, refinement=3, warm_start=True)
    for k in range(6):
        driver.apply(k)
        sim.step()
    occ = plume_scene.sphere_occupancy((n, n, n), (n / 2, n / 2, n / 2), n / 6)
    with torch.cuda.stream(cuda_stream):
        o = torch.from_numpy(occ).cuda()
        sim.update_occupancy(o)
    for k in range(6, 9):
        driver.apply(k)
        sim.step()
        cuda_stream.synchronize()
        st = sim.solver_status()
        assert st.status == abi.SOLVE_CONVERGED and st.true_relative_residual <= 1e-5, (k, st.status, st.true_relative_residual)
    with torch.cuda.stream(cuda_stream):
        p = sim.view(abi.VIEW_FLOW_PRESSURE).clone()
    cuda_stream.synchronize()
    sim.close()
    p = p.cpu().numpy()
    assert np.all(p[occ != 0] == 0.0)  # cells that were fluid before the change hold no stale pressure
    assert np.abs(p[occ == 0]).max() > 0.0
