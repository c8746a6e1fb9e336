"""Batched stepping (smoke_b200_batch_*_cuda): one graph launch advancing several scenes of different sizes and
boundary mixes gives each scene the state that stepping it alone gives (within the reduction-order rounding of the
solver's dot products), and the members stay usable through the single-context ABI afterwards."""
import numpy as np
import pytest
import torch

import scenes
import smoke_abi as abi
import smoke_b200

pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(shape=(16, 12, 8), boundary="plume", mode=abi.MONOTONIC_CUBIC, seed=5),
    dict(shape=(9, 11, 7), boundary="mixed", mode=abi.LINEAR, seed=6),
    dict(shape=(24, 16, 20), boundary="closed", mode=abi.MONOTONIC_CUBIC, seed=7),
]
KINDS = [abi.VIEW_DENSITY, abi.VIEW_TEMPERATURE, abi.VIEW_FLOW_VELOCITY, abi.VIEW_FLOW_PRESSURE]
TOL = 1e-5


def make(lib, stream, m, solver):
    cfg = scenes.make_config(*m["shape"], boundary=m["boundary"], mode=m["mode"])
    inp = scenes.random_inputs(cfg, seed=m["seed"], solids=True, cfl=0.8)
    sim = smoke_b200.Simulation(lib, cfg, stream)
    keep = scenes.load_gpu(sim, inp)
    sim.set_solver(*solver)
    return sim, keep


@pytest.mark.parametrize("solver", [(abi.SOLVER_MG_FCG, abi.REDUCTION_FP64, 500, 1e-7, 2), (abi.SOLVER_FIXED_CG, abi.REDUCTION_FP32, 500, 1e-5, 0)], ids=["multigrid", "fixed_cg"])
def test_batch_equals_individual_steps(smoke_lib, cuda_stream, solver):
    alone = [make(smoke_lib, torch.cuda.Stream(), m, solver) for m in MEMBERS]
    batched = [make(smoke_lib, torch.cuda.Stream(), m, solver) for m in MEMBERS]
    for sim, _ in alone:
        for _ in range(3):
            sim.step()
    with smoke_b200.Batch([s for s, _ in batched]) as batch:
        for _ in range(3):
            batch.step()
        times = batch.member_times()  # each member's completion time inside the last batch step
        assert times.shape == (len(MEMBERS),) and np.all(times > 0) and np.all(np.isfinite(times))
        for (a, _), (b, _) in zip(alone, batched):
            ra, rb = a.snapshot(KINDS), b.snapshot(KINDS)
            for key in ra:
                assert scenes.rel_err(rb[key], ra[key]) < TOL, key
            assert b.solver_status().status == a.solver_status().status
    # after the batch is gone the members step alone again
    for (a, _), (b, _) in zip(alone, batched):
        a.step()
        b.step()
        ra, rb = a.snapshot([abi.VIEW_DENSITY]), b.snapshot([abi.VIEW_DENSITY])
        assert scenes.rel_err(rb["density"], ra["density"]) < TOL
    for s, _ in alone + batched:
        s.close()


def test_batch_rejects_duplicates_and_empty(smoke_lib, cuda_stream):
    import ctypes as C

    sim, keep = make(smoke_lib, cuda_stream, MEMBERS[0], (abi.SOLVER_FIXED_CG, abi.REDUCTION_FP32, 500, 1e-5, 0))
    out = C.c_void_p()
    twice = (C.c_void_p * 2)(sim.handle.value, sim.handle.value)
    assert smoke_lib.lib.smoke_b200_batch_create_cuda(twice, 2, None, C.byref(out)) == abi.RESULT_BACKEND_FAILURE
    assert smoke_lib.lib.smoke_b200_batch_create_cuda(twice, 0, None, C.byref(out)) == abi.RESULT_BACKEND_FAILURE
    assert smoke_lib.lib.smoke_b200_batch_destroy_cuda(None) == abi.RESULT_OK
    sim.close()
