"""The learned preconditioner on the GPU: the tensor-core network against its float64 oracle (forward and gradient,
with the oracle rounding to BF16 where the GPU stores BF16), training, and the learned FCG solve (z = V(r) +
N(r - A V(r)): the network corrects what the multigrid V-cycle leaves), which must reach the same tolerance and the
same answer as the plain solvers (the network changes the iteration count, not the answer), compared with the same
FCG without the network (multigrid alone), with Jacobi-preconditioned CG, and with the untrained network."""
import json
import os

import numpy as np
import pytest
import torch

import smoke_abi as abi
import smoke_b200
import train_preconditioner as T
import unet_oracle as U

pytestmark = pytest.mark.gpu

OFFSETS = np.cumsum([0] + [27 * ci * co + co for ci, co, _ in U.LAYERS])
SHAPE = (48, 64, 48)  # nx, ny, nz of the solve tests
REPORT = os.environ.get("SMOKE_PARITY_REPORT")


def report(name, value):
    if REPORT:
        with open(REPORT, "a") as f:
            f.write(json.dumps({"check": name, "value": value}) + "\n")


def sample(shape_zyx, seed):
    rng = np.random.default_rng(seed)
    r = rng.standard_normal(shape_zyx).astype(np.float32)
    occ = (rng.random(shape_zyx) < 0.15).astype(np.uint8)
    t = rng.standard_normal(shape_zyx).astype(np.float32)
    return r, occ, t


@pytest.fixture(scope="module")
def net(smoke_lib):
    n = smoke_b200.Net(smoke_lib, seed=3)
    yield n
    n.close()


@pytest.mark.parametrize("shape", [(9, 11, 13), (16, 5, 33), (1, 7, 4)])
def test_apply_matches_oracle(net, shape):
    r, occ, _ = sample(shape, 1)
    p = U.initial_like(2)
    net.set_parameters(p)
    got = net.apply(torch.from_numpy(r).cuda(), torch.from_numpy(occ).cuda()).cpu().numpy()
    want = U.apply(p, r, occ, emulate=True)
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()
    assert not got[occ != 0].any()


@pytest.mark.parametrize("shape", [(9, 11, 13), (6, 17, 10)])
def test_gradient_matches_oracle(net, shape):
    """The backward-data and weight-gradient tensor-core kernels, layer by layer."""
    r, occ, t = sample(shape, 4)
    p = U.initial_like(5)
    net.set_parameters(p)
    loss, g = net.gradient(*(torch.from_numpy(a).cuda() for a in (r, occ, t)))
    want_loss, want = U.loss_and_gradient(p, r, occ, t, emulate=True)
    assert abs(loss - want_loss) <= 1e-5 * want_loss
    for L in range(len(U.LAYERS)):
        a, b = g[OFFSETS[L]:OFFSETS[L + 1]], want[OFFSETS[L]:OFFSETS[L + 1]]
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b), L


def test_parameters_round_trip(smoke_lib):
    with smoke_b200.Net(smoke_lib, seed=11) as a, smoke_b200.Net(smoke_lib, seed=11) as b, smoke_b200.Net(smoke_lib, seed=12) as c:
        pa, pb, pc = a.parameters(), b.parameters(), c.parameters()
        assert pa.size == U.param_count() and np.array_equal(pa, pb) and not np.array_equal(pa, pc)
        c.set_parameters(pa)
        assert np.array_equal(c.parameters(), pa)


@pytest.fixture(scope="module")
def trained(smoke_lib):
    """A network trained briefly on the V-cycle's leftover errors of plume systems of the solve tests' grid, and
    the losses."""
    data = T.generate(smoke_lib, SHAPE, 6, 3, seed=0, synthetic=6)
    n = smoke_b200.Net(smoke_lib, seed=0)
    losses = T.train(n, data, 800, 8, 1e-3, seed=0)
    yield n, losses
    n.close()


def test_training_reduces_the_loss(trained):
    """800 Adam steps on the V-cycle's leftover errors of six 48x64x48 scenes take the relative loss from about 1.0
    to about 0.7 (measured 0.69-0.71 of the first steps' mean); a quarter off is the property checked."""
    _, losses = trained
    assert np.mean(losses[-50:]) < 0.75 * np.mean(losses[:5])


def held_out_system(lib):
    cfg, occ, boxes, strength = T.scene(SHAPE, 999)
    s = torch.cuda.Stream()
    sim = smoke_b200.Simulation(lib, cfg, s)
    with torch.cuda.stream(s):
        o = torch.from_numpy(occ).cuda()
        sim.update_occupancy(o)
    sim.set_solver(**T.STEP_SOLVER)
    drv = __import__("plume_scene").SceneDriver(sim, boxes, seed=5, strength=strength)
    for k in range(12):
        drv.apply(k)
        sim.step()
    return sim, o


def solve(sim, form, net=None):
    if net is not None:
        sim.set_preconditioner_net(net)
    sim.set_solver(**form)
    sim.solve_pressure()
    st = sim.solver_status()
    return st, sim.snapshot([abi.VIEW_FLOW_PRESSURE])["pressure"]


LEARNED = dict(mode=abi.SOLVER_LEARNED_FCG, reduction=abi.REDUCTION_FP64, max_iterations=300, tolerance=1e-5, refinement=3)
MULTIGRID = dict(LEARNED, mode=abi.SOLVER_MG_FCG)
JACOBI = dict(mode=abi.SOLVER_JACOBI_PCG, reduction=abi.REDUCTION_FP64, max_iterations=4000, tolerance=1e-5, refinement=3)


def test_learned_solve_same_answer_and_gain(smoke_lib, trained):
    """The trained learned FCG against the same FCG without the network (multigrid alone), Jacobi-PCG and the
    untrained network: all reach the tolerance with the same answer (within its reach); the trained network needs no
    more iterations than the multigrid alone, nor than with the untrained network, and an order of magnitude fewer
    than Jacobi-PCG."""
    net, _ = trained
    sim, keep = held_out_system(smoke_lib)
    st_j, p_j = solve(sim, JACOBI)
    st_m, p_m = solve(sim, MULTIGRID)
    st_t, p_t = solve(sim, LEARNED, net)
    with smoke_b200.Net(smoke_lib, seed=0) as untrained:
        st_u, p_u = solve(sim, LEARNED, untrained)
    # the network's estimate as the initial guess as well
    st_w, p_w = solve(sim, dict(LEARNED, warm_start=2), net)
    sim.close()
    report("learned/held_out", {"jacobi": st_j.iterations, "multigrid": st_m.iterations, "learned_trained": st_t.iterations, "learned_untrained": st_u.iterations,
                                "learned_trained_net_warm_start": st_w.iterations, "dropped_trained": int(st_t.flags & 1), "dropped_untrained": int(st_u.flags & 1)})
    scale = np.abs(p_j).max()
    for st, p in ((st_j, p_j), (st_m, p_m), (st_t, p_t), (st_u, p_u), (st_w, p_w)):
        assert st.status == abi.SOLVE_CONVERGED and st.true_relative_residual <= 1e-5
        assert np.abs(p - p_j).max() <= 5e-3 * scale
    assert not (st_t.flags & 1)  # the trained network was kept
    assert st_t.iterations <= st_m.iterations
    assert st_t.iterations <= st_u.iterations or (st_u.flags & 1)
    assert st_t.iterations < 0.1 * st_j.iterations


def test_learned_mode_needs_a_network(smoke_lib):
    cfg, occ, boxes, _ = T.scene((16, 16, 16), 3)
    sim = smoke_b200.Simulation(smoke_lib, cfg, torch.cuda.Stream())
    with pytest.raises(smoke_b200.SmokeError):
        sim.set_solver(**LEARNED)
    with pytest.raises(smoke_b200.SmokeError):  # the network warm start exists only in the learned mode
        sim.set_solver(**dict(JACOBI, warm_start=2))
    sim.close()


def test_operator_apply_matches_solution(smoke_lib):
    """A p = b for the converged pressure of a step (the operator the learned trainer builds its pairs with)."""
    sim, keep = held_out_system(smoke_lib)
    st, p = solve(sim, dict(JACOBI, tolerance=1e-7, max_iterations=8000))
    b = sim.snapshot([abi.VIEW_FLOW_PRESSURE_RHS])["pressure_rhs"]
    with torch.cuda.stream(sim.stream):
        ap = sim.apply_operator(sim.view(abi.VIEW_FLOW_PRESSURE).clone())
    sim.stream.synchronize()
    assert np.linalg.norm(ap.cpu().numpy() - b) <= 1e-5 * np.linalg.norm(b)
    sim.close()


def test_multigrid_apply_is_the_solvers_preconditioner(smoke_lib):
    """The standalone V-cycle (smoke_b200_apply_multigrid_cuda, the trainer's) is the solve's preconditioner: flexible
    CG iterations with it, run in torch around the library's operator and V-cycle, reach the same relative residual
    in the same number of iterations as the library's multigrid FCG (up to one)."""
    sim, keep = held_out_system(smoke_lib)
    st_m, _ = solve(sim, dict(MULTIGRID, refinement=0, tolerance=1e-5))
    with torch.cuda.stream(sim.stream):
        b = sim.view(abi.VIEW_FLOW_PRESSURE_RHS).clone()
        r = b.clone()
        p_prev = q_prev = None
        its = 0
        bb = float(torch.sum(b.double() ** 2))
        while float(torch.sum(r.double() ** 2)) > 1e-10 * bb and its < 60:
            z = sim.apply_multigrid(r)
            if p_prev is None:
                p = z
            else:
                beta = -float(torch.sum(z.double() * q_prev.double())) / float(torch.sum(p_prev.double() * q_prev.double()))
                p = z + beta * p_prev
            q = sim.apply_operator(p)
            alpha = float(torch.sum(p.double() * r.double())) / float(torch.sum(p.double() * q.double()))
            r = r - alpha * q
            p_prev, q_prev = p, q
            its += 1
    sim.stream.synchronize()
    sim.close()
    assert st_m.status == abi.SOLVE_CONVERGED
    assert abs(its - st_m.iterations) <= 1, (its, st_m.iterations)


def test_useless_network_costs_no_iterations(smoke_lib):
    """A network of huge random weights is a useless correction: the energy-optimal step along it (or, if the solve
    stalls anyway, dropping it: flags bit 0) leaves the multigrid V-cycle's convergence, and the solve reaches the
    tolerance with the Jacobi-PCG answer in about the multigrid form's iterations."""
    sim, keep = held_out_system(smoke_lib)
    st_m, _ = solve(sim, MULTIGRID)
    with smoke_b200.Net(smoke_lib, seed=0) as bad:
        bad.set_parameters(U.initial_like(7, scale=30.0))
        st, p = solve(sim, dict(LEARNED, max_iterations=600), bad)
    st_j, p_j = solve(sim, JACOBI)
    report("learned/useless_network", {"iterations": st.iterations, "multigrid": st_m.iterations, "dropped": int(st.flags & 1)})
    assert st.status == abi.SOLVE_CONVERGED
    assert st.iterations <= st_m.iterations + 2
    assert np.abs(p - p_j).max() <= 5e-3 * np.abs(p_j).max()
    sim.close()


@pytest.mark.parametrize("schedule", [1, 3, 0])
def test_schedule_graph_matches_eager(smoke_lib, trained, schedule):
    """With the network in the first `schedule` iterations of each pass (0: all), the graph solve (a loop with the
    network, then a loop with the V-cycle alone) and the host-driven solve (which picks each iteration's body from
    the network flag the update left) take the same iterations to the same answer; every schedule reaches the
    tolerance."""
    net, _ = trained
    sim, keep = held_out_system(smoke_lib)
    sim.set_learned_iterations(schedule)
    st_g, p_g = solve(sim, LEARNED, net)
    sim.solve_pressure(eager=True)
    st_e = sim.solver_status()
    p_e = sim.snapshot([abi.VIEW_FLOW_PRESSURE])["pressure"]
    sim.set_learned_iterations(0)
    sim.close()
    report(f"learned/schedule{schedule}", {"graph": st_g.iterations, "eager": st_e.iterations})
    for st in (st_g, st_e):
        assert st.status == abi.SOLVE_CONVERGED and st.true_relative_residual <= 1e-5
    assert abs(st_g.iterations - st_e.iterations) <= 1 and st_g.passes == st_e.passes
    assert np.abs(p_g - p_e).max() <= 1e-5 * np.abs(p_g).max()
