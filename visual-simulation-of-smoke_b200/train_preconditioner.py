"""Training of the learned preconditioner (smoke_b200_net_*_cuda): pressure problems generated by the library's own
solver, training on the GPU through the network's tensor-core forward and backward kernels and its Adam kernel, and
the parameters saved as raw little-endian FP32 (smoke_b200_net_parameter_count() values).

The network corrects what one multigrid V-cycle leaves of an error (SMOKE_B200_SOLVER_LEARNED_FCG preconditions
with z = V(r) + P N(R (r - A V(r)))). For an error e with residual r = A e, the V-cycle gives z = V(r)
(smoke_b200_apply_multigrid_cuda) and leaves the error e - z, whose residual is r - A z, with A applied by
smoke_b200_apply_operator_cuda. The network runs on the multigrid hierarchy's level 1 (every extent halved): its
input is R(r - A z), the sums of the 2 x 2 x 2 children (as the solve restricts it), its mask marks the level-1
cells without a fluid child, and its target is the mean of e - z over each cell's fluid children; the solve prolongs
its output back with the V-cycle's trilinear prolongation. The errors come from two sources:

 - the solver's own iterates: plume scenes (seeded source position and strength U[0.5, 1.5], 0-3 solid spheres)
   are stepped with the multigrid FCG; at a step, the pressure system (b = the FLOW_PRESSURE_RHS view) is solved
   exactly (relative residual 1e-10, FP64 refinement) and with the FCG stopped after k iterations, and
   e = x_exact - x_k is the error the preconditioner sees at iteration k;
 - multi-scale random errors (smooth random fields on grids 2^j times coarser, trilinearly interpolated, plus a
   little white noise; 0 at solids and at the anchor), for the residuals of every frequency a Krylov solve produces.

Usage:

    python visual-simulation-of-smoke_b200/train_preconditioner.py --out learned_preconditioner.f32
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import plume_scene  # noqa: E402
import smoke_abi as abi  # noqa: E402

DEFAULT_WEIGHTS = os.path.join(HERE, "learned_preconditioner.f32")
STEP_SOLVER = dict(mode=abi.SOLVER_MG_FCG, reduction=abi.REDUCTION_FP64, max_iterations=200, tolerance=1e-5, refinement=1, warm_start=True)
EXACT_SOLVER = dict(mode=abi.SOLVER_MG_FCG, reduction=abi.REDUCTION_FP64, max_iterations=400, tolerance=1e-10, refinement=6)
ITERATES = (0, 1, 2, 4, 6)  # FCG iterations after which the iterate's error becomes a sample


def scene(shape, seed):
    """(config, occupancy, boxes, strength) of a plume scene on an nx x ny x nz grid with a seeded source position
    and strength (U[0.5, 1.5]) and 0-3 seeded solid spheres."""
    nx, ny, nz = shape
    u = plume_scene.uniform(seed, 7, np.arange(16), 0.0, 1.0)
    cfg = plume_scene.scene_config(nx, ny, nz)
    bx, by, bz = max(1, nx // 8), max(1, ny // 16), max(1, nz // 8)
    x0, z0 = int(u[3] * (nx - bx)), int(u[4] * (nz - bz))
    occ = np.zeros((nz, ny, nx), dtype=np.uint8)
    for k in range(int(u[5] * 4)):
        r = 2.0 + u[6 + k] * 0.15 * min(nx, nz)
        centre = (u[9 + k] * nx, (0.35 + 0.5 * u[12 + k]) * ny, (0.2 + 0.6 * u[6 + k]) * nz)
        occ |= plume_scene.sphere_occupancy((nz, ny, nx), centre, r)
    strength = 0.5 + float(u[15])
    return cfg, occ, [(slice(z0, z0 + bz), slice(0, by), slice(x0, x0 + bx))], strength


def synthetic_errors(shape_zyx, fluid, count: int, gen):
    """`count` multi-scale random fields on the device, 0 where `fluid` is 0 and at the anchor (first fluid cell)."""
    import torch
    import torch.nn.functional as F

    nz, ny, nx = shape_zyx
    anchor = int(torch.nonzero(fluid.reshape(-1) > 0)[0])
    out = []
    for _ in range(count):
        j = int(torch.randint(1, 6, (1,), generator=gen))
        e = torch.zeros(shape_zyx, device="cuda")
        for level, amp in ((j, 1.0), (max(0, j - 1), 0.5)):
            c = [max(2, -(-v // (1 << level))) for v in (nz, ny, nx)]
            coarse = torch.randn([1, 1] + c, generator=gen).cuda()
            e += amp * F.interpolate(coarse, size=(nz, ny, nx), mode="trilinear", align_corners=True)[0, 0]
        e += 0.05 * torch.randn(shape_zyx, generator=gen).cuda()
        e *= fluid
        e.view(-1)[anchor] = 0.0
        out.append(e)
    return out


def vcycle_pair(sim, e, r):
    """(r - A V(r), e - V(r)): the residual and the error one V-cycle leaves of the error e with residual r."""
    z = sim.apply_multigrid(r)
    return r - sim.apply_operator(z), e - z


def _children(x):
    """[nz, ny, nx] -> [nz', ny', nx', 8]: the 2 x 2 x 2 children of every level-1 cell (extents rounded up, missing
    children 0)."""
    import torch.nn.functional as F

    nz, ny, nx = x.shape
    x = F.pad(x, (0, nx % 2, 0, ny % 2, 0, nz % 2))
    z, y, w = x.shape
    return x.reshape(z // 2, 2, y // 2, 2, w // 2, 2).permute(0, 2, 4, 1, 3, 5).reshape(z // 2, y // 2, w // 2, 8)


def coarse_mask(occ):
    """The network's mask on level 1 (uint8, 1 = no fluid child) of a level-0 occupancy (1 = solid)."""
    return (_children((occ == 0).float()).sum(-1) == 0).to(occ.dtype)


def coarse_pair(r_in, t, occ):
    """A level-0 pair (input r - A z, target e - z) on level 1: the child sums of the input (the solve's restriction)
    and the mean of the target over the fluid children (0 where there is none)."""
    fluid = _children((occ == 0).float())
    count = fluid.sum(-1)
    target = (_children(t) * fluid).sum(-1) / count.clamp(min=1.0)
    return _children(r_in).sum(-1).contiguous(), target.contiguous()


def generate(lib, shape, scenes: int, per_scene: int, seed: int = 0, spin: int = 8, every: int = 3, synthetic: int = 0, iterates=ITERATES):
    """Samples (input, mask, target) on level 1 as CUDA tensors [count, nz', ny', nx'] (extents halved, rounding up)
    from `scenes` plume scenes on `shape`: `per_scene` pressure systems each (one every `every` steps after `spin`
    steps), one sample per iterate count in `iterates` of each, plus `synthetic` multi-scale random errors per scene."""
    import torch

    import smoke_b200

    inputs, occs, targets = [], [], []
    for k in range(scenes):
        cfg, occ, boxes, strength = scene(shape, seed * 1000 + k)
        stream = torch.cuda.Stream()
        sim = smoke_b200.Simulation(lib, cfg, stream)
        with torch.cuda.stream(stream):
            o = torch.from_numpy(occ).cuda()
            sim.update_occupancy(o)
            mask = coarse_mask(o)
        sim.set_solver(**STEP_SOLVER)
        driver = plume_scene.SceneDriver(sim, boxes, seed=seed * 1000 + k + 1, strength=strength)
        step = 0
        for j in range(spin + per_scene * every):
            driver.apply(step)
            sim.step()
            step += 1
            if j >= spin and (j - spin) % every == every - 1:
                sim.set_solver(**EXACT_SOLVER)
                sim.solve_pressure()
                with torch.cuda.stream(stream):
                    exact = sim.view(abi.VIEW_FLOW_PRESSURE).clone()
                for it in iterates:
                    if it > 0:  # the FP32 iterate after `it` FCG iterations from zero
                        sim.set_solver(**dict(EXACT_SOLVER, max_iterations=it, refinement=0, tolerance=1e-12))
                    with torch.cuda.stream(stream):
                        if it == 0:
                            e = exact.clone()  # x_0 = 0
                        else:
                            sim.solve_pressure()
                            e = exact - sim.view(abi.VIEW_FLOW_PRESSURE)
                        r_in, t = coarse_pair(*vcycle_pair(sim, e, sim.apply_operator(e)), o)
                        inputs.append(r_in)
                        targets.append(t)
                        occs.append(mask)
                sim.set_solver(**STEP_SOLVER)
        if synthetic:
            gen = torch.Generator().manual_seed(seed * 1000 + k)
            with torch.cuda.stream(stream):
                fluid = (o == 0).float()
                for e in synthetic_errors(o.shape, fluid, synthetic, gen):
                    r_in, t = coarse_pair(*vcycle_pair(sim, e, sim.apply_operator(e)), o)
                    inputs.append(r_in)
                    targets.append(t)
                    occs.append(mask)
        stream.synchronize()
        sim.close()
    return torch.stack(inputs), torch.stack(occs), torch.stack(targets)


def train(net, data, steps: int, batch: int = 4, lr: float = 1e-3, seed: int = 0, log_every: int = 0):
    """Adam steps on random batches of `data` (input, occupancy, target), or of a list of such groups of different
    grid sizes (each step draws its batch from one group, in turn); learning rate halved at 60% and 85%. Returns the
    mean batch loss of every step."""
    import torch

    groups = data if isinstance(data, list) else [data]
    g = np.random.default_rng(seed)
    losses = []
    for k in range(steps):
        rhs, occ, target = groups[k % len(groups)]
        count = rhs.shape[0]
        idx = torch.from_numpy(g.choice(count, size=min(batch, count), replace=False)).cuda()
        rate = lr * (0.5 if k >= 0.6 * steps else 1.0) * (0.5 if k >= 0.85 * steps else 1.0)
        loss = net.train_step(rhs[idx].contiguous(), occ[idx].contiguous(), target[idx].contiguous(), rate)
        losses.append(loss)
        if log_every and (k % log_every == 0 or k == steps - 1):
            print(f"step {k:5d}  loss {loss:.4f}", flush=True)
    return losses


def load(net, path: str = DEFAULT_WEIGHTS):
    values = np.fromfile(path, dtype="<f4")
    if values.size != net.parameter_count:
        raise ValueError(f"{path}: {values.size} parameters, the network has {net.parameter_count}")
    net.set_parameters(values)
    return net


def main():
    import torch

    import smoke_b200

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--scenes64", type=int, default=256, help="64^3 scenes")
    ap.add_argument("--scenes128", type=int, default=32, help="128^3 scenes")
    ap.add_argument("--per-scene", type=int, default=6, help="pressure systems per scene")
    ap.add_argument("--synthetic", type=int, default=12, help="random errors per scene")
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    lib = smoke_b200.SmokeLibrary()
    t0 = time.time()
    groups = []
    if args.scenes64:
        groups.append(generate(lib, (64, 64, 64), args.scenes64, args.per_scene, seed=args.seed, synthetic=args.synthetic))
    if args.scenes128:
        groups.append(generate(lib, (128, 128, 128), args.scenes128, args.per_scene, seed=args.seed + 1, synthetic=args.synthetic))
    torch.cuda.synchronize()
    print(f"{sum(g[0].shape[0] for g in groups)} samples in {time.time() - t0:.1f} s", flush=True)
    net = smoke_b200.Net(lib, seed=args.seed)
    t0 = time.time()
    losses = train(net, groups, args.steps, args.batch, args.lr, seed=args.seed, log_every=max(1, args.steps // 10))
    torch.cuda.synchronize()
    print(f"trained {args.steps} steps in {time.time() - t0:.1f} s: loss {np.mean(losses[:20]):.4f} -> {np.mean(losses[-20:]):.4f}", flush=True)
    net.parameters().astype("<f4").tofile(args.out)
    net.close()


if __name__ == "__main__":
    main()
