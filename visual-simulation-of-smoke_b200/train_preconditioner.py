"""Training of the learned preconditioner (smoke_b200_net_*_cuda): pressure problems generated by the library's own
solver, training on the GPU through the network's tensor-core forward and backward kernels and its Adam kernel, and
the parameters saved as raw little-endian FP32 (smoke_b200_net_parameter_count() values).

Samples: plume scenes on a fixed grid (one floor source at a random position, 0-3 solid spheres), stepped with the
Jacobi-preconditioned CG to relative residual 1e-6 (FP64 dot products and refinement). After each step, the step's
pressure system is one sample: (right-hand side = the FLOW_PRESSURE_RHS view, occupancy, pressure = the FLOW_PRESSURE
view). Inside a Krylov solve the preconditioner sees residuals of every frequency, not only right-hand sides of
physical flows, so each scene also gives synthetic pairs (A e, e) for multi-scale random e (smooth random fields on
grids 2^j times coarser, trilinearly interpolated, plus a little white noise; 0 at solids and at the anchor), with A
applied by smoke_b200_apply_operator_cuda. Usage:

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
DATA_SOLVER = dict(mode=abi.SOLVER_JACOBI_PCG, reduction=abi.REDUCTION_FP64, max_iterations=4000, tolerance=1e-6, refinement=3)


def scene(shape, seed):
    """(config, occupancy, boxes) of a plume scene on an nx x ny x nz grid with seeded source and spheres."""
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
    return cfg, occ, [(slice(z0, z0 + bz), slice(0, by), slice(x0, x0 + bx))]


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


def generate(lib, shape, scenes: int, per_scene: int, seed: int = 0, spin: int = 6, every: int = 3, synthetic: int = 0):
    """Samples (rhs, occupancy, pressure) as CUDA tensors [count, nz, ny, nx] from `scenes` plume scenes, `per_scene`
    systems each (one every `every` steps after `spin` steps) plus `synthetic` pairs (A e, e) per scene."""
    import torch

    import smoke_b200

    rhs, occs, prs = [], [], []
    for k in range(scenes):
        cfg, occ, boxes = scene(shape, seed * 1000 + k)
        stream = torch.cuda.Stream()
        sim = smoke_b200.Simulation(lib, cfg, stream)
        with torch.cuda.stream(stream):
            o = torch.from_numpy(occ).cuda()
            sim.update_occupancy(o)
        sim.set_solver(**DATA_SOLVER)
        driver = plume_scene.SceneDriver(sim, boxes, seed=seed * 1000 + k + 1)
        step = 0
        for j in range(spin + per_scene * every):
            driver.apply(step)
            sim.step()
            step += 1
            if j >= spin and (j - spin) % every == every - 1:
                with torch.cuda.stream(stream):
                    rhs.append(sim.view(abi.VIEW_FLOW_PRESSURE_RHS).clone())
                    prs.append(sim.view(abi.VIEW_FLOW_PRESSURE).clone())
                    occs.append(o.clone())
        if synthetic:
            gen = torch.Generator().manual_seed(seed * 1000 + k)
            with torch.cuda.stream(stream):
                fluid = (o == 0).float()
                for e in synthetic_errors(o.shape, fluid, synthetic, gen):
                    rhs.append(sim.apply_operator(e))
                    prs.append(e)
                    occs.append(o.clone())
        stream.synchronize()
        sim.close()
    return torch.stack(rhs), torch.stack(occs), torch.stack(prs)


def train(net, data, steps: int, batch: int = 4, lr: float = 2e-3, seed: int = 0, log_every: int = 0):
    """Adam steps on random batches of `data` (rhs, occupancy, pressure); learning rate halved at 60% and 85%.
    Returns the mean batch loss of every step."""
    import torch

    rhs, occ, prs = data
    count = rhs.shape[0]
    g = np.random.default_rng(seed)
    losses = []
    for k in range(steps):
        idx = torch.from_numpy(g.choice(count, size=min(batch, count), replace=False)).cuda()
        rate = lr * (0.5 if k >= 0.6 * steps else 1.0) * (0.5 if k >= 0.85 * steps else 1.0)
        loss = net.train_step(rhs[idx].contiguous(), occ[idx].contiguous(), prs[idx].contiguous(), rate)
        losses.append(loss)
        if log_every and (k % log_every == 0 or k == steps - 1):
            print(f"step {k:5d}  loss {loss:.4f}", flush=True)
    return losses


def load(net, path: str = DEFAULT_WEIGHTS):
    values = np.fromfile(path, dtype="<f4")
    net.set_parameters(values)
    return net


def main():
    import torch

    import smoke_b200

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--shape", type=int, nargs=3, default=[48, 64, 48])
    ap.add_argument("--scenes", type=int, default=12)
    ap.add_argument("--per-scene", type=int, default=6)
    ap.add_argument("--synthetic", type=int, default=18, help="synthetic (A e, e) pairs per scene")
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    lib = smoke_b200.SmokeLibrary()
    t0 = time.time()
    data = generate(lib, tuple(args.shape), args.scenes, args.per_scene, seed=args.seed, synthetic=args.synthetic)
    torch.cuda.synchronize()
    print(f"{data[0].shape[0]} samples of {tuple(args.shape)} in {time.time() - t0:.1f} s", flush=True)
    net = smoke_b200.Net(lib, seed=args.seed)
    t0 = time.time()
    losses = train(net, data, args.steps, args.batch, args.lr, seed=args.seed, log_every=max(1, args.steps // 10))
    print(f"trained {args.steps} steps in {time.time() - t0:.1f} s: loss {losses[0]:.4f} -> {np.mean(losses[-20:]):.4f}", flush=True)
    net.parameters().astype("<f4").tofile(args.out)
    net.close()


if __name__ == "__main__":
    main()
