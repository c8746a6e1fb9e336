"""The plume benchmark scene, expressed through the C ABI so that one driver feeds any library that exports it.

Scene (the metric's workload): an n^3 MAC grid, h = 1/n, dt = 0.01, closed no-slip walls, ZERO_FLUX scalars,
ambient temperature 0, buoyancy alpha = 0.08, beta = 0.97, vorticity confinement 0.35. A source box at the bottom
centre (n/8 x n/16 x n/8 cells: 16 x 8 x 16 at 128^3) holds density 1 and temperature 1 and drives an inflow of
v_y = 1 + xi, xi uniform in [-0.1, 0.1], drawn per source cell and per step from a counter-based generator
(splitmix64 of seed, step and cell), so every library sees identical inputs.

The ABI has no velocity or value-clamp input, so each step the driver (i) sets the box's density and temperature
SOURCES to (1 - value) / dt, which makes the advected temporaries exactly 1 in the box, and (ii) sets the box
force f_y = (v_target - v_y) / dt from the centred velocity view, which brings the box's face velocity to the
target. Outside the box the sources and forces are 0. The per-step host input is the xi of the source cells.
"""
from __future__ import annotations

import numpy as np

import smoke_abi as abi

MASK64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """Vectorised splitmix64 finaliser (Steele, Lea & Flood 2014) on uint64 arrays."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(MASK64)
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(MASK64)
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(MASK64)
    return x ^ (x >> np.uint64(31))


def uniform(seed: int, step: int, cells: np.ndarray, lo: float, hi: float) -> np.ndarray:
    key = (np.uint64(seed) << np.uint64(40)) ^ (np.uint64(step) << np.uint64(24))
    with np.errstate(over="ignore"):
        bits = splitmix64(cells.astype(np.uint64) ^ key)
    unit = (bits >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    return (lo + (hi - lo) * unit).astype(np.float32)


def plume_config(n: int = 128, mode: int = abi.MONOTONIC_CUBIC, pressure_iterations: int = 64) -> abi.Config:
    return abi.make_config(n, n, n, cell_size=1.0 / n, dt=0.01, pressure_iterations=pressure_iterations, ambient=0.0, alpha=0.08, beta=0.97, epsilon=0.35, mode=mode)


def source_box(n: int):
    """(z, y, x) slices of the source box: n/8 x n/16 x n/8 cells at the bottom centre
    (x, z in [56, 72) and y in [0, 8) at n = 128)."""
    bx, by = max(1, n // 8), max(1, n // 16)
    x0 = (n - bx) // 2
    return (slice(x0, x0 + bx), slice(0, by), slice(x0, x0 + bx))


class PlumeDriver:
    """Per-step inputs of the plume scene for one Simulation (any library). All work is enqueued on the
    simulation's stream; `inputs_for(step)` is the host-side input of that step (pinned)."""

    def __init__(self, sim, n: int, seed: int = 1):
        import torch

        self.sim = sim
        self.n = n
        self.seed = seed
        self.dt = float(sim.config.dt)
        zs, ys, xs = source_box(n)
        self.box = (zs, ys, xs)
        shape = (zs.stop - zs.start, ys.stop - ys.start, xs.stop - xs.start)
        self.box_shape = shape
        z, y, x = np.meshgrid(np.arange(zs.start, zs.stop), np.arange(ys.start, ys.stop), np.arange(xs.start, xs.stop), indexing="ij")
        self.box_cells = (z * n * n + y * n + x).reshape(-1)
        dev = torch.device("cuda")
        with torch.cuda.stream(sim.stream):
            self.force_y = torch.zeros((n, n, n), dtype=torch.float32, device=dev)
            self.density_source = torch.zeros((n, n, n), dtype=torch.float32, device=dev)
            self.temperature_source = torch.zeros((n, n, n), dtype=torch.float32, device=dev)
            self.xi_dev = torch.zeros(shape, dtype=torch.float32, device=dev)
            self.total_dev = torch.zeros(1, dtype=torch.float32, device=dev)
        self.xi_host = torch.zeros(shape, dtype=torch.float32).pin_memory()
        self.total_host = torch.zeros(1, dtype=torch.float32).pin_memory()
        self.h2d_bytes = self.xi_host.numel() * 4
        self.d2h_bytes = 4

    def inputs_for(self, step: int):
        self.xi_host.copy_(__import__("torch").from_numpy(uniform(self.seed, step, self.box_cells, -0.1, 0.1).reshape(self.box_shape)))
        return self.xi_host

    def apply(self, step: int, host_inputs=None):
        """Enqueue the H2D of the step's input and the source/force updates (before the step)."""
        import torch

        sim = self.sim
        xi = host_inputs if host_inputs is not None else self.inputs_for(step)
        zs, ys, xs = self.box
        with torch.cuda.stream(sim.stream):
            self.xi_dev.copy_(xi, non_blocking=True)
            _, vy, _ = sim.view(abi.VIEW_FLOW_VELOCITY)
            self.force_y[zs, ys, xs] = (1.0 + self.xi_dev - vy[zs, ys, xs]) / self.dt
            rho = sim.view(abi.VIEW_DENSITY)
            self.density_source[zs, ys, xs] = (1.0 - rho[zs, ys, xs]) / self.dt
            tem = sim.view(abi.VIEW_TEMPERATURE)
            self.temperature_source[zs, ys, xs] = (1.0 - tem[zs, ys, xs]) / self.dt
            sim.update_force(None, self.force_y, None)
            sim.update_density_source(self.density_source)
            sim.update_temperature_source(self.temperature_source)

    def read_result(self):
        """Enqueue the D2H of the step's result (total density)."""
        import torch

        with torch.cuda.stream(self.sim.stream):
            self.total_dev.copy_(torch.sum(self.sim.view(abi.VIEW_DENSITY)).reshape(1))
            self.total_host.copy_(self.total_dev, non_blocking=True)
        return self.total_host


def closed_box_residual(p, b):
    """||b - A p|| / ||b|| for the pressure operator of a closed box without solids (torch, on the device):
    the anchor is cell 0 (identity row, excluded from its neighbours' off-diagonals); every other row has the
    in-domain neighbour count on the diagonal and -1 per in-domain neighbour."""
    import torch

    pz = p.clone()
    pz.view(-1)[0] = 0.0
    s = torch.zeros_like(p)
    d = torch.zeros_like(p)
    ones = torch.ones_like(p)
    for axis in range(3):
        n = p.shape[axis]
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis] = slice(0, n - 1)
        hi[axis] = slice(1, n)
        s[tuple(hi)] += pz[tuple(lo)]
        s[tuple(lo)] += pz[tuple(hi)]
        d[tuple(hi)] += ones[tuple(lo)]
        d[tuple(lo)] += ones[tuple(hi)]
    ap = d * p - s
    ap.view(-1)[0] = p.view(-1)[0]
    bn = torch.linalg.vector_norm(b)
    return torch.linalg.vector_norm(b - ap) / bn if bn > 0 else bn
