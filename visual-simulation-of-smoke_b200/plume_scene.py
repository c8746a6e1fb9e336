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


class SceneDriver:
    """Per-step inputs of a plume scene with any grid and any source boxes, for one Simulation (any library). Every
    box holds density and temperature `strength` (1 by default) and drives an inflow v_y = strength * (1 + xi) (xi
    drawn per cell and step, the boxes' cells in box order). All work is enqueued on the simulation's stream;
    `inputs_for(step)` is the host-side input of that step (pinned)."""

    def __init__(self, sim, boxes, seed: int = 1, strength: float = 1.0):
        import torch

        self.sim = sim
        self.seed = seed
        self.strength = float(strength)
        self.dt = float(sim.config.dt)
        nx, ny, nz = sim.config.nx, sim.config.ny, sim.config.nz
        self.shape = (nz, ny, nx)
        self.boxes = list(boxes)
        cells, self.sizes = [], []
        for zs, ys, xs in self.boxes:
            z, y, x = np.meshgrid(np.arange(zs.start, zs.stop), np.arange(ys.start, ys.stop), np.arange(xs.start, xs.stop), indexing="ij")
            cells.append((z * ny * nx + y * nx + x).reshape(-1))
            self.sizes.append((zs.stop - zs.start, ys.stop - ys.start, xs.stop - xs.start))
        self.box_cells = np.concatenate(cells)
        dev = torch.device("cuda")
        with torch.cuda.stream(sim.stream):
            self.force_y = torch.zeros(self.shape, dtype=torch.float32, device=dev)
            self.density_source = torch.zeros(self.shape, dtype=torch.float32, device=dev)
            self.temperature_source = torch.zeros(self.shape, dtype=torch.float32, device=dev)
            self.xi_dev = torch.zeros(self.box_cells.size, dtype=torch.float32, device=dev)
            self.total_dev = torch.zeros(1, dtype=torch.float32, device=dev)
        self.xi_host = torch.zeros(self.box_cells.size, dtype=torch.float32).pin_memory()
        self.xi_read = None  # event: the last asynchronous copy out of xi_host has run
        self.total_host = torch.zeros(1, dtype=torch.float32).pin_memory()
        self.h2d_bytes = self.xi_host.numel() * 4
        self.d2h_bytes = 4

    def inputs_for(self, step: int):
        # the pinned buffer is read by an asynchronous copy: a step enqueued ahead of the GPU must not see the next
        # step's values, so wait for the previous copy before overwriting it
        if self.xi_read is not None:
            self.xi_read.synchronize()
        self.xi_host.copy_(__import__("torch").from_numpy(uniform(self.seed, step, self.box_cells, -0.1, 0.1)))
        return self.xi_host

    def apply(self, step: int, host_inputs=None):
        """Enqueue the H2D of the step's input and the source/force updates (before the step)."""
        import torch

        sim = self.sim
        xi = host_inputs if host_inputs is not None else self.inputs_for(step)
        with torch.cuda.stream(sim.stream):
            self.xi_dev.copy_(xi, non_blocking=True)
            if xi is self.xi_host:
                self.xi_read = torch.cuda.Event()
                self.xi_read.record(sim.stream)
            _, vy, _ = sim.view(abi.VIEW_FLOW_VELOCITY)
            rho = sim.view(abi.VIEW_DENSITY)
            tem = sim.view(abi.VIEW_TEMPERATURE)
            start = 0
            for (zs, ys, xs), size in zip(self.boxes, self.sizes):
                count = size[0] * size[1] * size[2]
                xi_box = self.xi_dev[start:start + count].reshape(size)
                start += count
                k = self.strength
                if k == 1.0:
                    self.force_y[zs, ys, xs] = (1.0 + xi_box - vy[zs, ys, xs]) / self.dt
                    self.density_source[zs, ys, xs] = (1.0 - rho[zs, ys, xs]) / self.dt
                    self.temperature_source[zs, ys, xs] = (1.0 - tem[zs, ys, xs]) / self.dt
                else:
                    self.force_y[zs, ys, xs] = (k * (1.0 + xi_box) - vy[zs, ys, xs]) / self.dt
                    self.density_source[zs, ys, xs] = (k - rho[zs, ys, xs]) / self.dt
                    self.temperature_source[zs, ys, xs] = (k - tem[zs, ys, xs]) / self.dt
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


class PlumeDriver(SceneDriver):
    """The n^3 plume: one source box at the bottom centre (source_box)."""

    def __init__(self, sim, n: int, seed: int = 1):
        self.n = n
        super().__init__(sim, [source_box(n)], seed)
        self.box = self.boxes[0]


# --------------------------------------------------------------------------------------------- other scenes
def scene_config(nx: int, ny: int, nz: int, mode: int = abi.MONOTONIC_CUBIC, pressure_iterations: int = 64) -> abi.Config:
    """The plume scene's parameters on an nx x ny x nz grid, h = 1/nx."""
    return abi.make_config(nx, ny, nz, cell_size=1.0 / nx, dt=0.01, pressure_iterations=pressure_iterations, ambient=0.0, alpha=0.08, beta=0.97, epsilon=0.35, mode=mode)


def sphere_occupancy(shape_zyx, centre_xyz, radius: float) -> np.ndarray:
    """uint8 occupancy (z, y, x): 1 where the cell centre lies within `radius` cells of `centre_xyz` (cell units)."""
    nz, ny, nx = shape_zyx
    z, y, x = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    cx, cy, cz = centre_xyz
    return (((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) <= radius * radius).astype(np.uint8)


def large_scene(seed: int = 1):
    """256 x 384 x 256 with a solid sphere (radius 40 cells, centred at x = z = 128 and 40% of the height) and two
    32 x 8 x 32 source boxes on the floor at seeded x, z positions. Returns (config, occupancy, boxes)."""
    nx, ny, nz = 256, 384, 256
    cfg = scene_config(nx, ny, nz)
    occ = sphere_occupancy((nz, ny, nx), (128.0, 0.4 * ny, 128.0), 40.0)
    pos = uniform(seed, 0, np.arange(4), 0.0, 1.0)
    boxes = []
    for k in range(2):
        x0 = int(pos[2 * k] * (nx - 32))
        z0 = int(pos[2 * k + 1] * (nz - 32))
        boxes.append((slice(z0, z0 + 32), slice(0, 8), slice(x0, x0 + 32)))
    return cfg, occ, boxes


def batched_scenes(count: int = 48, seed: int = 1):
    """`count` independent plume scenes of uneven sizes: per-axis extents drawn in [32, 128] x [32, 192] x
    [32, 128], one source box (nx/8 x ny/16 x nz/8) at a random floor position and 0-3 solid spheres above it.
    Returns a list of (config, occupancy, boxes)."""
    out = []
    for s in range(count):
        u = uniform(seed, 1000 + s, np.arange(16), 0.0, 1.0)
        nx, ny, nz = 32 + int(u[0] * 97), 32 + int(u[1] * 161), 32 + int(u[2] * 97)
        cfg = scene_config(nx, ny, nz)
        bx, by, bz = max(1, nx // 8), max(1, ny // 16), max(1, nz // 8)
        x0, z0 = int(u[3] * (nx - bx)), int(u[4] * (nz - bz))
        occ = np.zeros((nz, ny, nx), dtype=np.uint8)
        for k in range(int(u[5] * 4)):  # 0-3 spheres in the upper part of the domain
            r = 3.0 + u[6 + k] * 0.12 * min(nx, nz)
            centre = (u[9 + k] * nx, (0.45 + 0.4 * u[12 + k]) * ny, (0.25 + 0.5 * u[6 + k]) * nz)
            occ |= sphere_occupancy((nz, ny, nx), centre, r)
        out.append((cfg, occ, [(slice(z0, z0 + bz), slice(0, by), slice(x0, x0 + bx))]))
    return out


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
