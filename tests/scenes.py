"""Seeded scenes shared by the parity tests: boundary configurations, random inputs, and loaders that put the
same inputs into a GPU context (through the ABI) and into the oracle."""
from __future__ import annotations

import numpy as np

import smoke_abi as abi

FACES = ("x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus")

# name -> (flow, density, temperature) boundary dicts
BOUNDARIES = {
    "closed": ({}, {}, {}),
    "plume": (  # the reference benchmark's layout: periodic x/z, no-slip floor, outflow top (benchmark.cu:96-123)
        {"x_minus": abi.PERIODIC, "x_plus": abi.PERIODIC, "y_plus": (abi.OUTFLOW, 0.0, 0.0, 0.0, 0.0), "z_minus": abi.PERIODIC, "z_plus": abi.PERIODIC},
        {"x_minus": abi.SCALAR_PERIODIC, "x_plus": abi.SCALAR_PERIODIC, "y_minus": (abi.FIXED_VALUE, 0.0), "y_plus": (abi.FIXED_VALUE, 0.0), "z_minus": abi.SCALAR_PERIODIC, "z_plus": abi.SCALAR_PERIODIC},
        {"x_minus": abi.SCALAR_PERIODIC, "x_plus": abi.SCALAR_PERIODIC, "y_minus": (abi.FIXED_VALUE, 0.0), "y_plus": (abi.FIXED_VALUE, 0.0), "z_minus": abi.SCALAR_PERIODIC, "z_plus": abi.SCALAR_PERIODIC},
    ),
    "mixed": (  # every flow type at least once, moving walls, outflow pressures
        {"x_minus": (abi.NO_SLIP_WALL, 0.3, -0.2, 0.1, 0.0), "x_plus": (abi.FREE_SLIP_WALL, -0.1, 0.2, 0.05, 0.0), "y_minus": (abi.OUTFLOW, 0.0, 0.0, 0.0, 0.25),
         "y_plus": (abi.OUTFLOW, 0.0, 0.0, 0.0, -0.5), "z_minus": abi.PERIODIC, "z_plus": abi.PERIODIC},
        {"x_minus": (abi.FIXED_VALUE, 0.7), "x_plus": abi.ZERO_FLUX, "y_minus": (abi.FIXED_VALUE, 0.2), "y_plus": abi.ZERO_FLUX, "z_minus": abi.SCALAR_PERIODIC, "z_plus": abi.SCALAR_PERIODIC},
        {"x_minus": abi.ZERO_FLUX, "x_plus": (abi.FIXED_VALUE, 1.5), "y_minus": abi.ZERO_FLUX, "y_plus": (abi.FIXED_VALUE, -0.3), "z_minus": abi.SCALAR_PERIODIC, "z_plus": abi.SCALAR_PERIODIC},
    ),
    "slip": (
        {f: abi.FREE_SLIP_WALL for f in FACES} | {"z_plus": (abi.OUTFLOW, 0.0, 0.0, 0.0, 0.1)},
        {}, {},
    ),
    "zout": (  # outflow on the low x and z faces (their face 0 copies face 1), periodic y, a moving wall
        {"x_minus": (abi.OUTFLOW, 0.0, 0.0, 0.0, 0.1), "x_plus": (abi.NO_SLIP_WALL, 0.0, 0.2, -0.1, 0.0), "y_minus": abi.PERIODIC, "y_plus": abi.PERIODIC,
         "z_minus": (abi.OUTFLOW, 0.0, 0.0, 0.0, -0.2), "z_plus": abi.FREE_SLIP_WALL},
        {"x_minus": (abi.FIXED_VALUE, 0.4), "y_minus": abi.SCALAR_PERIODIC, "y_plus": abi.SCALAR_PERIODIC, "z_plus": (abi.FIXED_VALUE, 0.0)},
        {"x_plus": (abi.FIXED_VALUE, 1.0), "y_minus": abi.SCALAR_PERIODIC, "y_plus": abi.SCALAR_PERIODIC},
    ),
}


def make_config(nx, ny, nz, boundary="closed", mode=abi.LINEAR, dt=0.01, pressure_iterations=64, **kw):
    flow, den, tem = BOUNDARIES[boundary]
    return abi.make_config(nx, ny, nz, dt=dt, mode=mode, pressure_iterations=pressure_iterations, flow=flow, density=den, temperature=tem, **kw)


def occupancy_spheres(cfg, rng, count=2):
    nz, ny, nx = abi.cell_shape(cfg)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    occ = np.zeros((nz, ny, nx), np.uint8)
    for _ in range(count):
        c = rng.uniform([0.2 * nz, 0.2 * ny, 0.2 * nx], [0.8 * nz, 0.8 * ny, 0.8 * nx])
        r = rng.uniform(1.2, max(1.6, 0.18 * min(nx, ny, nz)))
        occ[((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) <= r * r] = 1
    return occ


def random_inputs(cfg, seed=0, solids=True, cfl=0.6):
    """Seeded inputs for every ABI field plus a face velocity state. Velocities are scaled so that one step moves
    at most about `cfl` cells."""
    rng = np.random.default_rng(seed)
    cs = abi.cell_shape(cfg)
    su, sv, sw = abi.face_shapes(cfg)
    vmax = cfl * cfg.cell_size / cfg.dt
    out = {
        "u": rng.uniform(-vmax, vmax, su).astype(np.float32),
        "v": rng.uniform(-vmax, vmax, sv).astype(np.float32),
        "w": rng.uniform(-vmax, vmax, sw).astype(np.float32),
        "density": rng.uniform(0.0, 1.0, cs).astype(np.float32),
        "temperature": rng.uniform(-0.5, 1.5, cs).astype(np.float32),
        "density_source": np.where(rng.uniform(size=cs) < 0.1, rng.uniform(0, 5, cs), 0).astype(np.float32),
        "temperature_source": np.where(rng.uniform(size=cs) < 0.1, rng.uniform(-2, 5, cs), 0).astype(np.float32),
        "force_x": rng.uniform(-2, 2, cs).astype(np.float32),
        "force_y": rng.uniform(-2, 2, cs).astype(np.float32),
        "force_z": rng.uniform(-2, 2, cs).astype(np.float32),
        "occupancy": occupancy_spheres(cfg, rng) if solids else np.zeros(cs, np.uint8),
        "solid_velocity_x": rng.uniform(-0.3, 0.3, cs).astype(np.float32),
        "solid_velocity_y": rng.uniform(-0.3, 0.3, cs).astype(np.float32),
        "solid_velocity_z": rng.uniform(-0.3, 0.3, cs).astype(np.float32),
        "solid_temperature": rng.uniform(0.0, 2.0, cs).astype(np.float32),
    }
    return out


def load_gpu(sim, inp):
    """Put inputs into a GPU context through the ABI (+ the face-velocity extension when `u` is present)."""
    import torch

    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inp.items()}
    sim.stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(sim.stream):
        sim.update_density(d["density"])
        sim.update_temperature(d["temperature"])
        sim.update_density_source(d["density_source"])
        sim.update_temperature_source(d["temperature_source"])
        sim.update_force(d["force_x"], d["force_y"], d["force_z"])
        sim.update_occupancy(d["occupancy"])
        sim.update_solid_velocity(d["solid_velocity_x"], d["solid_velocity_y"], d["solid_velocity_z"])
        sim.update_solid_temperature(d["solid_temperature"])
        if "u" in d:
            sim.set_face_velocity(d["u"], d["v"], d["w"])
    sim.stream.synchronize()
    return d  # keep the device copies alive until the stream has consumed them


def load_oracle(state, inp):
    for k, v in inp.items():
        state.set(k, v)


def rel_err(a, b):
    """max|a-b| / max|b| (normwise L-infinity relative error; absolute when b is all zero)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    diff = np.abs(a - b).max() if b.size else 0.0
    return float(diff / scale) if scale > 0 else float(diff)


def rel_err_either(a, b32, b64, tol):
    """Normwise error of `a` against the FP32 oracle `b32` where each element may match the FP64 oracle `b64`
    instead: max over elements of min(|a - b32|, |a - b64|) / max|b32|, and the number of elements that match only
    the FP64 oracle (|a - b32| > tol * max|b32|). A back-trace whose end point lies within rounding of a domain or
    solid-cell boundary is bisected differently depending on the last bit of its position, and the GPU (which
    contracts a*b+c into FMAs) and the FP32 mirror (which does not) can round it apart; the GPU's element is then the
    FP64 truth's, not the mirror's."""
    a = np.asarray(a, np.float64)
    b32 = np.asarray(b32, np.float64)
    b64 = np.asarray(b64, np.float64)
    scale = np.abs(b32).max() if b32.size else 0.0
    if not scale > 0:
        scale = 1.0
    d32 = np.abs(a - b32)
    d = np.minimum(d32, np.abs(a - b64))
    return float(d.max() / scale) if d.size else 0.0, int(np.count_nonzero(d32 > tol * scale))
