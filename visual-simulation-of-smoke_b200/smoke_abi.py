"""ctypes mirror of the smoke C ABI (include/visual-simulation-of-smoke-3d.h and include/smoke_b200_ext.h).

The struct layouts are the reference's (visual-simulation-of-smoke-3d.h:22-154); tests/test_abi_layout.py pins
sizes and offsets. `make_config` builds a SmokeSimulationConfig from keyword arguments.
"""
from __future__ import annotations

import ctypes as C

# result codes (reference header :22-26)
RESULT_OK = 0
RESULT_OUT_OF_MEMORY = 1
RESULT_BACKEND_FAILURE = 2

# flow boundary types (:28-33)
NO_SLIP_WALL = 0
FREE_SLIP_WALL = 1
OUTFLOW = 2
PERIODIC = 3

# scalar boundary types (:35-39)
FIXED_VALUE = 0
ZERO_FLUX = 1
SCALAR_PERIODIC = 2

# advection modes (:72-75)
LINEAR = 0
MONOTONIC_CUBIC = 1

# view kinds (:116-132)
VIEW_DENSITY = 0
VIEW_DENSITY_SOURCE = 1
VIEW_TEMPERATURE = 2
VIEW_TEMPERATURE_SOURCE = 3
VIEW_FORCE = 4
VIEW_SOLID_VELOCITY = 5
VIEW_SOLID_TEMPERATURE = 6
VIEW_FLOW_VELOCITY = 7
VIEW_FLOW_VELOCITY_MAGNITUDE = 8
VIEW_FLOW_PRESSURE = 9
VIEW_FLOW_PRESSURE_RHS = 10
VIEW_FLOW_DIVERGENCE = 11
VIEW_FLOW_VORTICITY = 12
VIEW_FLOW_VORTICITY_MAGNITUDE = 13
VIEW_OCCUPANCY = 14
VIEW_NAMES = {
    VIEW_DENSITY: "density", VIEW_DENSITY_SOURCE: "density_source", VIEW_TEMPERATURE: "temperature",
    VIEW_TEMPERATURE_SOURCE: "temperature_source", VIEW_FORCE: "force", VIEW_SOLID_VELOCITY: "solid_velocity",
    VIEW_SOLID_TEMPERATURE: "solid_temperature", VIEW_FLOW_VELOCITY: "velocity",
    VIEW_FLOW_VELOCITY_MAGNITUDE: "velocity_magnitude", VIEW_FLOW_PRESSURE: "pressure",
    VIEW_FLOW_PRESSURE_RHS: "pressure_rhs", VIEW_FLOW_DIVERGENCE: "divergence", VIEW_FLOW_VORTICITY: "vorticity",
    VIEW_FLOW_VORTICITY_MAGNITUDE: "vorticity_magnitude", VIEW_OCCUPANCY: "occupancy",
}
LAYOUT_F32_3D = 0
LAYOUT_F32_3D_SOA3 = 1

# extension enums (smoke_b200_ext.h)
SOLVER_FIXED_CG = 0
SOLVER_JACOBI_PCG = 1
SOLVER_MG_FCG = 2
SOLVER_LEARNED_FCG = 3
REDUCTION_FP32 = 0
REDUCTION_FP64 = 1
SOLVE_CONVERGED = 0
SOLVE_ITERATION_CAP = 1
SOLVE_BREAKDOWN = 2
SOLVE_NOT_FINITE = 3
SOLVE_BARRIER_TIMEOUT = 4
SOLVE_NOT_RUN = 5
STAGE_FORCES = 0
STAGE_ADVECT_VELOCITY = 1
STAGE_PRESSURE = 2
STAGE_PROJECT = 3
STAGE_SCALARS = 4


class FlowFace(C.Structure):
    _fields_ = [("type", C.c_uint32), ("velocity_x", C.c_float), ("velocity_y", C.c_float), ("velocity_z", C.c_float), ("pressure", C.c_float)]


class FlowBoundary(C.Structure):
    _fields_ = [(n, FlowFace) for n in ("x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus")]


class ScalarFace(C.Structure):
    _fields_ = [("type", C.c_uint32), ("value", C.c_float)]


class ScalarBoundary(C.Structure):
    _fields_ = [(n, ScalarFace) for n in ("x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus")]


class Config(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("cell_size", C.c_float), ("dt", C.c_float),
        ("pressure_iterations", C.c_int32), ("ambient_temperature", C.c_float), ("buoyancy_density_factor", C.c_float),
        ("buoyancy_temperature_factor", C.c_float), ("vorticity_confinement", C.c_float), ("scalar_advection_mode", C.c_uint32),
        ("flow_boundary", FlowBoundary), ("density_boundary", ScalarBoundary), ("temperature_boundary", ScalarBoundary),
    ]


class CreateDesc(C.Structure):
    _fields_ = [("config", Config), ("stream", C.c_void_p), ("initial_density", C.c_float), ("initial_temperature", C.c_float)]


class ViewRequest(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("consumer_stream", C.c_void_p)]


class View(C.Structure):
    _fields_ = [
        ("layout", C.c_uint32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("row_stride_bytes", C.c_uint64),
        ("slice_stride_bytes", C.c_uint64), ("data0", C.c_void_p), ("data1", C.c_void_p), ("data2", C.c_void_p),
    ]


class SolverDesc(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("reduction", C.c_uint32), ("max_iterations", C.c_int32), ("tolerance", C.c_float), ("refinement", C.c_uint32), ("warm_start", C.c_uint32)]


class SolverStatus(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("passes", C.c_int32), ("status", C.c_uint32), ("flags", C.c_uint32), ("rhs_norm", C.c_double),
        ("relative_residual", C.c_double), ("true_relative_residual", C.c_double),
    ]


class LaunchTune(C.Structure):
    _fields_ = [("advect_tile", C.c_uint32), ("mg_wave", C.c_uint32), ("pcg_grid", C.c_uint32), ("pcg_regs", C.c_uint32)]


class TuneRecord(C.Structure):
    _fields_ = [("tune", LaunchTune), ("ms_per_step", C.c_float), ("iterations", C.c_uint32)]


TUNE_MAX_RECORDS = 16
TUNE_FORCE = 1
ADVECT_TILE_NAMES = ("flat", "32x8x1", "32x4x2", "16x4x4", "8x8x4")
MG_WAVE_NAMES = ("0.5 wave", "1 wave", "2 waves", "4 waves", "tile per block")
PCG_GRID_NAMES = ("all resident", "half", "quarter")
PCG_REGS_NAMES = ("uncapped", "64 registers")


class TuneReport(C.Structure):
    _fields_ = [
        ("chosen", LaunchTune), ("default_ms", C.c_float), ("chosen_ms", C.c_float), ("from_cache", C.c_uint32), ("record_count", C.c_uint32),
        ("records", TuneRecord * TUNE_MAX_RECORDS),
    ]


AXES = ("x", "y", "z")


def _flow_face(spec) -> FlowFace:
    if isinstance(spec, int):
        return FlowFace(spec, 0.0, 0.0, 0.0, 0.0)
    t, *rest = spec
    vals = list(rest) + [0.0] * (4 - len(rest))
    return FlowFace(t, *vals)


def _scalar_face(spec) -> ScalarFace:
    if isinstance(spec, int):
        return ScalarFace(spec, 0.0)
    return ScalarFace(spec[0], spec[1])


def make_config(nx, ny, nz, *, cell_size=None, dt=0.01, pressure_iterations=64, ambient=0.0, alpha=0.08, beta=0.97, epsilon=0.35,
                mode=LINEAR, flow=None, density=None, temperature=None) -> Config:
    """flow / density / temperature: dict face-name -> type or (type, values...), default closed no-slip walls
    and ZERO_FLUX scalars. cell_size defaults to 1/nx."""
    cfg = Config()
    cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
    cfg.cell_size = 1.0 / nx if cell_size is None else cell_size
    cfg.dt = dt
    cfg.pressure_iterations = pressure_iterations
    cfg.ambient_temperature = ambient
    cfg.buoyancy_density_factor = alpha
    cfg.buoyancy_temperature_factor = beta
    cfg.vorticity_confinement = epsilon
    cfg.scalar_advection_mode = mode
    names = ("x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus")
    for n in names:
        setattr(cfg.flow_boundary, n, _flow_face((flow or {}).get(n, NO_SLIP_WALL)))
        setattr(cfg.density_boundary, n, _scalar_face((density or {}).get(n, ZERO_FLUX)))
        setattr(cfg.temperature_boundary, n, _scalar_face((temperature or {}).get(n, (ZERO_FLUX, ambient))))
    return cfg


def face_shapes(cfg: Config):
    """numpy shapes (z, y, x) of the u, v, w face arrays."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    return (nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)


def cell_shape(cfg: Config):
    return (cfg.nz, cfg.ny, cfg.nx)
