"""TEST INFRASTRUCTURE -- numpy front end of the oracle (smoke_oracle.c), a CPU restatement of the reference step.

Only tests/, the smoke() check and bench.py's CPU-baseline leg use this module; the product library never
does. `OracleState` holds every field of a context as numpy arrays (z, y, x); `step` runs stages of the step
in FP32 ("mirror") or FP64 ("truth").
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "visual-simulation-of-smoke_b200"))
import smoke_abi as abi  # noqa: E402

sys.path.insert(0, HERE)
import build_oracle as oracle_build  # noqa: E402

FIELDS = ["u", "v", "w", "temp_u", "temp_v", "temp_w", "density", "temperature", "density_source", "temperature_source", "force_x", "force_y", "force_z",
          "solid_velocity_x", "solid_velocity_y", "solid_velocity_z", "solid_temperature", "occupancy", "pressure", "pressure_rhs", "centered_x", "centered_y",
          "centered_z", "velocity_magnitude", "vorticity_x", "vorticity_y", "vorticity_z", "vorticity_magnitude", "divergence"]


class _Fields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in FIELDS]


class OracleSolver(C.Structure):
    _fields_ = [("mode", C.c_int32), ("max_iterations", C.c_int32), ("tolerance", C.c_double), ("iterations", C.c_int32), ("reserved", C.c_int32),
                ("relative_residual", C.c_double)]


_LIBS = {}


def library(bits: int):
    if bits not in _LIBS:
        path = oracle_build.oracle_path(bits)
        if not os.path.exists(path):
            oracle_build.build_oracle()
        lib = C.CDLL(path)
        p = f"oracle{bits}_"
        getattr(lib, p + "step").argtypes = [C.POINTER(abi.Config), C.POINTER(_Fields), C.POINTER(OracleSolver), C.c_int, C.c_int]
        getattr(lib, p + "step").restype = C.c_int
        getattr(lib, p + "apply_pressure_operator").argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.c_void_p]
        getattr(lib, p + "pressure_diagonal").argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_void_p]
        getattr(lib, p + "pressure_diagonal").restype = C.c_longlong
        getattr(lib, p + "solve_pressure").argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(OracleSolver)]
        getattr(lib, p + "sample").argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        getattr(lib, p + "sample").restype = C.c_double
        getattr(lib, p + "monotonic_cubic").argtypes = [C.c_double] * 5
        getattr(lib, p + "monotonic_cubic").restype = C.c_double
        getattr(lib, p + "real_bytes").restype = C.c_int
        _LIBS[bits] = lib
    return _LIBS[bits]


class OracleState:
    """All fields of one scene. Face arrays u (nz,ny,nx+1), v (nz,ny+1,nx), w (nz+1,ny,nx); cells (nz,ny,nx)."""

    def __init__(self, cfg: abi.Config, bits: int = 32, initial_density: float = 0.0, initial_temperature: float | None = None):
        self.cfg = cfg
        self.bits = bits
        self.dtype = np.float32 if bits == 32 else np.float64
        cs = abi.cell_shape(cfg)
        su, sv, sw = abi.face_shapes(cfg)
        z = lambda s: np.zeros(s, self.dtype)  # noqa: E731
        self.arrays = {"u": z(su), "v": z(sv), "w": z(sw), "temp_u": z(su), "temp_v": z(sv), "temp_w": z(sw)}
        for n in FIELDS[6:]:
            self.arrays[n] = np.zeros(cs, np.uint8) if n == "occupancy" else z(cs)
        self.arrays["density"][:] = initial_density
        self.arrays["temperature"][:] = cfg.ambient_temperature if initial_temperature is None else initial_temperature
        self.arrays["solid_temperature"][:] = cfg.ambient_temperature

    def __getitem__(self, k):
        return self.arrays[k]

    def set(self, name, values):
        a = self.arrays[name]
        a[...] = np.asarray(values, dtype=a.dtype).reshape(a.shape)

    def copy(self):
        o = OracleState.__new__(OracleState)
        o.cfg, o.bits, o.dtype = self.cfg, self.bits, self.dtype
        o.arrays = {k: v.copy() for k, v in self.arrays.items()}
        return o

    def _struct(self):
        f = _Fields()
        for n in FIELDS:
            a = self.arrays[n]
            assert a.flags.c_contiguous
            setattr(f, n, a.ctypes.data)
        return f

    def step(self, first: int = 0, last: int = 5, mode: int = 0, max_iterations: int = 500, tolerance: float = 1e-5) -> OracleSolver:
        """Stages: 0 forces, 1 velocity advection, 2 pressure, 3 projection, 4 scalars, 5 views.
        mode 0: the reference's fixed-iteration CG; 1: Jacobi PCG to `tolerance`."""
        lib = library(self.bits)
        s = OracleSolver(mode, max_iterations, tolerance, 0, 0, 0.0)
        f = self._struct()
        rc = getattr(lib, f"oracle{self.bits}_step")(C.byref(self.cfg), C.byref(f), C.byref(s), first, last)
        if rc != 0:
            raise RuntimeError(f"oracle step failed: {rc}")
        return s


def apply_operator(cfg: abi.Config, occupancy: np.ndarray, x: np.ndarray) -> np.ndarray:
    """A x for the pressure operator of `cfg` and `occupancy` (FP64)."""
    x64 = np.ascontiguousarray(x, dtype=np.float64)
    occ = np.ascontiguousarray(occupancy, dtype=np.uint8)
    out = np.zeros_like(x64)
    library(64).oracle64_apply_pressure_operator(C.byref(cfg), occ.ctypes.data, x64.ctypes.data, out.ctypes.data)
    return out


def pressure_diagonal(cfg: abi.Config, occupancy: np.ndarray):
    occ = np.ascontiguousarray(occupancy, dtype=np.uint8)
    d = np.zeros(occ.shape, np.float64)
    anchor = library(64).oracle64_pressure_diagonal(C.byref(cfg), occ.ctypes.data, d.ctypes.data)
    return d, int(anchor)


def relative_residual(cfg: abi.Config, occupancy: np.ndarray, b: np.ndarray, x: np.ndarray) -> float:
    """||b - A x|| / ||b|| in FP64 (0 when b = 0)."""
    b64 = np.asarray(b, np.float64)
    bn = np.linalg.norm(b64)
    if bn == 0:
        return 0.0
    return float(np.linalg.norm(b64 - apply_operator(cfg, occupancy, x)) / bn)


def solve_pressure(cfg: abi.Config, occupancy: np.ndarray, b: np.ndarray, bits: int = 64, mode: int = 1, max_iterations: int = 5000, tolerance: float = 1e-10):
    dt = np.float32 if bits == 32 else np.float64
    bb = np.ascontiguousarray(b, dtype=dt)
    x = np.zeros_like(bb)
    occ = np.ascontiguousarray(occupancy, dtype=np.uint8)
    s = OracleSolver(mode, max_iterations, tolerance, 0, 0, 0.0)
    getattr(library(bits), f"oracle{bits}_solve_pressure")(C.byref(cfg), occ.ctypes.data, bb.ctypes.data, x.ctypes.data, C.byref(s))
    return x, s


def sample(cfg: abi.Config, field: np.ndarray, kind: int, cubic: bool, x: float, y: float, z: float, bits: int = 32, density_bc: bool = True) -> float:
    dt = np.float32 if bits == 32 else np.float64
    f = np.ascontiguousarray(field, dtype=dt)
    return getattr(library(bits), f"oracle{bits}_sample")(C.byref(cfg), f.ctypes.data, kind, int(cubic), int(density_bc), x, y, z)


def monotonic_cubic(p0, p1, p2, p3, t, bits: int = 32) -> float:
    return getattr(library(bits), f"oracle{bits}_monotonic_cubic")(p0, p1, p2, p3, t)
