"""Python binding of the smoke C ABI (ctypes), used by the tests, bench.py and the smoke() check.

`SmokeLibrary(path)` binds any library that exports the reference ABI (visual-simulation-of-smoke-3d.h): this
package's libsmoke_b200.so, or the reference's own libvisual-simulation-of-smoke.so, through the same calls.
`Simulation` owns one context. Device buffers are torch CUDA tensors; views come back as borrowed torch
tensors over the library's device memory.

The library must have been built (build_smoke.py); a missing library raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

import smoke_abi as abi

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIBRARY = os.path.join(HERE, "libsmoke_b200.so")


class SmokeError(RuntimeError):
    pass


def _check(code: int, what: str) -> None:
    if code != abi.RESULT_OK:
        raise SmokeError(f"{what} failed with result {code}")


class SmokeLibrary:
    """ctypes binding of one smoke library. extensions=True also binds the smoke_b200_ext.h entry points."""

    ABI = [
        ("smoke_simulation_create_context_cuda", [C.POINTER(abi.CreateDesc), C.POINTER(C.c_void_p)]),
        ("smoke_simulation_destroy_context_cuda", [C.c_void_p]),
        ("smoke_simulation_update_density_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_simulation_update_density_source_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_simulation_update_temperature_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_simulation_update_temperature_source_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_simulation_update_force_cuda", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        ("smoke_simulation_update_occupancy_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_simulation_update_solid_velocity_cuda", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        ("smoke_simulation_update_solid_temperature_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_simulation_step_cuda", [C.c_void_p]),
        ("smoke_simulation_get_view_cuda", [C.c_void_p, C.POINTER(abi.ViewRequest), C.POINTER(abi.View)]),
    ]
    EXTENSIONS = [
        ("smoke_b200_set_solver_cuda", [C.c_void_p, C.POINTER(abi.SolverDesc)]),
        ("smoke_b200_get_solver_status_cuda", [C.c_void_p, C.POINTER(abi.SolverStatus)]),
        ("smoke_b200_set_face_velocity_cuda", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        ("smoke_b200_get_face_velocity_cuda", [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
        ("smoke_b200_step_stages_cuda", [C.c_void_p, C.c_uint32]),
        ("smoke_b200_solve_pressure_cuda", [C.c_void_p]),
        ("smoke_b200_solve_pressure_eager_cuda", [C.c_void_p]),
        ("smoke_b200_batch_create_cuda", [C.POINTER(C.c_void_p), C.c_uint32, C.c_void_p, C.POINTER(C.c_void_p)]),
        ("smoke_b200_batch_step_cuda", [C.c_void_p]),
        ("smoke_b200_batch_destroy_cuda", [C.c_void_p]),
    ]

    def __init__(self, path: str = DEFAULT_LIBRARY, extensions: bool = True):
        if not os.path.exists(path):
            raise SmokeError(f"smoke library not found: {path} (build it with build_smoke.py)")
        self.path = path
        self.lib = C.CDLL(path)
        self.extensions = extensions
        for name, args in self.ABI + (self.EXTENSIONS if extensions else []):
            fn = getattr(self.lib, name)
            fn.argtypes = args
            fn.restype = C.c_int

    def symbols(self):
        return [n for n, _ in self.ABI + (self.EXTENSIONS if self.extensions else [])]


def _ptr(t):
    if t is None:
        return None
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
        raise SmokeError("device inputs must be contiguous torch CUDA tensors")
    return C.c_void_p(t.data_ptr())


class _DeviceArray:
    """__cuda_array_interface__ wrapper so torch can view library-owned device memory without a copy."""

    def __init__(self, ptr: int, shape, typestr: str = "<f4"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False), "version": 3, "strides": None}


def device_view(ptr: int, shape):
    import torch

    return torch.as_tensor(_DeviceArray(ptr, shape), device="cuda")


class Simulation:
    """One smoke context on `stream` (a torch.cuda.Stream, required to be non-default so the library and torch
    work are ordered on the same stream)."""

    def __init__(self, library: SmokeLibrary, config: abi.Config, stream, initial_density: float = 0.0, initial_temperature: float | None = None):
        self.L = library
        self.lib = library.lib
        self.config = config
        self.stream = stream
        desc = abi.CreateDesc()
        desc.config = config
        desc.stream = C.c_void_p(stream.cuda_stream)
        desc.initial_density = initial_density
        desc.initial_temperature = config.ambient_temperature if initial_temperature is None else initial_temperature
        handle = C.c_void_p()
        _check(self.lib.smoke_simulation_create_context_cuda(C.byref(desc), C.byref(handle)), "create_context")
        self.handle = handle

    # ------------------------------------------------------------------ lifetime
    def close(self):
        if self.handle is not None and self.handle.value:
            _check(self.lib.smoke_simulation_destroy_context_cuda(self.handle), "destroy_context")
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ inputs (device tensors or None)
    def update_density(self, t):
        _check(self.lib.smoke_simulation_update_density_cuda(self.handle, _ptr(t)), "update_density")

    def update_density_source(self, t):
        _check(self.lib.smoke_simulation_update_density_source_cuda(self.handle, _ptr(t)), "update_density_source")

    def update_temperature(self, t):
        _check(self.lib.smoke_simulation_update_temperature_cuda(self.handle, _ptr(t)), "update_temperature")

    def update_temperature_source(self, t):
        _check(self.lib.smoke_simulation_update_temperature_source_cuda(self.handle, _ptr(t)), "update_temperature_source")

    def update_force(self, x, y, z):
        _check(self.lib.smoke_simulation_update_force_cuda(self.handle, _ptr(x), _ptr(y), _ptr(z)), "update_force")

    def update_occupancy(self, t):
        _check(self.lib.smoke_simulation_update_occupancy_cuda(self.handle, _ptr(t)), "update_occupancy")

    def update_solid_velocity(self, x, y, z):
        _check(self.lib.smoke_simulation_update_solid_velocity_cuda(self.handle, _ptr(x), _ptr(y), _ptr(z)), "update_solid_velocity")

    def update_solid_temperature(self, t):
        _check(self.lib.smoke_simulation_update_solid_temperature_cuda(self.handle, _ptr(t)), "update_solid_temperature")

    def step(self):
        _check(self.lib.smoke_simulation_step_cuda(self.handle), "step")

    # ------------------------------------------------------------------ views
    def view_raw(self, kind: int, consumer_stream=None) -> abi.View:
        req = abi.ViewRequest(kind, C.c_void_p(consumer_stream.cuda_stream if consumer_stream is not None else 0))
        out = abi.View()
        _check(self.lib.smoke_simulation_get_view_cuda(self.handle, C.byref(req), C.byref(out)), "get_view")
        return out

    def view(self, kind: int):
        """Borrowed torch tensor(s) (z, y, x) over the view; valid until the next step/update/destroy."""
        v = self.view_raw(kind)
        shape = (v.nz, v.ny, v.nx)
        if v.layout == abi.LAYOUT_F32_3D:
            return device_view(v.data0, shape)
        return tuple(device_view(p, shape) for p in (v.data0, v.data1, v.data2))

    def snapshot(self, kinds=None):
        """Host numpy copies of views, keyed by name (vector views split into name_x/_y/_z)."""
        import torch

        out = {}
        with torch.cuda.stream(self.stream):  # copies ordered after the library's work on its stream
            for kind in kinds if kinds is not None else range(15):
                v = self.view(kind)
                name = abi.VIEW_NAMES[kind]
                if isinstance(v, tuple):
                    for ax, t in zip(abi.AXES, v):
                        out[f"{name}_{ax}"] = t.clone()
                else:
                    out[name] = v.clone()
        self.stream.synchronize()
        return {k: t.cpu().numpy() for k, t in out.items()}

    # ------------------------------------------------------------------ extensions (libsmoke_b200.so only)
    def set_solver(self, mode=abi.SOLVER_JACOBI_PCG, reduction=abi.REDUCTION_FP64, max_iterations=500, tolerance=1e-5, refinement=0, warm_start=False):
        d = abi.SolverDesc(mode, reduction, max_iterations, tolerance, refinement, 1 if warm_start else 0)
        _check(self.lib.smoke_b200_set_solver_cuda(self.handle, C.byref(d)), "set_solver")

    def solver_status(self) -> abi.SolverStatus:
        s = abi.SolverStatus()
        _check(self.lib.smoke_b200_get_solver_status_cuda(self.handle, C.byref(s)), "get_solver_status")
        return s

    def set_face_velocity(self, u, v, w):
        _check(self.lib.smoke_b200_set_face_velocity_cuda(self.handle, _ptr(u), _ptr(v), _ptr(w)), "set_face_velocity")

    def face_velocity(self, which: int = 0):
        pu, pv, pw = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _check(self.lib.smoke_b200_get_face_velocity_cuda(self.handle, which, C.byref(pu), C.byref(pv), C.byref(pw)), "get_face_velocity")
        su, sv, sw = abi.face_shapes(self.config)
        return device_view(pu.value, su), device_view(pv.value, sv), device_view(pw.value, sw)

    def face_velocity_host(self, which: int = 0):
        """Host numpy copies of the face velocities (ordered after the library's work)."""
        import torch

        with torch.cuda.stream(self.stream):
            t = [x.clone() for x in self.face_velocity(which)]
        self.stream.synchronize()
        return [x.cpu().numpy() for x in t]

    def step_stages(self, last_stage: int):
        _check(self.lib.smoke_b200_step_stages_cuda(self.handle, last_stage), "step_stages")

    def solve_pressure(self, eager: bool = False):
        """Pressure solve of the current right-hand side (eager: every kernel launched directly, host-driven loop)."""
        fn = self.lib.smoke_b200_solve_pressure_eager_cuda if eager else self.lib.smoke_b200_solve_pressure_cuda
        _check(fn(self.handle), "solve_pressure")


class Batch:
    """Several Simulations advanced by one graph launch (smoke_b200_batch_*_cuda). Create it after the members are
    configured (solver, occupancy); `stream` (a torch.cuda.Stream, optional) runs the batch graph."""

    def __init__(self, sims, stream=None):
        self.sims = list(sims)
        self.lib = self.sims[0].lib
        handles = (C.c_void_p * len(self.sims))(*[s.handle.value for s in self.sims])
        out = C.c_void_p()
        _check(self.lib.smoke_b200_batch_create_cuda(handles, len(self.sims), C.c_void_p(stream.cuda_stream if stream is not None else 0), C.byref(out)), "batch_create")
        self.handle = out

    def step(self):
        _check(self.lib.smoke_b200_batch_step_cuda(self.handle), "batch_step")

    def close(self):
        if self.handle is not None and self.handle.value:
            _check(self.lib.smoke_b200_batch_destroy_cuda(self.handle), "batch_destroy")
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
