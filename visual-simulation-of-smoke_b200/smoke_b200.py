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

import numpy as np

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
        ("smoke_b200_batch_member_times_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_b200_set_launch_tune_cuda", [C.c_void_p, C.POINTER(abi.LaunchTune)]),
        ("smoke_b200_get_launch_tune_cuda", [C.c_void_p, C.POINTER(abi.LaunchTune)]),
        ("smoke_b200_autotune_cuda", [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(abi.TuneReport)]),
        ("smoke_b200_net_create_cuda", [C.c_uint32, C.POINTER(C.c_void_p)]),
        ("smoke_b200_net_destroy_cuda", [C.c_void_p]),
        ("smoke_b200_net_get_parameters_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_b200_net_set_parameters_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_b200_net_apply_cuda", [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        ("smoke_b200_net_gradient_cuda", [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
        ("smoke_b200_net_train_cuda", [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.POINTER(C.c_double), C.c_void_p]),
        ("smoke_b200_set_preconditioner_net_cuda", [C.c_void_p, C.c_void_p]),
        ("smoke_b200_set_learned_iterations_cuda", [C.c_void_p, C.c_uint32]),
        ("smoke_b200_apply_operator_cuda", [C.c_void_p, C.c_void_p, C.c_void_p]),
        ("smoke_b200_apply_multigrid_cuda", [C.c_void_p, C.c_void_p, C.c_void_p]),
        ("smoke_b200_conv3d_cuda", [C.c_int] * 5 + [C.c_void_p] * 3 + [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
        ("smoke_b200_test_barrier_timeout_cuda", [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(abi.SolverStatus)]),
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
        if extensions and hasattr(self.lib, "smoke_b200_net_parameter_count"):
            self.lib.smoke_b200_net_parameter_count.argtypes = []
            self.lib.smoke_b200_net_parameter_count.restype = C.c_uint32

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
        d = abi.SolverDesc(mode, reduction, max_iterations, tolerance, refinement, int(warm_start))
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

    def set_launch_tune(self, advect_tile: int = 0, mg_wave: int = 1, pcg_grid: int = 0, pcg_regs: int = 0):
        t = _tune_struct({"advect_tile": advect_tile, "mg_wave": mg_wave, "pcg_grid": pcg_grid, "pcg_regs": pcg_regs})
        _check(self.lib.smoke_b200_set_launch_tune_cuda(self.handle, C.byref(t)), "set_launch_tune")

    def launch_tune(self) -> dict:
        t = abi.LaunchTune()
        _check(self.lib.smoke_b200_get_launch_tune_cuda(self.handle, C.byref(t)), "get_launch_tune")
        return _tune_dict(t)

    def autotune(self, steps: int = 4, force: bool = False) -> dict:
        """Times the step under candidate launch shapes, keeps the fastest (state restored afterwards)."""
        rep = abi.TuneReport()
        flags = abi.TUNE_FORCE if force else 0
        _check(self.lib.smoke_b200_autotune_cuda(self.handle, steps, flags, C.byref(rep)), "autotune")
        records = [dict(_tune_dict(r.tune), ms_per_step=r.ms_per_step, iterations=r.iterations) for r in rep.records[: rep.record_count]]
        return {"chosen": _tune_dict(rep.chosen), "default_ms": rep.default_ms, "chosen_ms": rep.chosen_ms, "from_cache": bool(rep.from_cache), "records": records}

    def apply_operator(self, x):
        """A x with the context's pressure matrix (x: float32 CUDA tensor of nz x ny x nx values)."""
        import torch

        out = torch.empty_like(x)
        with torch.cuda.stream(self.stream):
            _check(self.lib.smoke_b200_apply_operator_cuda(self.handle, _ptr(x), _ptr(out)), "apply_operator")
        return out

    def apply_multigrid(self, r):
        """V(r), one V-cycle of the multigrid preconditioner (r: float32 CUDA tensor of nz x ny x nx values)."""
        import torch

        out = torch.empty_like(r)
        with torch.cuda.stream(self.stream):
            _check(self.lib.smoke_b200_apply_multigrid_cuda(self.handle, _ptr(r), _ptr(out)), "apply_multigrid")
        return out

    def set_preconditioner_net(self, net: "Net"):
        _check(self.lib.smoke_b200_set_preconditioner_net_cuda(self.handle, net.handle), "set_preconditioner_net")

    def set_learned_iterations(self, count: int):
        """The network corrects the first `count` iterations of each refinement pass (0: all)."""
        _check(self.lib.smoke_b200_set_learned_iterations_cuda(self.handle, count), "set_learned_iterations")

    def solve_pressure(self, eager: bool = False):
        """Pressure solve of the current right-hand side (eager: every kernel launched directly, host-driven loop)."""
        fn = self.lib.smoke_b200_solve_pressure_eager_cuda if eager else self.lib.smoke_b200_solve_pressure_cuda
        _check(fn(self.handle), "solve_pressure")


class Net:
    """The learned preconditioner's network (smoke_b200_net_*_cuda). Device inputs are contiguous torch CUDA tensors;
    every call synchronises the current torch stream."""

    def __init__(self, library: SmokeLibrary, seed: int = 0):
        self.L = library
        self.lib = library.lib
        self.handle = C.c_void_p()
        _check(self.lib.smoke_b200_net_create_cuda(seed, C.byref(self.handle)), "net_create")

    @property
    def parameter_count(self) -> int:
        return int(self.lib.smoke_b200_net_parameter_count())

    def close(self):
        if self.handle:
            self.lib.smoke_b200_net_destroy_cuda(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _stream():
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def parameters(self):
        import numpy as np

        out = np.zeros(self.parameter_count, np.float32)
        _check(self.lib.smoke_b200_net_get_parameters_cuda(self.handle, out.ctypes.data_as(C.c_void_p)), "net_get_parameters")
        return out

    def set_parameters(self, values):
        import numpy as np

        v = np.ascontiguousarray(values, np.float32)
        if v.size != self.parameter_count:
            raise SmokeError(f"expected {self.parameter_count} parameters, got {v.size}")
        _check(self.lib.smoke_b200_net_set_parameters_cuda(self.handle, v.ctypes.data_as(C.c_void_p)), "net_set_parameters")

    def apply(self, rhs, occupancy):
        """N(rhs) for one volume: rhs float32 [nz, ny, nx], occupancy uint8 [nz, ny, nx] (CUDA tensors)."""
        import torch

        nz, ny, nx = rhs.shape
        out = torch.empty_like(rhs)
        _check(self.lib.smoke_b200_net_apply_cuda(self.handle, nx, ny, nz, _ptr(rhs), _ptr(occupancy), _ptr(out), self._stream()), "net_apply")
        return out

    def gradient(self, rhs, occupancy, target):
        """(loss, gradient) of one sample; the gradient in parameter layout (numpy float32)."""
        import numpy as np

        nz, ny, nx = rhs.shape
        g = np.zeros(self.parameter_count, np.float32)
        loss = C.c_double()
        _check(self.lib.smoke_b200_net_gradient_cuda(self.handle, nx, ny, nz, _ptr(rhs), _ptr(occupancy), _ptr(target), g.ctypes.data_as(C.c_void_p), C.byref(loss), self._stream()), "net_gradient")
        return loss.value, g

    def train_step(self, rhs, occupancy, target, learning_rate: float) -> float:
        """One Adam step on a batch: rhs / target float32 [count, nz, ny, nx], occupancy uint8 of the same shape."""
        count, nz, ny, nx = rhs.shape
        loss = C.c_double()
        _check(self.lib.smoke_b200_net_train_cuda(self.handle, nx, ny, nz, count, _ptr(rhs), _ptr(occupancy), _ptr(target), float(learning_rate), C.byref(loss), self._stream()), "net_train")
        return loss.value


def _tune_dict(t: abi.LaunchTune) -> dict:
    return {"advect_tile": t.advect_tile, "mg_wave": t.mg_wave, "pcg_grid": t.pcg_grid, "pcg_regs": t.pcg_regs}


def _tune_struct(d: dict) -> abi.LaunchTune:
    t = abi.LaunchTune()
    t.advect_tile = d.get("advect_tile", 0)
    t.mg_wave = d.get("mg_wave", 1)
    t.pcg_grid = d.get("pcg_grid", 0)
    t.pcg_regs = d.get("pcg_regs", 0)
    return t


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

    def member_times(self):
        """Milliseconds from the start of the last batch step to the end of each member's step inside it."""
        out = (C.c_float * len(self.sims))()
        _check(self.lib.smoke_b200_batch_member_times_cuda(self.handle, out), "batch_member_times")
        return np.array(out[:], dtype=np.float64)

    def close(self):
        if self.handle is not None and self.handle.value:
            _check(self.lib.smoke_b200_batch_destroy_cuda(self.handle), "batch_destroy")
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
