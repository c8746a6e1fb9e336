"""CPU checks of the drop-in boundary (no GPU needed):

 - the ctypes mirror (smoke_abi.py) has the sizes and field offsets a C compiler gives the structs of
   include/visual-simulation-of-smoke-3d.h and include/smoke_b200_ext.h (the reference layout,
   visual-simulation-of-smoke-3d.h:22-154);
 - libsmoke_b200.so loads and exports every function the headers declare;
 - the host-side checks that precede any CUDA call behave like the reference's (backend-cuda.cu:1835-1863,
   2063-2083): an invalid configuration fails with BACKEND_FAILURE, destroy(NULL) succeeds, step(NULL) and
   get_view(NULL) fail.
"""
import ctypes as C
import os
import re
import subprocess

import pytest

import smoke_abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
HEADERS = [os.path.join(INCLUDE, h) for h in ("visual-simulation-of-smoke-3d.h", "smoke_b200_ext.h")]

# (C type, ctypes class, fields whose offsets are compared)
STRUCTS = [
    ("SmokeSimulationFlowBoundaryFaceDesc", abi.FlowFace, ["type", "velocity_x", "pressure"]),
    ("SmokeSimulationFlowBoundaryConfig", abi.FlowBoundary, ["x_minus", "y_plus", "z_plus"]),
    ("SmokeSimulationScalarBoundaryFaceDesc", abi.ScalarFace, ["type", "value"]),
    ("SmokeSimulationConfig", abi.Config, ["nx", "cell_size", "pressure_iterations", "scalar_advection_mode", "flow_boundary", "density_boundary", "temperature_boundary"]),
    ("SmokeSimulationContextCreateDesc", abi.CreateDesc, ["config", "stream", "initial_density", "initial_temperature"]),
    ("SmokeSimulationViewRequest", abi.ViewRequest, ["kind", "consumer_stream"]),
    ("SmokeSimulationView", abi.View, ["layout", "nx", "row_stride_bytes", "slice_stride_bytes", "data0", "data2"]),
    ("SmokeB200SolverDesc", abi.SolverDesc, ["mode", "reduction", "max_iterations", "tolerance", "refinement", "warm_start"]),
    ("SmokeB200SolverStatus", abi.SolverStatus, ["iterations", "status", "rhs_norm", "true_relative_residual"]),
    ("SmokeB200LaunchTune", abi.LaunchTune, ["advect_tile", "mg_wave", "pcg_grid", "pcg_regs"]),
    ("SmokeB200TuneRecord", abi.TuneRecord, ["tune", "ms_per_step", "iterations"]),
    ("SmokeB200TuneReport", abi.TuneReport, ["chosen", "default_ms", "chosen_ms", "from_cache", "record_count", "records"]),
]


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    """sizeof/offsetof of every struct above, printed by a C program compiled against the headers."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "visual-simulation-of-smoke-3d.h"', '#include "smoke_b200_ext.h"', "int main(void) {"]
    for ctype, _, fields in STRUCTS:
        lines.append(f'printf("{ctype} size %zu\\n", sizeof({ctype}));')
        for f in fields:
            lines.append(f'printf("{ctype} {f} %zu\\n", offsetof({ctype}, {f}));')
    lines += ["return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-std=c11", f"-I{INCLUDE}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for ln in out.splitlines():
        name, key, value = ln.split()
        table[(name, key)] = int(value)
    return table


@pytest.mark.parametrize("ctype,cls,fields", STRUCTS, ids=[s[0] for s in STRUCTS])
def test_struct_layout_matches_c_header(c_layout, ctype, cls, fields):
    assert C.sizeof(cls) == c_layout[(ctype, "size")]
    for f in fields:
        assert getattr(cls, f).offset == c_layout[(ctype, f)], f


def test_reference_struct_sizes():
    # the reference's layout on x86-64 (visual-simulation-of-smoke-3d.h:66-92, 96-101, 116-154)
    assert C.sizeof(abi.Config) == 260
    assert C.sizeof(abi.CreateDesc) == 280
    assert abi.CreateDesc.stream.offset == 264
    assert C.sizeof(abi.View) == 56


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        names += re.findall(r"SMOKE_SIMULATION_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def library():
    import build_smoke

    path = build_smoke.build()  # incremental; a no-op when the library is current
    return C.CDLL(path)


def test_headers_declare_the_reference_abi():
    names = declared_functions()
    for sym in ("smoke_simulation_create_context_cuda", "smoke_simulation_destroy_context_cuda", "smoke_simulation_step_cuda", "smoke_simulation_get_view_cuda",
                "smoke_simulation_update_occupancy_cuda", "smoke_simulation_update_force_cuda"):
        assert sym in names
    assert len(names) >= 12 + 10


def test_library_exports_every_declared_function(library):
    missing = [n for n in declared_functions() if not hasattr(library, n)]
    assert missing == []


def test_python_binding_covers_the_library(library):
    import smoke_b200

    bound = {n for n, _ in smoke_b200.SmokeLibrary.ABI + smoke_b200.SmokeLibrary.EXTENSIONS}
    assert bound <= set(declared_functions())


def _create(library, cfg):
    desc = abi.CreateDesc()
    desc.config = cfg
    handle = C.c_void_p()
    fn = library.smoke_simulation_create_context_cuda
    fn.argtypes = [C.POINTER(abi.CreateDesc), C.POINTER(C.c_void_p)]
    fn.restype = C.c_int
    return fn(C.byref(desc), C.byref(handle)), handle


@pytest.mark.parametrize("bad", ["nx0", "negative_ny", "dt0", "cell0", "iterations0", "periodic_mismatch", "too_large", "bad_flow_type"])
def test_invalid_config_fails_before_any_device_work(library, bad):
    cfg = abi.make_config(8, 8, 8)
    if bad == "nx0":
        cfg.nx = 0
    elif bad == "negative_ny":
        cfg.ny = -4
    elif bad == "dt0":
        cfg.dt = 0.0
    elif bad == "cell0":
        cfg.cell_size = 0.0
    elif bad == "iterations0":
        cfg.pressure_iterations = 0
    elif bad == "periodic_mismatch":  # a periodic face needs a periodic partner (backend-cuda.cu:1844-1856)
        cfg.flow_boundary.x_minus.type = abi.PERIODIC
    elif bad == "too_large":
        cfg.nx = cfg.ny = cfg.nz = 2048
    elif bad == "bad_flow_type":
        cfg.flow_boundary.y_plus.type = 17
    code, handle = _create(library, cfg)
    assert code == abi.RESULT_BACKEND_FAILURE
    assert not handle.value


def test_null_arguments(library):
    library.smoke_simulation_destroy_context_cuda.argtypes = [C.c_void_p]
    library.smoke_simulation_step_cuda.argtypes = [C.c_void_p]
    library.smoke_simulation_get_view_cuda.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    library.smoke_simulation_create_context_cuda.argtypes = [C.c_void_p, C.c_void_p]
    assert library.smoke_simulation_destroy_context_cuda(None) == abi.RESULT_OK
    assert library.smoke_simulation_step_cuda(None) == abi.RESULT_BACKEND_FAILURE
    assert library.smoke_simulation_get_view_cuda(None, None, None) == abi.RESULT_BACKEND_FAILURE
    assert library.smoke_simulation_create_context_cuda(None, None) == abi.RESULT_BACKEND_FAILURE
    for name in ("smoke_b200_set_solver_cuda", "smoke_b200_get_solver_status_cuda"):
        fn = getattr(library, name)
        fn.argtypes = [C.c_void_p, C.c_void_p]
        assert fn(None, None) == abi.RESULT_BACKEND_FAILURE
    for name in ("smoke_b200_set_launch_tune_cuda", "smoke_b200_get_launch_tune_cuda"):
        fn = getattr(library, name)
        fn.argtypes = [C.c_void_p, C.c_void_p]
        assert fn(None, None) == abi.RESULT_BACKEND_FAILURE
    library.smoke_b200_autotune_cuda.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
    assert library.smoke_b200_autotune_cuda(None, 0, 0, None) == abi.RESULT_BACKEND_FAILURE
    for name in ("smoke_b200_solve_pressure_cuda", "smoke_b200_solve_pressure_eager_cuda", "smoke_b200_step_stages_cuda"):
        fn = getattr(library, name)
        assert fn(None, 0) if name.endswith("stages_cuda") else fn(None)  # nonzero: BACKEND_FAILURE


def test_noalloc_limit_is_reported(library):
    library.smoke_b200_noalloc_max_cells.restype = C.c_ulonglong
    assert library.smoke_b200_noalloc_max_cells() == 64 ** 3


def _bind_noalloc(library):
    fn = library.smoke_b200_solve_pressure_noalloc_cuda
    fn.argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(abi.SolverDesc), C.c_void_p, C.POINTER(abi.SolverStatus)]
    fn.restype = C.c_int
    library.smoke_b200_last_error.restype = C.c_char_p
    return fn


@pytest.mark.parametrize("bad", ["periodic_one_side", "dt0", "cell0", "bad_flow_type", "bad_scalar_type"])
def test_noalloc_refuses_the_configs_context_creation_refuses(library, bad):
    """The allocation-free solve validates its configuration as context creation does (backend-cuda.cu:1835-1863),
    before any device work, so these refusals need no GPU. Dummy non-NULL pointers are never dereferenced."""
    solve = _bind_noalloc(library)
    cfg = abi.make_config(8, 8, 8)
    if bad == "periodic_one_side":
        cfg.flow_boundary.z_plus.type = abi.PERIODIC
    elif bad == "dt0":
        cfg.dt = 0.0
    elif bad == "cell0":
        cfg.cell_size = -1.0
    elif bad == "bad_flow_type":
        cfg.flow_boundary.x_plus.type = 9
    elif bad == "bad_scalar_type":
        cfg.density_boundary.y_minus.type = 9
    assert _create(library, cfg)[0] == abi.RESULT_BACKEND_FAILURE
    fake = C.c_void_p(0x1000)
    rc = solve(C.byref(cfg), None, fake, fake, None, None, None)
    assert rc == abi.RESULT_BACKEND_FAILURE
    assert library.smoke_b200_last_error().startswith(b"invalid configuration")


@pytest.mark.parametrize("mode", ["multigrid", "learned", "refinement", "jacobi_no_tolerance"])
def test_noalloc_refuses_solver_modes_it_cannot_run(library, mode):
    """Only the fixed-count CG and Jacobi-PCG run without a context; the multigrid and learned modes are refused
    with the reason, as is an out-of-range refinement count."""
    solve = _bind_noalloc(library)
    cfg = abi.make_config(8, 8, 8)
    desc = abi.SolverDesc(abi.SOLVER_JACOBI_PCG, abi.REDUCTION_FP64, 100, 1e-5, 1, 0)
    if mode == "multigrid":
        desc.mode = abi.SOLVER_MG_FCG
    elif mode == "learned":
        desc.mode = abi.SOLVER_LEARNED_FCG
    elif mode == "refinement":
        desc.refinement = 65
    elif mode == "jacobi_no_tolerance":
        desc.tolerance = 0.0
    fake = C.c_void_p(0x1000)
    rc = solve(C.byref(cfg), None, fake, fake, C.byref(desc), None, None)
    assert rc == abi.RESULT_BACKEND_FAILURE
    assert library.smoke_b200_last_error().startswith(b"invalid solver description")
