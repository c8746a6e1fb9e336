// Validation of a SmokeSimulationConfig, shared by context creation (context.cpp) and the allocation-free solve
// (noalloc.cu), so both refuse exactly the same configurations.
//
// Reference behaviour: backend-cuda.cu:1835-1863 (positive extents, cell size, time step and iteration count;
// boundary types in range; a periodic face only opposite another periodic face), plus the 32-bit index range this
// library's kernels use.
#pragma once

#include <cstdint>

#include "visual-simulation-of-smoke-3d.h"

namespace smoke_b200 {

inline bool valid_flow_axis(const SmokeSimulationFlowBoundaryFaceDesc& a, const SmokeSimulationFlowBoundaryFaceDesc& b) {
    auto ok = [](uint32_t t) { return t <= SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC; };
    if (!ok(a.type) || !ok(b.type)) return false;
    return (a.type == SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC) == (b.type == SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC);
}

inline bool valid_scalar_axis(const SmokeSimulationScalarBoundaryFaceDesc& a, const SmokeSimulationScalarBoundaryFaceDesc& b) {
    auto ok = [](uint32_t t) { return t <= SMOKE_SIMULATION_SCALAR_BOUNDARY_PERIODIC; };
    if (!ok(a.type) || !ok(b.type)) return false;
    return (a.type == SMOKE_SIMULATION_SCALAR_BOUNDARY_PERIODIC) == (b.type == SMOKE_SIMULATION_SCALAR_BOUNDARY_PERIODIC);
}

inline bool valid_config(const SmokeSimulationConfig& c) {
    if (c.nx <= 0 || c.ny <= 0 || c.nz <= 0 || !(c.cell_size > 0.0f) || !(c.dt > 0.0f) || c.pressure_iterations <= 0) return false;
    const auto& f = c.flow_boundary;
    const auto& d = c.density_boundary;
    const auto& t = c.temperature_boundary;
    if (!valid_flow_axis(f.x_minus, f.x_plus) || !valid_flow_axis(f.y_minus, f.y_plus) || !valid_flow_axis(f.z_minus, f.z_plus)) return false;
    if (!valid_scalar_axis(d.x_minus, d.x_plus) || !valid_scalar_axis(d.y_minus, d.y_plus) || !valid_scalar_axis(d.z_minus, d.z_plus)) return false;
    if (!valid_scalar_axis(t.x_minus, t.x_plus) || !valid_scalar_axis(t.y_minus, t.y_plus) || !valid_scalar_axis(t.z_minus, t.z_plus)) return false;
    const uint64_t nx = c.nx, ny = c.ny, nz = c.nz;
    const uint64_t biggest = (nx + 1) * (ny + 1) * (nz + 1);
    return biggest < (1ull << 31);
}

}  // namespace smoke_b200
