/*
 * C ABI of the smoke step (Fedkiw, Stam & Jensen 2001), re-declared for the B200 library libsmoke_b200.so.
 *
 * Every enum value, struct layout and function signature here is the one the reference library
 * exports, so a program built against the reference header links and runs against this library
 * unchanged (reference: visual-simulation-of-smoke-3d.h:1-162). The layouts are pinned by
 * static_asserts in visual-simulation-of-smoke_b200/csrc/context.cpp and by tests/test_abi_host.py.
 *
 * Semantics shared with the reference (backend-cuda.cu:1833-2282):
 *   - every call enqueues work on the context stream and returns without synchronising,
 *     except create (which may synchronise once) and destroy (which synchronises first);
 *   - update_* copy from caller DEVICE pointers (device-to-device); NULL means zero, except
 *     update_solid_temperature(NULL), which means "ambient temperature everywhere";
 *   - views are borrowed device pointers, valid until the next step/update/destroy;
 *   - errors: OK, OUT_OF_MEMORY (host allocation failed), BACKEND_FAILURE (everything else).
 * Extensions that the reference does not have live in smoke_b200_ext.h.
 */
#ifndef VISUAL_SIMULATION_OF_SMOKE_3D_H
#define VISUAL_SIMULATION_OF_SMOKE_3D_H

#include <stdint.h>

#if defined(_WIN32)
#  if defined(VISUAL_SIMULATION_OF_SMOKE_BUILD_SHARED)
#    define SMOKE_SIMULATION_API __declspec(dllexport)
#  else
#    define SMOKE_SIMULATION_API __declspec(dllimport)
#  endif
#elif defined(__GNUC__) || defined(__clang__)
#  define SMOKE_SIMULATION_API __attribute__((visibility("default")))
#else
#  define SMOKE_SIMULATION_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Result codes (reference header :22-26). */
typedef enum SmokeSimulationResult {
    SMOKE_SIMULATION_RESULT_OK              = 0,
    SMOKE_SIMULATION_RESULT_OUT_OF_MEMORY   = 1,
    SMOKE_SIMULATION_RESULT_BACKEND_FAILURE = 2,
} SmokeSimulationResult;

/* Velocity boundary condition of one domain face (reference header :28-33). PERIODIC must be set on
 * both faces of an axis or on neither. */
typedef enum SmokeSimulationFlowBoundaryType {
    SMOKE_SIMULATION_FLOW_BOUNDARY_NO_SLIP_WALL   = 0,
    SMOKE_SIMULATION_FLOW_BOUNDARY_FREE_SLIP_WALL = 1,
    SMOKE_SIMULATION_FLOW_BOUNDARY_OUTFLOW        = 2,
    SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC       = 3,
} SmokeSimulationFlowBoundaryType;

/* Boundary condition of a transported scalar (density or temperature) on one face (:35-39). */
typedef enum SmokeSimulationScalarBoundaryType {
    SMOKE_SIMULATION_SCALAR_BOUNDARY_FIXED_VALUE = 0,
    SMOKE_SIMULATION_SCALAR_BOUNDARY_ZERO_FLUX   = 1,
    SMOKE_SIMULATION_SCALAR_BOUNDARY_PERIODIC    = 2,
} SmokeSimulationScalarBoundaryType;

/* One flow face: its type, the wall velocity (walls) and the face pressure (OUTFLOW) (:41-47). */
typedef struct SmokeSimulationFlowBoundaryFaceDesc {
    uint32_t type;
    float velocity_x;
    float velocity_y;
    float velocity_z;
    float pressure;
} SmokeSimulationFlowBoundaryFaceDesc;

typedef struct SmokeSimulationFlowBoundaryConfig {
    SmokeSimulationFlowBoundaryFaceDesc x_minus;
    SmokeSimulationFlowBoundaryFaceDesc x_plus;
    SmokeSimulationFlowBoundaryFaceDesc y_minus;
    SmokeSimulationFlowBoundaryFaceDesc y_plus;
    SmokeSimulationFlowBoundaryFaceDesc z_minus;
    SmokeSimulationFlowBoundaryFaceDesc z_plus;
} SmokeSimulationFlowBoundaryConfig;

/* One scalar face: its type and the ghost value used by FIXED_VALUE (:58-61). */
typedef struct SmokeSimulationScalarBoundaryFaceDesc {
    uint32_t type;
    float value;
} SmokeSimulationScalarBoundaryFaceDesc;

typedef struct SmokeSimulationScalarBoundaryConfig {
    SmokeSimulationScalarBoundaryFaceDesc x_minus;
    SmokeSimulationScalarBoundaryFaceDesc x_plus;
    SmokeSimulationScalarBoundaryFaceDesc y_minus;
    SmokeSimulationScalarBoundaryFaceDesc y_plus;
    SmokeSimulationScalarBoundaryFaceDesc z_minus;
    SmokeSimulationScalarBoundaryFaceDesc z_plus;
} SmokeSimulationScalarBoundaryConfig;

/* Interpolation used by semi-Lagrangian advection of velocity AND scalars (:72-75). */
typedef enum SmokeSimulationScalarAdvectionMode {
    SMOKE_SIMULATION_SCALAR_ADVECTION_LINEAR          = 0,
    SMOKE_SIMULATION_SCALAR_ADVECTION_MONOTONIC_CUBIC = 1,
} SmokeSimulationScalarAdvectionMode;

/* Scene parameters, immutable after create (:77-92). Cells are nx*ny*nz, x fastest; h = cell_size. */
typedef struct SmokeSimulationConfig {
    int32_t nx;
    int32_t ny;
    int32_t nz;
    float cell_size;
    float dt;
    int32_t pressure_iterations;
    float ambient_temperature;
    float buoyancy_density_factor;
    float buoyancy_temperature_factor;
    float vorticity_confinement;
    SmokeSimulationScalarAdvectionMode scalar_advection_mode;
    SmokeSimulationFlowBoundaryConfig flow_boundary;
    SmokeSimulationScalarBoundaryConfig density_boundary;
    SmokeSimulationScalarBoundaryConfig temperature_boundary;
} SmokeSimulationConfig;

typedef struct SmokeSimulationContext_t* SmokeSimulationContext;

/* stream: a cudaStream_t to run on, or NULL for a library-owned non-blocking stream (:96-101). */
typedef struct SmokeSimulationContextCreateDesc {
    SmokeSimulationConfig config;
    void* stream;
    float initial_density;
    float initial_temperature;
} SmokeSimulationContextCreateDesc;

/* Lifetime (:103-104). destroy(NULL) is OK. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_create_context_cuda(const SmokeSimulationContextCreateDesc* desc, SmokeSimulationContext* out_context);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_destroy_context_cuda(SmokeSimulationContext context);

/* Inputs, copied device-to-device on the context stream (:106-113). Cell fields hold nx*ny*nz floats
 * (occupancy: bytes, nonzero = solid). */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_density_cuda(SmokeSimulationContext context, const float* values);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_density_source_cuda(SmokeSimulationContext context, const float* values);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_temperature_cuda(SmokeSimulationContext context, const float* values);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_temperature_source_cuda(SmokeSimulationContext context, const float* values);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_force_cuda(SmokeSimulationContext context, const float* values_x, const float* values_y, const float* values_z);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_occupancy_cuda(SmokeSimulationContext context, const uint8_t* values);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_solid_velocity_cuda(SmokeSimulationContext context, const float* values_x, const float* values_y, const float* values_z);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_update_solid_temperature_cuda(SmokeSimulationContext context, const float* values);

/* One smoke step, enqueued on the context stream (:114). */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_step_cuda(SmokeSimulationContext context);

/* Fields a caller can read (:116-132). */
typedef enum SmokeSimulationViewKind {
    SMOKE_SIMULATION_VIEW_DENSITY                  = 0,
    SMOKE_SIMULATION_VIEW_DENSITY_SOURCE           = 1,
    SMOKE_SIMULATION_VIEW_TEMPERATURE              = 2,
    SMOKE_SIMULATION_VIEW_TEMPERATURE_SOURCE       = 3,
    SMOKE_SIMULATION_VIEW_FORCE                    = 4,
    SMOKE_SIMULATION_VIEW_SOLID_VELOCITY           = 5,
    SMOKE_SIMULATION_VIEW_SOLID_TEMPERATURE        = 6,
    SMOKE_SIMULATION_VIEW_FLOW_VELOCITY            = 7,
    SMOKE_SIMULATION_VIEW_FLOW_VELOCITY_MAGNITUDE  = 8,
    SMOKE_SIMULATION_VIEW_FLOW_PRESSURE            = 9,
    SMOKE_SIMULATION_VIEW_FLOW_PRESSURE_RHS        = 10,
    SMOKE_SIMULATION_VIEW_FLOW_DIVERGENCE          = 11,
    SMOKE_SIMULATION_VIEW_FLOW_VORTICITY           = 12,
    SMOKE_SIMULATION_VIEW_FLOW_VORTICITY_MAGNITUDE = 13,
    SMOKE_SIMULATION_VIEW_OCCUPANCY                = 14,
} SmokeSimulationViewKind;

/* F32_3D: one field in data0. F32_3D_SOA3: x/y/z components in data0/data1/data2 (:134-137). */
typedef enum SmokeSimulationViewLayout {
    SMOKE_SIMULATION_VIEW_LAYOUT_F32_3D      = 0,
    SMOKE_SIMULATION_VIEW_LAYOUT_F32_3D_SOA3 = 1,
} SmokeSimulationViewLayout;

/* consumer_stream: if non-NULL and not the context stream, it is made to wait for the context stream. */
typedef struct SmokeSimulationViewRequest {
    uint32_t kind;
    void* consumer_stream;
} SmokeSimulationViewRequest;

typedef struct SmokeSimulationView {
    uint32_t layout;
    int32_t nx;
    int32_t ny;
    int32_t nz;
    uint64_t row_stride_bytes;
    uint64_t slice_stride_bytes;
    const float* data0;
    const float* data1;
    const float* data2;
} SmokeSimulationView;

/* Borrowed device pointers to a field (:156). Unknown kind -> BACKEND_FAILURE. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_simulation_get_view_cuda(SmokeSimulationContext context, const SmokeSimulationViewRequest* request, SmokeSimulationView* out_view);

#ifdef __cplusplus
}
#endif

#endif /* VISUAL_SIMULATION_OF_SMOKE_3D_H */
