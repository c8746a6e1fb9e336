/*
 * Additive extensions of libsmoke_b200.so. None of them changes a symbol of visual-simulation-of-smoke-3d.h;
 * a caller that never calls them gets the reference's behaviour.
 *
 *  - solver selection: the reference runs exactly `pressure_iterations` iterations of unpreconditioned FP32 CG
 *    from x0 = 0 (backend-cuda.cu:1788-1824) and that is this library's default. The extension selects a
 *    Jacobi-preconditioned CG that stops at a relative residual, FP64 dot products, FP64 iterative
 *    refinement of the true residual and warm starts;
 *  - solver status: iterations, residuals and a status word of the last step's pressure solve (the reference
 *    computes none of these);
 *  - face-velocity access: the reference has no velocity setter (backend-cuda.cu:2085-2159), so a scene can
 *    only be seeded from rest; the setter lets a test or a checkpoint restore an arbitrary MAC state;
 *  - stage-wise stepping: runs the step's stages in order up to a given one, so each stage can be compared
 *    with a CPU restatement on its own;
 *  - batches: one call advances many independent scenes (the reference steps one context per call, each with its
 *    own graph launch).
 */
#ifndef SMOKE_B200_EXT_H
#define SMOKE_B200_EXT_H

#include "visual-simulation-of-smoke-3d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum SmokeB200SolverMode {
    /* Reference semantics: unpreconditioned CG, x0 = 0, exactly config.pressure_iterations iterations,
     * alpha/beta set to 0 when |denominator| <= 1e-20 (backend-cuda.cu:1414-1418, 1788-1824). */
    SMOKE_B200_SOLVER_FIXED_CG = 0,
    /* Jacobi-preconditioned CG that stops once ||r|| <= tolerance * ||b|| or after max_iterations. */
    SMOKE_B200_SOLVER_JACOBI_PCG = 1,
    /* Flexible CG preconditioned by one geometric multigrid V(1,1) cycle; same stopping rule as JACOBI_PCG. */
    SMOKE_B200_SOLVER_MG_FCG = 2,
} SmokeB200SolverMode;

typedef enum SmokeB200Reduction {
    SMOKE_B200_REDUCTION_FP32 = 0, /* dot products accumulated and kept in FP32, as cublasSdot does */
    SMOKE_B200_REDUCTION_FP64 = 1, /* dot products, alpha and beta in FP64; vectors stay FP32 */
} SmokeB200Reduction;

typedef struct SmokeB200SolverDesc {
    uint32_t mode;           /* SmokeB200SolverMode */
    uint32_t reduction;      /* SmokeB200Reduction */
    int32_t max_iterations;  /* JACOBI_PCG: iteration cap per refinement pass (FIXED_CG uses pressure_iterations) */
    float tolerance;         /* JACOBI_PCG: target ||b - A x||_2 / ||b||_2 */
    uint32_t refinement;     /* number of extra passes allowed when the FP64 true residual misses tolerance */
    uint32_t warm_start;     /* 1: start from the previous step's pressure instead of 0 */
} SmokeB200SolverDesc;

typedef enum SmokeB200SolveStatus {
    SMOKE_B200_SOLVE_CONVERGED      = 0, /* reached tolerance (JACOBI_PCG) */
    SMOKE_B200_SOLVE_ITERATION_CAP  = 1, /* ran all iterations (always the case for FIXED_CG) */
    SMOKE_B200_SOLVE_BREAKDOWN      = 2, /* a CG denominator vanished before convergence */
    SMOKE_B200_SOLVE_NOT_FINITE     = 3, /* NaN or Inf in a reduction */
    SMOKE_B200_SOLVE_BARRIER_TIMEOUT = 4, /* a grid barrier of the persistent solver gave up waiting */
    SMOKE_B200_SOLVE_NOT_RUN        = 5, /* no step has run yet */
} SmokeB200SolveStatus;

typedef struct SmokeB200SolverStatus {
    int32_t iterations;             /* inner iterations of the last solve, all refinement passes */
    int32_t passes;                 /* refinement passes run (1 = no refinement needed) */
    uint32_t status;                /* SmokeB200SolveStatus */
    uint32_t reserved;
    double rhs_norm;                /* ||b||_2 */
    double relative_residual;       /* recurrence residual ||r||/||b|| at exit */
    double true_relative_residual;  /* ||b - A x||/||b|| recomputed in FP64 at exit, -1 if not computed */
} SmokeB200SolverStatus;

/* Selects the pressure solver for every later step; re-captures the step graph. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_set_solver_cuda(SmokeSimulationContext context, const SmokeB200SolverDesc* desc);

/* Synchronises the context stream and reports the last step's pressure solve. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_get_solver_status_cuda(SmokeSimulationContext context, SmokeB200SolverStatus* out_status);

/* Copies face velocities from device pointers: u has (nx+1)*ny*nz values, v nx*(ny+1)*nz, w nx*ny*(nz+1),
 * x fastest, the reference's MAC layout (backend-cuda.cu:125-135). NULL means zero. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_set_face_velocity_cuda(SmokeSimulationContext context, const float* u, const float* v, const float* w);

/* Borrowed device pointers to the face velocities. which = 0: the step's velocity; which = 1: the advected
 * velocity before projection (the reference's temp_velocity_*). */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_get_face_velocity_cuda(SmokeSimulationContext context, uint32_t which, const float** out_u, const float** out_v, const float** out_w);

typedef enum SmokeB200Stage {
    SMOKE_B200_STAGE_FORCES          = 0, /* vorticity, buoyancy, confinement, face update, boundaries */
    SMOKE_B200_STAGE_ADVECT_VELOCITY = 1, /* semi-Lagrangian velocity advection into the temp velocity */
    SMOKE_B200_STAGE_PRESSURE        = 2, /* right-hand side and pressure solve */
    SMOKE_B200_STAGE_PROJECT         = 3, /* gradient subtract, boundaries, temp velocity -> velocity */
    SMOKE_B200_STAGE_SCALARS         = 4, /* temperature and density: source, advection, solid rules */
} SmokeB200Stage;

/* Runs the stages of one step from the first one through `last_stage` (eagerly, outside the step graph). */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_step_stages_cuda(SmokeSimulationContext context, uint32_t last_stage);

/* Solves the pressure system of the context's current right-hand side (the FLOW_PRESSURE_RHS view) into the
 * pressure buffer with the selected solver: the step's pressure stage without the right-hand-side kernel. Enqueued
 * on the context stream without a host wait (the multigrid solve is one CUDA-graph launch whose loop runs on the
 * device; the Jacobi and fixed CG solves are one cooperative kernel); the outcome is read with
 * smoke_b200_get_solver_status_cuda. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_solve_pressure_cuda(SmokeSimulationContext context);

/* A batch: a fixed set of contexts advanced together, one step each, by one CUDA-graph launch in which every
 * context's step is an independent branch, so scenes of any (different) sizes fill the GPU together. No reference
 * counterpart (the reference launches one graph per context, backend-cuda.cu:2161-2172).
 *  - create: the contexts must be distinct, on the current device, and idle (create waits for their streams). The
 *    batch records each context's step as it is configured now; after smoke_b200_set_solver_cuda or
 *    update_occupancy on a member, create the batch again. `stream` (NULL: a new stream) runs the batch graph;
 *  - step: ordered after all work enqueued so far on every member's stream, and every member's later work is
 *    ordered after it, so update_*, get_view and the status calls keep working per context;
 *  - destroy: waits for the batch stream; the contexts stay alive and usable alone. */
typedef struct SmokeB200Batch_t* SmokeB200Batch;
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_batch_create_cuda(const SmokeSimulationContext* contexts, uint32_t count, void* stream, SmokeB200Batch* out_batch);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_batch_step_cuda(SmokeB200Batch batch);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_batch_destroy_cuda(SmokeB200Batch batch);

/* The same solve with every solver kernel launched directly on the context stream, no graph: the multigrid loop is
 * driven from the host, which reads the loop condition after each iteration (one stream synchronisation per
 * iteration, so slower). For profilers that do not follow graph loops, and for hosts that cannot use CUDA graphs.
 * Results equal smoke_b200_solve_pressure_cuda's up to the summation order of the FP64 dot products. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_solve_pressure_eager_cuda(SmokeSimulationContext context);

/* Pressure solve that allocates nothing. No counterpart in the reference (which has no standalone solve and
 * allocates all its buffers with cudaMalloc when a context is created).
 *
 * For callers that cannot call cudaMalloc while they run: a renderer or engine that reserves its GPU memory up
 * front and forbids allocations in its frame loop (cudaMalloc can synchronise the device and stall a frame), or
 * a plug-in that lives inside another application's memory budget. The solver's scratch memory is one device
 * array inside the library image, so the call allocates no memory, neither directly nor through a library.
 *
 * Solves the system of the step's pressure stage for `config`, `occupancy` (nx*ny*nz bytes on the device, nonzero =
 * solid; NULL = no solids) and the right-hand side `rhs` (nx*ny*nz floats on the device) into `pressure` (device,
 * nx*ny*nz floats), on `stream`, with `solver` (NULL = the reference's fixed-count CG; warm_start is ignored).
 * The result equals smoke_b200_solve_pressure_cuda on a context holding the same occupancy and right-hand side.
 *
 * Limits and rules:
 *  - at most smoke_b200_noalloc_max_cells() = 64^3 = 262,144 cells; a larger grid returns BACKEND_FAILURE and
 *    smoke_b200_last_error() says why. The scratch array (about 11 MB) is held on every GPU that loads the library
 *    until the process exits;
 *  - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with that device
 *    current; make that first call before capturing any stream into a CUDA graph;
 *  - every call shares the one array: calls that overlap on the GPU (different streams, or several host threads)
 *    race and corrupt each other. Serialise them on one stream. The array keeps the last call's contents; the
 *    call itself clears whatever must start at zero;
 *  - out_status (optional) synchronises `stream` and reports like smoke_b200_get_solver_status_cuda. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_solve_pressure_noalloc_cuda(const SmokeSimulationConfig* config, const uint8_t* occupancy, const float* rhs, float* pressure,
                                                                                 const SmokeB200SolverDesc* solver, void* stream, SmokeB200SolverStatus* out_status);

/* Largest grid (cells) smoke_b200_solve_pressure_noalloc_cuda accepts. */
SMOKE_SIMULATION_API unsigned long long smoke_b200_noalloc_max_cells(void);

/* Reason of the last failure of smoke_b200_solve_pressure_noalloc_cuda on this host thread ("" if none). */
SMOKE_SIMULATION_API const char* smoke_b200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SMOKE_B200_EXT_H */
