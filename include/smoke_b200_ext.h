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
    /* Flexible CG preconditioned by the MG_FCG V-cycle V, corrected by the learned network U set with
     * smoke_b200_set_preconditioner_net_cuda: with r_V = r - A V(r) and N = P U(R r_V) (U on the multigrid level 1,
     * every extent halved; R the 2x2x2 child sums, P the V-cycle's prolongation), z = V(r) + g N + w D^-1 (r_V - g A N),
     * g = (N, r_V) / (N, A N). Same stopping rule, so the network changes the iteration count, not the answer. When
     * ||r||^2 shrinks by less than 1e-2 over 6 iterations the solve drops the network and goes on with the V-cycle
     * alone (flags bit 0). With warm_start = 2 the network's estimate P U(R b) is also the initial guess (needs
     * refinement >= 1). */
    SMOKE_B200_SOLVER_LEARNED_FCG = 3,
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
    uint32_t warm_start;     /* 1: start from the previous step's pressure instead of 0 (with refinement >= 1);
                                2 (LEARNED_FCG): start from the network's estimate of the pressure */
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
    uint32_t flags;                 /* bit 0: a LEARNED_FCG solve dropped the network for the V-cycle alone */
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
/* Per-member latency of the last batch step: ms_out[i] = milliseconds from the start of the batch graph to the end of
 * member i's step inside it (the device's global timer, stamped by the graph itself). Waits for the last batch step. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_batch_member_times_cuda(SmokeB200Batch batch, float* ms_out);

/* Launch shapes of a context's step (no reference counterpart; the reference fixes its launch shapes at compile
 * time). Every shape computes the same values: the advection shape changes which faces or cells a block of 256
 * threads covers, bit for bit the same results; the two solver grids change only the order in which the FP64 dot
 * products are summed. */
typedef struct SmokeB200LaunchTune {
    uint32_t advect_tile;  /* advection blocks: 0 flat (256 consecutive faces or cells, the default); boxes of
                              1: 32x8x1, 2: 32x4x2, 3: 16x4x4, 4: 8x8x4 faces or cells */
    uint32_t mg_wave;      /* multigrid level kernels, grid depth: 0, 1 (default), 2, 3: 1/2, 1, 2, 4 waves of
                              resident blocks; 4: one block per 32x4x2 tile */
    uint32_t pcg_grid;     /* persistent CG kernel (FIXED_CG, JACOBI_PCG): 0 all resident blocks (default), 1 half,
                              2 a quarter */
    uint32_t pcg_regs;     /* persistent CG kernel: 0 compiled without a register cap (default, 2 blocks per SM),
                              1 capped at 64 registers (4 blocks per SM, more loads in flight, a few spills) */
} SmokeB200LaunchTune;

/* One timed candidate of smoke_b200_autotune_cuda. */
typedef struct SmokeB200TuneRecord {
    SmokeB200LaunchTune tune;
    float ms_per_step;     /* best of the timed repeats, device time (CUDA events) */
    uint32_t iterations;   /* pressure iterations of the last timed step */
} SmokeB200TuneRecord;

#define SMOKE_B200_TUNE_MAX_RECORDS 16
#define SMOKE_B200_TUNE_FORCE 1u /* autotune flag: time the candidates even when the process has a result cached */

typedef struct SmokeB200TuneReport {
    SmokeB200LaunchTune chosen;
    float default_ms;      /* ms per step of the default shapes (0 when the result came from the cache) */
    float chosen_ms;       /* ms per step of the chosen shapes (0 when the result came from the cache) */
    uint32_t from_cache;   /* 1: an earlier call in this process tuned the same grid, solver and device */
    uint32_t record_count;
    SmokeB200TuneRecord records[SMOKE_B200_TUNE_MAX_RECORDS];
} SmokeB200TuneReport;

/* Sets the launch shapes of the context's step and rebuilds its step graph (BACKEND_FAILURE for an unknown code).
 * Like smoke_b200_set_solver_cuda, this is not ordered against work in flight on other streams. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_set_launch_tune_cuda(SmokeSimulationContext context, const SmokeB200LaunchTune* tune);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_get_launch_tune_cuda(SmokeSimulationContext context, SmokeB200LaunchTune* out);

/* Autotuner: times the context's own step under candidate launch shapes and keeps the fastest. Coordinate search
 * from the current shapes: every advection shape, then every grid of the selected solver (multigrid depth, or the
 * persistent CG grid and register variant), each candidate timed as `steps` (0: 4) graph steps from the same state, best of two
 * repeats, after one untimed step. The context's device state is saved before and restored after (one temporary
 * device allocation of the context's size), so tuning does not advance the simulation. The result is cached per
 * process by device, grid extents, advection mode and solver settings: a later call for a context with the same
 * key applies the cached shapes without timing unless `flags` has SMOKE_B200_TUNE_FORCE. Synchronises the context
 * stream. `report` (optional) receives the candidates and their times. Tune before creating a batch that holds
 * the context: a batch keeps the shapes its members had when it was created. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_autotune_cuda(SmokeSimulationContext context, uint32_t steps, uint32_t flags, SmokeB200TuneReport* report);

/* Learned preconditioner (no reference counterpart): a 3-level 3-D U-Net on (r * s, fluid mask), s = sqrt(n) / ||r||,
 * whose output y gives N(r) = y / s on fluid cells (0 on solids), so N(c r) = c N(r) for c > 0. Its 3x3x3
 * convolutions run on the tensor cores (BF16 operands, FP32 accumulation), forward and backward; the parameters, their
 * gradient and the Adam moments are FP32. Trained on (rhs, occupancy) -> pressure pairs with the relative loss
 * ||N(b) - p||^2 / ||p||^2 over fluid cells.
 *  - create: parameters drawn from `seed` (He-normal weights, zero biases);
 *  - get/set_parameters: smoke_b200_net_parameter_count() FP32 values on the host, layer by layer, each layer its
 *    weights [27][cin][cout] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)) then its cout biases; set resets the Adam state;
 *  - apply: out = N(rhs) for one volume (device pointers, nx*ny*nz values each);
 *  - gradient: the loss of one (rhs, occupancy, target) sample and its gradient (host, parameter layout);
 *  - train: one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the mean gradient of `count` samples stored one after
 *    another (count * nx*ny*nz values each); mean loss to *mean_loss_out.
 * Every call synchronises `stream` and may grow the network's evaluation workspace (cudaMalloc). A network is used by
 * one host thread at a time. */
typedef struct SmokeB200Net_t* SmokeB200Net;
SMOKE_SIMULATION_API uint32_t smoke_b200_net_parameter_count(void);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_net_create_cuda(uint32_t seed, SmokeB200Net* out_net);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_net_destroy_cuda(SmokeB200Net net);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_net_get_parameters_cuda(SmokeB200Net net, float* out);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_net_set_parameters_cuda(SmokeB200Net net, const float* values);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_net_apply_cuda(SmokeB200Net net, int nx, int ny, int nz, const float* rhs, const uint8_t* occupancy, float* out, void* stream);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_net_gradient_cuda(SmokeB200Net net, int nx, int ny, int nz, const float* rhs, const uint8_t* occupancy, const float* target, float* grad_out, double* loss_out, void* stream);
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_net_train_cuda(SmokeB200Net net, int nx, int ny, int nz, uint32_t count, const float* rhs, const uint8_t* occupancy, const float* target, float learning_rate, double* mean_loss_out, void* stream);

/* out = A x, the matrix of the context's pressure system (the step's Poisson operator for the current occupancy:
 * identity rows at solid cells and at the anchor cell), applied matrix-free; x and out: nx*ny*nz floats on the
 * device, distinct. Enqueued on the context stream. For residual checks and for building training pairs
 * (A e, e) of the learned preconditioner. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_apply_operator_cuda(SmokeSimulationContext context, const float* x, float* out);

/* z = V(r): one V(1,1) cycle of the multigrid preconditioner of SMOKE_B200_SOLVER_MG_FCG on the residual r, over the
 * context's hierarchy (current occupancy). r and z: nx*ny*nz floats on the device, distinct; z is 0 at solid cells and
 * the anchor. Enqueued on the context stream; uses the hierarchy's scratch, so it must not overlap a solve of this
 * context. For building the learned preconditioner's training pairs (what the V-cycle leaves of an error). */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_apply_multigrid_cuda(SmokeSimulationContext context, const float* r, float* z);

/* The context's copy of the network for SMOKE_B200_SOLVER_LEARNED_FCG (the parameters as they are now; later training
 * of `net` does not change the context until this is called again). Allocates the context's evaluation workspace and
 * rebuilds the step graph. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_set_preconditioner_net_cuda(SmokeSimulationContext context, SmokeB200Net net);

/* Schedule of the learned solve: the network corrects the V-cycle in the first `count` iterations of every
 * refinement pass and the V-cycle preconditions alone after them (0, the default: every iteration). Rebuilds the step
 * graph. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_set_learned_iterations_cuda(SmokeSimulationContext context, uint32_t count);

/* 3x3x3 convolution (zero padding) of a channels-last BF16 volume on the tensor cores, the layer of the learned
 * preconditioner's network. `in`: nx*ny*nz cells x S(cin) BF16 values, S(c) = 8 for c <= 8, else c rounded up to a
 * multiple of 16 (channels past cin must be 0); `weights`: FP32 [27][cin][cout] on the device, tap = (dz+1)*9 +
 * (dy+1)*3 + (dx+1); `bias`: cout FP32 on the device or NULL. out = act(conv + bias), act = ReLU when `relu`: `out`
 * (optional) gets nx*ny*nz x S(cout) BF16 values, `out_f32` (optional) channel 0 as FP32. Allocates a small scratch
 * buffer and synchronises `stream`. S(cin) in {8, 16, 32, 64, 128} and 1 <= cout <= 128. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_conv3d_cuda(int nx, int ny, int nz, int cin, int cout, const void* in, const float* weights, const float* bias, int relu, void* out, float* out_f32, void* stream);

/* Test hook of the convolution kernels' bounded waits (no counterpart in the reference, which has no tensor-core
 * code). Runs the 16-channel convolution over an nx*ny*nz zero volume with every TMA load expected but never
 * issued, and every wait bounded by `wait_cycles` clock cycles (1..4e9): each block's first wait runs out, the block
 * frees its tensor memory and leaves, and the error word (bit 0 set) is written to *error_out. Synchronises `stream`;
 * allocates a scratch buffer. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_test_conv_wait_timeout_cuda(int nx, int ny, int nz, unsigned long long wait_cycles, unsigned* error_out, void* stream);

/* The same solve with every solver kernel launched directly on the context stream, no graph: the multigrid loop is
 * driven from the host, which reads the loop condition after each iteration (one stream synchronisation per
 * iteration, so slower). For profilers that do not follow graph loops, and for hosts that cannot use CUDA graphs.
 * Results equal smoke_b200_solve_pressure_cuda's up to the summation order of the FP64 dot products. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_solve_pressure_eager_cuda(SmokeSimulationContext context);

/* Test hook of the solver's bounded waits (no counterpart in the reference, whose waits are library calls that
 * return error codes, backend-cuda.cu:1611-1614, 2063-2071). Runs the context's persistent CG solve (solver mode
 * FIXED_CG or JACOBI_PCG; the multigrid modes have no grid barrier and are refused) on its current right-hand side
 * with block `block` (>= 1) of the cooperative grid leaving before its first grid barrier, and every barrier wait
 * bounded by `timeout_ms` (1..10000). The other blocks' waits run out, the solve aborts and the status (synchronised,
 * written to out_status) reads SMOKE_B200_SOLVE_BARRIER_TIMEOUT; the context stays usable. A block index beyond the
 * grid withholds nothing, and the solve runs normally. */
SMOKE_SIMULATION_API SmokeSimulationResult smoke_b200_test_barrier_timeout_cuda(SmokeSimulationContext context, uint32_t block, uint32_t timeout_ms, SmokeB200SolverStatus* out_status);

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
 * `config` is checked as smoke_simulation_create_context_cuda checks it (extents, cell size, dt and
 * pressure_iterations positive; boundary types in range; a periodic face only opposite a periodic face).
 * `solver` may select SMOKE_B200_SOLVER_FIXED_CG or SMOKE_B200_SOLVER_JACOBI_PCG (the persistent CG kernel), with
 * FP32 or FP64 reductions and refinement <= 64; the multigrid and learned modes need a context's hierarchy and are
 * refused. Every refusal returns BACKEND_FAILURE with its reason in smoke_b200_last_error() ("invalid
 * configuration ...", "invalid solver description ...", "... exceeds the no-allocation limit ...").
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
 *  - out_status (optional) synchronises `stream` and reports like smoke_b200_get_solver_status_cuda. Without it
 *    the call returns as soon as the work is enqueued; a failure of a CUDA call is also reported with its name and
 *    CUDA's error text in smoke_b200_last_error(). */
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
