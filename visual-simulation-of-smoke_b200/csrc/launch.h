// Host-side launchers of the B200 smoke kernels. Plain pointers and sizes only; every launcher enqueues on
// `stream` and returns the launch status.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "smoke_device.cuh"

namespace smoke_b200 {

// Face velocity triple (u: (nx+1)*ny*nz, v: nx*(ny+1)*nz, w: nx*ny*(nz+1)).
struct Faces {
    float* u;
    float* v;
    float* w;
};
struct ConstFaces {
    const float* u;
    const float* v;
    const float* w;
};
// The scalar stage's sourced fields, which the force kernel forms too when t_tmp is set: t_tmp = (solid ? solid
// temperature : temperature) + dt * temperature source, d_tmp = density + dt * density source, and (t_pad set) the
// interiors of their padded copies.
struct ScalarSources {
    const float* ts;
    const float* ds;
    const float* solid_t;
    float* t_tmp;
    float* d_tmp;
    float* t_pad;
    float* d_pad;
};
inline ConstFaces as_const(const Faces& f) { return {f.u, f.v, f.w}; }

// One entry of the density fill list: a solid cell and the fluid cell it copies (-1: none, value 0).
struct FillEntry {
    uint32_t cell;
    int32_t source;
};

StepParams make_params(const SmokeSimulationConfig& cfg);

// Launch shapes the autotuner chooses between (every choice computes the same values).
// Advection blocks of 256 threads: flat (256 consecutive faces or cells), or a box of 2^x x 2^y x 2^z of them.
constexpr int kAdvectTileCount = 5;
constexpr int kAdvectTiles[kAdvectTileCount][3] = {{-1, 0, 0}, {5, 3, 0}, {5, 2, 1}, {4, 2, 2}, {3, 3, 2}};
// Sets P.tile to the advection shape `code` (index into kAdvectTiles); false for an unknown code.
bool set_advect_tile(StepParams& P, int code);
// Multigrid level kernels: grid depth along z as a multiple of one wave of resident blocks (x 1/2, 1, 2, 4), or
// one z tile per block.
constexpr int kMgWaveCount = 5;
constexpr int kMgWaveDefault = 1;
// Persistent CG kernel: all resident blocks, half of them, a quarter; and its register-capped variant or not.
constexpr int kPcgGridCount = 3;
constexpr int kPcgRegsCount = 2;

// Forces: vorticity of the cell-centred velocity (writes the four vorticity buffers).
cudaError_t launch_vorticity(const StepParams& P, ConstFaces vel, const uint8_t* occ, float* wx, float* wy, float* wz, float* wmag, cudaStream_t s);
// Forces: f = user force + buoyancy + vorticity confinement per cell.
cudaError_t launch_cell_force(const StepParams& P, const float* wx, const float* wy, const float* wz, const float* wmag, const float* density, const float* temperature, const float* ufx, const float* ufy, const float* ufz, const uint8_t* occ, float* fx, float* fy, float* fz, cudaStream_t s, const ScalarSources& S = ScalarSources{});
// Forces: out = settled(in + dt * face-average of f) (domain, solid and periodic face rules applied).
cudaError_t launch_face_force(const StepParams& P, ConstFaces in, const float* fx, const float* fy, const float* fz, const uint8_t* occ, ConstFaces solid, Faces out, cudaStream_t s, Faces pad = Faces{});
// Padded copies (PadField): element count of the copy of field kind (0-2 face components, 3 density, 4
// temperature).
size_t pad_count(const StepParams& P, int kind);
// Fills the padded copies of `count` (1..3) fields of the given kinds in one launch.
cudaError_t launch_pads(const StepParams& P, int count, const int* kinds, const float* const* fields, float* const* pads, cudaStream_t s, int ghost_only = 0);
// Velocity self-advection: out = settled(semi-Lagrangian sample of in along in); pad holds the padded copies of in.
cudaError_t launch_advect_velocity(const StepParams& P, ConstFaces in, ConstFaces pad, const uint8_t* occ, ConstFaces solid, Faces out, cudaStream_t s);
// Pressure right-hand side from the advected velocity.
cudaError_t launch_rhs(const StepParams& P, ConstFaces vel, const uint8_t* occ, const int32_t* anchor, float* rhs, cudaStream_t s);
// Projection: out = settled(in - dt * grad p / h); pressure64 (optional) is the FP64 solution of a refined solve.
cudaError_t launch_project(const StepParams& P, ConstFaces in, const float* pressure, const double* pressure64, const uint8_t* occ, ConstFaces solid, Faces out, cudaStream_t s, Faces pad = Faces{});
// Scalars: one shared back-trace per cell, sample both scalars, solid rules (vel_pad, t_pad, d_pad: padded copies).
cudaError_t launch_advect_scalars(const StepParams& P, ConstFaces vel, ConstFaces vel_pad, const uint8_t* occ, const float* t_tmp, const float* t_pad, const float* d_tmp, const float* d_pad, const float* solid_temperature, float* temperature, float* density, cudaStream_t s);
// Scalars: solid cells copy their nearest fluid cell's density.
cudaError_t launch_density_fill(const FillEntry* list, const uint32_t* count, float* density, int max_blocks, cudaStream_t s);
// Derived views: centred velocity, |u|, vorticity, |w|, divergence of the step's final velocity.
// View groups the views kernel computes: centred velocity and its magnitude; vorticity, its magnitude and divergence.
constexpr uint32_t kViewsVelocity = 1, kViewsVorticity = 2, kViewsAll = 3;
cudaError_t launch_views(const StepParams& P, ConstFaces vel, const uint8_t* occ, float* cx, float* cy, float* cz, float* vmag, float* wx, float* wy, float* wz, float* wmag, float* div, uint32_t groups, cudaStream_t s);

// Occupancy-derived data (run when occupancy changes).
cudaError_t launch_occupancy_float(const StepParams& P, const uint8_t* occ, float* out, cudaStream_t s);
cudaError_t launch_anchor(const StepParams& P, const uint8_t* occ, int32_t* anchor, cudaStream_t s);
cudaError_t launch_stencil_codes(const StepParams& P, const uint8_t* occ, const int32_t* anchor, uint16_t* codes, cudaStream_t s);
cudaError_t launch_fill_build(const StepParams& P, const uint8_t* occ, const int32_t* anchor, FillEntry* list, uint32_t* count, cudaStream_t s);

cudaError_t launch_fill_value(float* dst, float value, uint64_t count, cudaStream_t s);

// ------------------------------------------------------------------------------------------ pressure solve
// Persistent, cooperative conjugate-gradient solver (pcg.cu). One launch solves A x = b for the masked
// 7-point operator encoded in `codes` (bits 0-5: active neighbours -x,+x,-y,+y,-z,+z; bits 8-10: diagonal).
struct PcgSettings {
    int32_t jacobi;          // 0: M = I (reference CG), 1: M = diag(A)^-1
    int32_t fp64;            // reductions in FP64 (1) or FP32 (0)
    int32_t fixed;           // 1: run exactly max_iterations (reference semantics), 0: stop at tolerance
    int32_t max_iterations;
    float tolerance;
    int32_t refinement;      // extra passes on the FP64 true residual
    int32_t warm_start;      // start from x instead of 0
    int32_t withhold_block;  // test only: > 0 makes block withhold_block - 1 leave before its first grid barrier
    uint32_t barrier_timeout_ms;  // bound of every grid-barrier wait (0: the default, 2000 ms)
    uint32_t pad;
};

struct PcgStatusDevice {
    int32_t iterations;
    int32_t passes;
    uint32_t status;
    uint32_t flags;     // bit 0: the learned solve fell back to the plain preconditioner
    double rhs_norm;
    double relative_residual;
    double true_relative_residual;
};

// Device-resident control block: grid barrier counter (its top bit flips once every block has arrived), abort flag,
// a ring of three all-reduce slots (each spread over kPcgSumCopies cache lines so that concurrent atomic adds
// contend less) and the status of the last solve. Zeroed (up to `status`) before every launch.
constexpr int kPcgMaxBlocks = 148 * 16;
constexpr int kPcgSumCopies = 8;
struct PcgControl {
    unsigned int bar;
    unsigned int pad0;
    int abort;
    int pad1;
    unsigned int pad2[28];
    double totals[3][kPcgSumCopies][16];  // 4 sums per copy, one 128-byte line per copy
    PcgStatusDevice status;
};
constexpr size_t kPcgControlResetBytes = offsetof(PcgControl, status);

struct PcgWork {
    float* r[2];
    float* s[2];
    float* w[2];
    float* p;
    float* e;      // FP32 correction iterate of a refinement pass
    double* x64;   // FP64 solution accumulator (refinement); kept between steps as the warm start
    double* part;  // per-block partial sums of the dot products, [kAccCount][part_stride] (FP64)
    uint32_t part_stride;  // blocks of the largest level-0 grid (mg_partial_blocks)
};
// Blocks of the largest grid a level-0 kernel of the multigrid solve launches on an nx x ny x nz grid (one
// 32 x 4 x 2 tile per block): the length of each accumulator's row of per-block partial sums.
uint32_t mg_partial_blocks(int nx, int ny, int nz);

struct PcgLaunchShape {
    int blocks;
    int threads;
    int grid;  // kPcgGridCount code: the persistent grid is the resident blocks divided by 1 << grid
    int regs;  // 0: kernel compiled without a register cap (2 blocks per SM); 1: capped to 64 (4 blocks per SM)
};

// ------------------------------------------------------------------------------------------ multigrid hierarchy
// Geometric multigrid for the pressure operator (mgsolve.cu). Level 0 is the grid itself; level l+1 halves every
// extent (rounding up). A coarse cell is fluid when any of its children is; every level's operator is the masked
// 7-point stencil of its fluid cells (the fine rules without the anchor).
constexpr int kMgMaxLevels = 12;
constexpr uint32_t kMgBlockLevelCells = 512;   // levels this small may run inside one block, in shared memory
constexpr uint32_t kMgBlockBytes = 16 * 1024;  // shared memory for those levels (3 floats + 1 code per cell)
// Shared-memory words of one block-level level of n cells: r, zp, t and the 16-bit codes (padded pairs).
__host__ __device__ constexpr uint32_t mg_block_words(uint32_t n) { return 3u * n + (n + 2u) / 2u; }
// Bit of the operator code that marks a cell whose unknown is solved for (fluid; at level 0 also not the anchor).
constexpr uint16_t kCodeActive = 1u << 12;
struct MgLevel {
    int nx, ny, nz;
    uint32_t n;
    FastDiv div_nx, div_slab;
    uint16_t* code;   // row codes (level 0: the fine operator's codes); arrays hold n + 2 entries
    uint8_t* fluid;   // 1 = fluid cell
    float* r;         // right-hand side / residual of the level (level 0: the solver residual)
    float* zp;        // correction (level 0: the preconditioned residual z)
    float* t;         // scratch of the level
};
struct MgHierarchy {
    int levels;       // >= 2
    int grid_levels;  // levels [0, grid_levels) run on the whole grid; coarser ones inside block 0's shared memory
    int fper[3];
    int fout[6];      // non-periodic OUTFLOW faces (x-, x+, y-, y+, z-, z+): prolongation extrapolates to -parent there
    MgLevel L[kMgMaxLevels];
};
// Level-0 vectors of the multigrid FCG solve (the residual and search direction are double-buffered: a pass reads
// one buffer and writes the other, and the device-side parity picks which).
struct MgWork {
    float* r[2];
    float* p[2];
    float* q;
    float* e;      // FP32 correction iterate of a refinement pass
    double* x64;   // FP64 solution accumulator (refinement); kept between steps as the warm start
    double* part;  // per-block partial sums of the dot products, [kAccCount][part_stride] (FP64)
    uint32_t part_stride;  // blocks of the largest level-0 grid (mg_partial_blocks)
};
// Blocks of the largest grid a level-0 kernel of the multigrid solve launches on an nx x ny x nz grid (one
// 32 x 4 x 2 tile per block): the length of each accumulator's row of per-block partial sums.
uint32_t mg_partial_blocks(int nx, int ny, int nz);
// Device-side scalars of one multigrid solve (reset at the start of every solve).
enum MgAccumulator { kAccBB = 0, kAccRR, kAccZR, kAccZQ, kAccPQ, kAccPR, kAccNet, kAccNetA, kAccCount };
struct MgState {
    double bb, rnorm2, pq_prev, target2, pass_rr0, true_rel;
    double net_rr;         // learned solve: ||r - A z_V||^2, the squared norm of the network's input
    double net_gamma;      // learned solve: the energy-optimal step along the network's correction
    float alpha, beta;     // step sizes, computed by the last block of the kernel that completes their sums
    unsigned int done[7];  // last-block election counters
    int parity, first_iter, it, passes;
    uint32_t status, fail, halt, zero_solution;
    uint32_t loop;         // the loop condition the last update set (read by the host in eager mode)
    uint32_t fallback;     // learned solve: 1 once the network is dropped (the V-cycle alone preconditions)
    int stall_it;          // learned solve: iteration of the last stagnation checkpoint
    double stall_ref;      // learned solve: ||r||^2 at that checkpoint
    int pass_it0;          // learned solve: iteration count when the current refinement pass started
    uint32_t net_off;      // learned solve: 1 when this iteration runs without the network (fallback or schedule)
};
// Learned solve: the network is dropped, leaving the V-cycle alone, when ||r|| shrank less than 10x
// (||r||^2 less than kLearnedStallReduction2) over kLearnedStallWindow iterations; the V-cycle alone gains about
// 3x per iteration.
constexpr int kLearnedStallWindow = 6;
constexpr double kLearnedStallReduction2 = 1e-2;
struct MgSolveArgs {
    MgHierarchy H;
    MgWork W;
    const float* b;
    float* x;
    float* e;  // the FP32 iterate: x itself without refinement, else W.e
    MgState* st;
    int ir, warm, max_iterations, refinement;
    float tol;
    int wave;                        // grid depth of the level kernels (kMgWaveCount codes)
    int learned;                     // 1: the V-cycle's result is corrected by the network of `net`
    int net_warm;                    // 1 (learned): the initial guess is the network's estimate N(b)
    int net_iterations;              // learned: the network corrects the first this many iterations of a pass (0: all)
    const struct LearnedSolve* net;  // host-side: the network's images, workspace and mask (learned only)
};
// Level extents and the number of grid-wide levels for a fine grid.
int mg_level_count(int nx, int ny, int nz);
// Largest refinement count the multigrid solve honours (the graph unrolls refinement + 1 passes).
int mg_max_refinement();
// Writes the device's global nanosecond timer into *slot when the stream reaches it (batch member latencies).
cudaError_t launch_time_stamp(unsigned long long* slot, cudaStream_t s);
// z = V(r): one V-cycle of the multigrid preconditioner on the residual r (the solve's preconditioner, standalone).
cudaError_t launch_mg_vcycle(const MgHierarchy& H, int wave_depth, const float* r, float* z, cudaStream_t s);
// out = A x with the fine operator (the pressure system's matrix, matrix-free from the level-0 codes).
cudaError_t launch_mg_apply(const MgHierarchy& H, const float* x, float* out, cudaStream_t s);
// Builds level fluid masks and codes from the occupancy (after the fine codes and anchor exist).
cudaError_t launch_mg_setup(const StepParams& P, const MgHierarchy& H, const uint8_t* occ, cudaStream_t s);
// The learned preconditioner network's solid mask on level 1 (1 where a cell has no fluid child), after the setup.
cudaError_t launch_mg_net_mask(const MgHierarchy& H, uint8_t* solid, cudaStream_t s);
// Records the multigrid-preconditioned FCG solve of A x = b into the graph being captured on `s` (kernels, and
// one `while` node per pass whose body is captured on `body_stream`); the outcome lands in *status_out.
cudaError_t enqueue_mg_solve(const MgSolveArgs& args, bool fp64, PcgStatusDevice* status_out, cudaStream_t s, cudaStream_t body_stream);
// The same solve launched kernel by kernel on `s` (no graph): the host reads the loop condition after every update
// (one stream synchronisation per iteration). For profilers that do not enter graph loops and hosts without graphs.
cudaError_t run_mg_solve_eager(const MgSolveArgs& args, bool fp64, PcgStatusDevice* status_out, cudaStream_t s);

// Picks the persistent grid (all blocks co-resident) for the current device.
cudaError_t pcg_launch_shape(PcgLaunchShape* out);
// Enqueues: reset of the control header, then the cooperative solver launch.
cudaError_t launch_pcg(const StepParams& P, const PcgSettings& S, const PcgLaunchShape& shape, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s);

}  // namespace smoke_b200
