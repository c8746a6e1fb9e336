// C ABI of libsmoke_b200.so: context lifetime, inputs, step, views (visual-simulation-of-smoke-3d.h) and the
// extensions of smoke_b200_ext.h. Host code only; kernels are reached through launch.h.
//
// Reference behaviour: backend-cuda.cu:1833-2282. Design:
//  - one device arena per context (256-byte aligned sub-buffers), so a context is one cudaMalloc;
//  - three face-velocity sets: A (state), B (after forces), C (after advection); the projection writes A, so a
//    step needs no device-to-device copies;
//  - the step is captured once into a CUDA graph on a private stream and launched on the context stream;
//  - derived views (centred velocity, |u|, vorticity, |w|, divergence) are computed on demand in get_view, and
//    materialised before an occupancy or velocity change so they always reflect the state right after the step;
//  - occupancy-derived data (pressure anchor, operator row codes, density fill list) is rebuilt only when
//    occupancy changes.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include <nvtx3/nvtx3.hpp>

#include "config_check.h"
#include "launch.h"
#include "smoke_b200_ext.h"
#include "unet.h"
#include "visual-simulation-of-smoke-3d.h"

static_assert(sizeof(SmokeSimulationFlowBoundaryFaceDesc) == 20);
static_assert(sizeof(SmokeSimulationFlowBoundaryConfig) == 120);
static_assert(sizeof(SmokeSimulationScalarBoundaryFaceDesc) == 8);
static_assert(sizeof(SmokeSimulationScalarBoundaryConfig) == 48);
static_assert(sizeof(SmokeSimulationConfig) == 44 + 120 + 48 + 48);
static_assert(offsetof(SmokeSimulationConfig, flow_boundary) == 44);
static_assert(offsetof(SmokeSimulationConfig, density_boundary) == 164);
static_assert(offsetof(SmokeSimulationConfig, temperature_boundary) == 212);
static_assert(sizeof(SmokeSimulationContextCreateDesc) == 280);
static_assert(offsetof(SmokeSimulationContextCreateDesc, stream) == 264);
static_assert(sizeof(SmokeSimulationViewRequest) == 16);
static_assert(sizeof(SmokeSimulationView) == 56);
static_assert(offsetof(SmokeSimulationView, row_stride_bytes) == 16);
static_assert(offsetof(SmokeSimulationView, data0) == 32);
static_assert(sizeof(SmokeB200SolverStatus) == sizeof(smoke_b200::PcgStatusDevice));

namespace smoke_b200 {
namespace {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace smoke_b200

using namespace smoke_b200;

struct SmokeSimulationContext_t {
    SmokeSimulationConfig config{};
    StepParams P{};
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    cudaStream_t capture_stream = nullptr;
    cudaStream_t body_stream = nullptr;      // captures the bodies of the solver's graph loops
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphExec_t solve_exec = nullptr;    // the multigrid solve alone (solve_pressure / eager stages)
    void* arena = nullptr;
    size_t arena_bytes = 0;
    int fill_blocks = 0;

    Faces A{}, B{}, C{};
    float *density = nullptr, *density_tmp = nullptr, *density_source = nullptr;
    float *temperature = nullptr, *temperature_tmp = nullptr, *temperature_source = nullptr;
    float *force_x = nullptr, *force_y = nullptr, *force_z = nullptr;
    float *solid_vx = nullptr, *solid_vy = nullptr, *solid_vz = nullptr, *solid_temperature = nullptr;
    float* occupancy_float = nullptr;
    float *pressure = nullptr, *rhs = nullptr;
    float *cx = nullptr, *cy = nullptr, *cz = nullptr, *vmag = nullptr;
    float *wx = nullptr, *wy = nullptr, *wz = nullptr, *wmag = nullptr, *divergence = nullptr;
    float *fx = nullptr, *fy = nullptr, *fz = nullptr;
    Faces pad{};                                       // padded copies of the velocity being sampled
    float *pad_t = nullptr, *pad_d = nullptr;          // padded copies of the scalar sources
    PcgWork pcg{};
    uint16_t* codes = nullptr;
    uint8_t* occupancy = nullptr;
    FillEntry* fill_list = nullptr;
    uint32_t* fill_count = nullptr;
    int32_t* anchor = nullptr;
    PcgControl* control = nullptr;
    MgHierarchy mg{};
    MgWork mg_work{};
    MgState* mg_state = nullptr;

    SmokeB200SolverDesc solver{SMOKE_B200_SOLVER_FIXED_CG, SMOKE_B200_REDUCTION_FP32, 500, 1.0e-5f, 0, 0};
    SmokeB200LaunchTune tune{0, kMgWaveDefault, 0, 0};
    PcgLaunchShape pcg_shape{};
    void* learned_mem = nullptr;  // the preconditioner network's images and workspace (LEARNED_FCG)
    size_t learned_bytes = 0;
    LearnedSolve learned{};
    bool has_net = false;
    uint32_t views_stale = 0;  // view groups (kViews*) not yet computed for the current state
    bool stepped = false;

    ~SmokeSimulationContext_t() { release(); }

    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (solve_exec) cudaGraphExecDestroy(solve_exec);
        exec = nullptr;
        graph = nullptr;
        solve_exec = nullptr;
        if (arena) cudaFree(arena);
        arena = nullptr;
        if (learned_mem) cudaFree(learned_mem);
        learned_mem = nullptr;
        if (capture_stream) cudaStreamDestroy(capture_stream);
        capture_stream = nullptr;
        if (body_stream) cudaStreamDestroy(body_stream);
        body_stream = nullptr;
        if (owns_stream && stream) cudaStreamDestroy(stream);
        stream = nullptr;
        owns_stream = false;
    }

    void allocate() {
        const size_t n = P.n, nu = P.nu, nv = P.nv, nw = P.nw;
        struct Slot {
            void** ptr;
            size_t bytes;
        };
        std::vector<Slot> slots;
        auto f32 = [&](float** p, size_t count) { slots.push_back({reinterpret_cast<void**>(p), count * sizeof(float)}); };
        for (Faces* f : {&A, &B, &C}) {
            f32(&f->u, nu);
            f32(&f->v, nv);
            f32(&f->w, nw);
        }
        for (float** p : {&density, &density_tmp, &density_source, &temperature, &temperature_tmp, &temperature_source, &force_x, &force_y, &force_z, &solid_vx, &solid_vy, &solid_vz, &solid_temperature, &occupancy_float, &pressure, &rhs, &cx, &cy, &cz, &vmag, &wx, &wy, &wz, &wmag,
                          &divergence, &fx, &fy, &fz, &pcg.r[0], &pcg.r[1], &pcg.s[0], &pcg.s[1], &pcg.w[0], &pcg.w[1], &pcg.p, &pcg.e})
            f32(p, n);
        slots.push_back({reinterpret_cast<void**>(&pcg.x64), n * sizeof(double)});
        f32(&pad.u, pad_count(P, 0));
        f32(&pad.v, pad_count(P, 1));
        f32(&pad.w, pad_count(P, 2));
        f32(&pad_t, pad_count(P, 4));
        f32(&pad_d, pad_count(P, 3));
        slots.push_back({reinterpret_cast<void**>(&codes), (n + 2) * sizeof(uint16_t)});
        slots.push_back({reinterpret_cast<void**>(&occupancy), n});
        slots.push_back({reinterpret_cast<void**>(&fill_list), n * sizeof(FillEntry)});
        slots.push_back({reinterpret_cast<void**>(&fill_count), sizeof(uint32_t)});
        slots.push_back({reinterpret_cast<void**>(&anchor), sizeof(int32_t)});
        slots.push_back({reinterpret_cast<void**>(&control), sizeof(PcgControl)});
        slots.push_back({reinterpret_cast<void**>(&mg_state), sizeof(MgState)});
        mg_work.part_stride = mg_partial_blocks(P.nx, P.ny, P.nz);
        slots.push_back({reinterpret_cast<void**>(&mg_work.part), static_cast<size_t>(kAccCount) * mg_work.part_stride * sizeof(double)});
        // multigrid levels: level 0 shares the Jacobi solver's vectors; coarser levels get their own arrays
        mg.levels = mg_level_count(P.nx, P.ny, P.nz);
        for (int a = 0; a < 3; ++a) mg.fper[a] = P.fper[a];
        for (int e = 0; e < 6; ++e) mg.fout[e] = !P.fper[e >> 1] && P.flow[e].type == kFlowOutflow ? 1 : 0;
        int lx = P.nx, ly = P.ny, lz = P.nz;
        for (int l = 0; l < mg.levels; ++l) {
            MgLevel& L = mg.L[l];
            L.nx = lx;
            L.ny = ly;
            L.nz = lz;
            L.n = static_cast<uint32_t>(lx) * ly * lz;
            L.div_nx = FastDiv(lx);
            L.div_slab = FastDiv(static_cast<uint32_t>(lx) * ly);
            slots.push_back({reinterpret_cast<void**>(&L.fluid), L.n});
            if (l > 0) {
                slots.push_back({reinterpret_cast<void**>(&L.code), (L.n + 2) * sizeof(uint16_t)});
                for (float** p : {&L.r, &L.zp, &L.t}) slots.push_back({reinterpret_cast<void**>(p), L.n * sizeof(float)});
            }
            lx = (lx + 1) / 2;
            ly = (ly + 1) / 2;
            lz = (lz + 1) / 2;
        }
        // block levels: the coarsest levels of at most kMgBlockLevelCells cells whose arrays fit kMgBlockBytes
        mg.grid_levels = mg.levels - 1;
        uint32_t block_words = 0;
        for (int l = mg.levels - 1; l >= 1; --l) {
            block_words += mg_block_words(mg.L[l].n);
            if (mg.L[l].n > kMgBlockLevelCells || block_words * 4u > kMgBlockBytes) break;
            mg.grid_levels = l;
        }
        auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
        size_t total = 0;
        for (const Slot& s : slots) total += align(s.bytes);
        check(cudaMalloc(&arena, total), "cudaMalloc arena");
        arena_bytes = total;
        size_t off = 0;
        for (const Slot& s : slots) {
            *s.ptr = static_cast<char*>(arena) + off;
            off += align(s.bytes);
        }
        MgLevel& L0 = mg.L[0];
        L0.code = codes;
        L0.r = pcg.r[0];
        L0.zp = pcg.r[1];
        L0.t = pcg.w[0];
        mg_work.r[0] = pcg.r[0];
        mg_work.r[1] = pcg.p;
        mg_work.p[0] = pcg.s[0];
        mg_work.p[1] = pcg.s[1];
        mg_work.q = pcg.w[1];
        mg_work.e = pcg.e;
        mg_work.x64 = pcg.x64;
    }

    // Occupancy-derived data: anchor, operator codes, density fill list, float occupancy view.
    void rebuild_occupancy_data() {
        check(launch_occupancy_float(P, occupancy, occupancy_float, stream), "occupancy view");
        check(launch_anchor(P, occupancy, anchor, stream), "pressure anchor");
        check(launch_stencil_codes(P, occupancy, anchor, codes, stream), "operator codes");
        check(launch_fill_build(P, occupancy, anchor, fill_list, fill_count, stream), "density fill list");
        check(launch_mg_setup(P, mg, occupancy, stream), "multigrid levels");
        if (has_net) check(launch_mg_net_mask(mg, learned.occupancy, stream), "preconditioner network mask");
    }

    // The pressure solve of the selected mode on the context's right-hand side. The multigrid solve is a graph:
    // recorded into the capture when `s` is capturing, else launched as the prebuilt solve graph.
    void enqueue_solve(cudaStream_t s, bool capturing) {
        const PcgSettings S = pcg_settings();
        if (!uses_mg()) {
            check(launch_pcg(P, S, pcg_shape, codes, rhs, pressure, pcg, control, s), "pressure solve");
            return;
        }
        if (!capturing) {
            check(cudaGraphLaunch(solve_exec, s), "pressure solve (multigrid FCG graph)");
            return;
        }
        check(enqueue_mg_solve(mg_args(S), S.fp64 != 0, &control->status, s, body_stream), "pressure solve (multigrid FCG)");
    }

    // The same solve with every kernel launched directly (the multigrid loop driven from the host).
    void run_solve_eager(cudaStream_t s) {
        const PcgSettings S = pcg_settings();
        if (!uses_mg()) {
            check(launch_pcg(P, S, pcg_shape, codes, rhs, pressure, pcg, control, s), "pressure solve");
            return;
        }
        check(run_mg_solve_eager(mg_args(S), S.fp64 != 0, &control->status, s), "pressure solve (multigrid FCG, eager)");
    }

    MgSolveArgs mg_args(const PcgSettings& S) const {
        MgSolveArgs A{};
        A.H = mg;
        A.W = mg_work;
        A.b = rhs;
        A.x = pressure;
        A.ir = S.refinement > 0 ? 1 : 0;
        A.e = A.ir ? mg_work.e : pressure;
        A.st = mg_state;
        A.warm = A.ir && S.warm_start ? 1 : 0;
        A.max_iterations = S.max_iterations;
        A.refinement = S.refinement < mg_max_refinement() ? S.refinement : mg_max_refinement();
        A.tol = S.tolerance;
        A.wave = static_cast<int>(tune.mg_wave);
        A.learned = solver.mode == SMOKE_B200_SOLVER_LEARNED_FCG ? 1 : 0;
        A.net = A.learned ? &learned : nullptr;
        A.net_warm = A.learned && A.warm && solver.warm_start == 2 ? 1 : 0;
        A.net_iterations = static_cast<int>(net_iterations);
        return A;
    }

    // The multigrid FCG machinery runs the multigrid and the learned solves.
    uint32_t net_iterations = 0;  // learned solve: network iterations per refinement pass (0: all)

    bool uses_mg() const { return solver.mode == SMOKE_B200_SOLVER_MG_FCG || solver.mode == SMOKE_B200_SOLVER_LEARNED_FCG; }

    // The context's copy of a network: its packed images, an activation workspace on the multigrid level 1 (where the
    // network runs), that level's solid mask and a level-0 array for the prolonged correction.
    void set_net(const SmokeB200Net_t* net) {
        const VolumeDims d = volume_dims(mg.L[1].nx, mg.L[1].ny, mg.L[1].nz);
        auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
        const size_t ib = align(net_images_bytes()), ab = align(net_acts_bytes(d)), fb = align(static_cast<size_t>(P.n) * sizeof(float));
        const size_t need = ib + ab + fb + align(d.n);
        check(cudaStreamSynchronize(stream), "preconditioner network: idle");
        if (need > learned_bytes) {
            if (learned_mem) check(cudaFree(learned_mem), "preconditioner network");
            learned_mem = nullptr;
            learned_bytes = 0;
            check(cudaMalloc(&learned_mem, need), "preconditioner network");
            learned_bytes = need;
        }
        check(cudaMemcpy(learned_mem, smoke_b200_net_images_block(net), net_images_bytes(), cudaMemcpyDeviceToDevice), "preconditioner network");
        net_images_bind(learned.images, learned_mem);
        char* base = static_cast<char*>(learned_mem);
        net_acts_bind(learned.acts, base + ib, d);
        learned.fine = reinterpret_cast<float*>(base + ib + ab);
        learned.occupancy = reinterpret_cast<uint8_t*>(base + ib + ab + fb);
        check(cudaMemset(learned.acts.error, 0, sizeof(unsigned)), "preconditioner network");
        check(launch_mg_net_mask(mg, learned.occupancy, stream), "preconditioner network mask");
        has_net = true;
    }

    // Launch shapes: takes effect in the step graph, which is recaptured.
    void apply_tune(const SmokeB200LaunchTune& t) {
        if (!valid_tune(t)) throw std::invalid_argument("launch tune");
        tune = t;
        set_advect_tile(P, static_cast<int>(t.advect_tile));
        pcg_shape.grid = static_cast<int>(t.pcg_grid);
        pcg_shape.regs = static_cast<int>(t.pcg_regs);
        capture_step_graph();
    }
    static bool valid_tune(const SmokeB200LaunchTune& t) {
        return t.advect_tile < static_cast<uint32_t>(kAdvectTileCount) && t.mg_wave < static_cast<uint32_t>(kMgWaveCount) && t.pcg_grid < static_cast<uint32_t>(kPcgGridCount) && t.pcg_regs < static_cast<uint32_t>(kPcgRegsCount);
    }

    PcgSettings pcg_settings() const {
        PcgSettings S{};
        const bool fixed = solver.mode == SMOKE_B200_SOLVER_FIXED_CG;
        S.jacobi = fixed ? 0 : 1;
        S.fp64 = solver.reduction == SMOKE_B200_REDUCTION_FP64;
        S.fixed = fixed ? 1 : 0;
        S.max_iterations = fixed ? config.pressure_iterations : solver.max_iterations;
        S.tolerance = solver.tolerance;
        S.refinement = fixed ? 0 : static_cast<int32_t>(solver.refinement);
        S.warm_start = solver.warm_start ? 1 : 0;
        return S;
    }

    // The ghost cells of the velocity's padded copies (the producing kernel wrote their interiors).
    cudaError_t pad_velocity(ConstFaces v, cudaStream_t s) {
        const int kinds[3] = {0, 1, 2};
        const float* fields[3] = {v.u, v.v, v.w};
        float* pads[3] = {pad.u, pad.v, pad.w};
        return launch_pads(P, 3, kinds, fields, pads, s, 1);
    }

    // Stages of one step, in the reference's order (backend-cuda.cu:2000-2057, views excluded).
    void enqueue_stages(cudaStream_t s, uint32_t last_stage, bool capturing) {
        const ConstFaces solid{solid_vx, solid_vy, solid_vz};
        check(launch_vorticity(P, as_const(A), occupancy, wx, wy, wz, wmag, s), "vorticity");
        // the force kernel also forms the scalar stage's sourced temperature and density (neither changes before that
        // stage) with their padded copies' interiors; the face kernels write the velocity's padded copies' interiors
        const ScalarSources sources{temperature_source, density_source, solid_temperature, temperature_tmp, density_tmp, pad_t, pad_d};
        check(launch_cell_force(P, wx, wy, wz, wmag, density, temperature, force_x, force_y, force_z, occupancy, fx, fy, fz, s, sources), "cell force");
        check(launch_face_force(P, as_const(A), fx, fy, fz, occupancy, solid, B, s, pad), "face force");
        if (last_stage < SMOKE_B200_STAGE_ADVECT_VELOCITY) return;
        check(pad_velocity(as_const(B), s), "pad velocity");
        check(launch_advect_velocity(P, as_const(B), as_const(pad), occupancy, solid, C, s), "advect velocity");
        if (last_stage < SMOKE_B200_STAGE_PRESSURE) return;
        check(launch_rhs(P, as_const(C), occupancy, anchor, rhs, s), "pressure rhs");
        enqueue_solve(s, capturing);
        if (last_stage < SMOKE_B200_STAGE_PROJECT) return;
        const PcgSettings S = pcg_settings();
        const double* p64 = (!S.fixed && S.refinement > 0) ? pcg.x64 : nullptr;
        check(launch_project(P, as_const(C), pressure, p64, occupancy, solid, A, s, pad), "project");
        if (last_stage < SMOKE_B200_STAGE_SCALARS) return;
        check(pad_velocity(as_const(A), s), "pad velocity");
        {
            const int kinds[2] = {4, 3};
            const float* fields[2] = {temperature_tmp, density_tmp};
            float* pads[2] = {pad_t, pad_d};
            check(launch_pads(P, 2, kinds, fields, pads, s, 1), "pad scalars");
        }
        check(launch_advect_scalars(P, as_const(A), as_const(pad), occupancy, temperature_tmp, pad_t, density_tmp, pad_d, solid_temperature, temperature, density, s), "advect scalars");
        check(launch_density_fill(fill_list, fill_count, density, fill_blocks, s), "density fill");
    }

    void capture_step_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        check(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal), "begin step capture");
        try {
            enqueue_stages(capture_stream, SMOKE_B200_STAGE_SCALARS, true);
        } catch (...) {
            cudaGraph_t broken = nullptr;
            cudaStreamEndCapture(capture_stream, &broken);
            if (broken) cudaGraphDestroy(broken);
            throw;
        }
        check(cudaStreamEndCapture(capture_stream, &graph), "end step capture");
        check(cudaGraphInstantiate(&exec, graph, 0), "instantiate step graph");
        if (solve_exec) cudaGraphExecDestroy(solve_exec);
        solve_exec = nullptr;
        if (!uses_mg()) return;
        cudaGraph_t solve_graph = nullptr;
        check(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal), "begin solve capture");
        try {
            enqueue_solve(capture_stream, true);
        } catch (...) {
            cudaGraph_t broken = nullptr;
            cudaStreamEndCapture(capture_stream, &broken);
            if (broken) cudaGraphDestroy(broken);
            throw;
        }
        check(cudaStreamEndCapture(capture_stream, &solve_graph), "end solve capture");
        const cudaError_t e = cudaGraphInstantiate(&solve_exec, solve_graph, 0);
        cudaGraphDestroy(solve_graph);
        check(e, "instantiate solve graph");
    }

    void materialise_views(uint32_t groups = kViewsAll) {
        const uint32_t todo = views_stale & groups;
        if (!todo) return;
        check(launch_views(P, as_const(A), occupancy, cx, cy, cz, vmag, wx, wy, wz, wmag, divergence, todo, stream), "views");
        views_stale &= ~todo;
    }
};

// A batch of contexts advanced by one graph launch: the step of every context, recorded into one graph by stream
// capture with one branch per context (each context's capture stream), branches independent of one another.
struct SmokeB200Batch_t {
    std::vector<SmokeSimulationContext_t*> contexts;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> ready;     // one per context: the context's stream reached the batch step
    cudaEvent_t done = nullptr;         // the batch step finished
    // globaltimer stamps written by the graph: [0] when the batch step starts, [1 + i] when member i's step is done
    unsigned long long* stamps = nullptr;

    ~SmokeB200Batch_t() {
        if (exec) cudaGraphExecDestroy(exec);
        for (cudaEvent_t e : ready) cudaEventDestroy(e);
        if (stamps) cudaFree(stamps);
        if (done) cudaEventDestroy(done);
        if (owns_stream && stream) cudaStreamDestroy(stream);
    }

    void build() {
        const cudaStream_t root = contexts.front()->capture_stream;
        cudaEvent_t fork = nullptr;
        check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "batch fork event");
        std::vector<cudaEvent_t> joins(contexts.size(), nullptr);
        cudaGraph_t graph = nullptr;
        cudaError_t err = cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal);
        try {
            check(err, "begin batch capture");
            check(launch_time_stamp(stamps, root), "batch start time");
            check(cudaEventRecord(fork, root), "batch fork");
            for (size_t i = 0; i < contexts.size(); ++i) {
                SmokeSimulationContext_t* c = contexts[i];
                if (i > 0) check(cudaStreamWaitEvent(c->capture_stream, fork, 0), "batch branch");
                c->enqueue_stages(c->capture_stream, SMOKE_B200_STAGE_SCALARS, true);
                check(launch_time_stamp(stamps + 1 + i, c->capture_stream), "batch member time");
                if (i > 0) {
                    check(cudaEventCreateWithFlags(&joins[i], cudaEventDisableTiming), "batch join event");
                    check(cudaEventRecord(joins[i], c->capture_stream), "batch join");
                    check(cudaStreamWaitEvent(root, joins[i], 0), "batch join");
                }
            }
            check(cudaStreamEndCapture(root, &graph), "end batch capture");
        } catch (...) {
            if (err == cudaSuccess) {
                cudaGraph_t broken = nullptr;
                cudaStreamEndCapture(root, &broken);
                if (broken) cudaGraphDestroy(broken);
            }
            cudaEventDestroy(fork);
            for (cudaEvent_t e : joins)
                if (e) cudaEventDestroy(e);
            throw;
        }
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        cudaEventDestroy(fork);
        for (cudaEvent_t e : joins)
            if (e) cudaEventDestroy(e);
        check(ie, "instantiate batch graph");
    }
};

namespace {

SmokeSimulationResult ok_or_fail(cudaError_t e) { return e == cudaSuccess ? SMOKE_SIMULATION_RESULT_OK : SMOKE_SIMULATION_RESULT_BACKEND_FAILURE; }

template <class F>
SmokeSimulationResult guarded(F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return SMOKE_SIMULATION_RESULT_OUT_OF_MEMORY;
    } catch (...) {
        return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    }
}

cudaError_t copy_or_zero(float* dst, const float* src, size_t count, cudaStream_t s) {
    if (src == nullptr) return cudaMemsetAsync(dst, 0, count * sizeof(float), s);
    return cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyDeviceToDevice, s);
}

// ---------------------------------------------------------------------------------------------- autotuner
// Tuned shapes, per process: (device, nx, ny, nz, cubic, solver mode, reduction, refinement, max iterations,
// tolerance bits).
using TuneKey = std::tuple<int, int, int, int, int, uint32_t, uint32_t, uint32_t, int32_t, uint32_t>;
std::mutex tune_lock;
std::map<TuneKey, SmokeB200LaunchTune> tune_cache;

TuneKey tune_key(const SmokeSimulationContext_t& c) {
    int dev = 0;
    check(cudaGetDevice(&dev), "device");
    uint32_t tol_bits = 0;
    std::memcpy(&tol_bits, &c.solver.tolerance, sizeof(tol_bits));
    const bool fixed = c.solver.mode == SMOKE_B200_SOLVER_FIXED_CG;
    return TuneKey{dev, c.P.nx, c.P.ny, c.P.nz, c.P.cubic, c.solver.mode, c.solver.reduction, fixed ? 0u : c.solver.refinement, fixed ? c.config.pressure_iterations : c.solver.max_iterations, fixed ? 0u : tol_bits};
}

// Device buffer freed on scope exit.
struct DeviceBuffer {
    void* p = nullptr;
    ~DeviceBuffer() {
        if (p) cudaFree(p);
    }
};
struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

// Times `steps` graph steps of `c` under shapes `t`, each repeat from the state saved in `snapshot`.
SmokeB200TuneRecord time_candidate(SmokeSimulationContext_t& c, const SmokeB200LaunchTune& t, uint32_t steps, const void* snapshot, Events& ev) {
    const cudaStream_t s = c.stream;
    check(cudaStreamSynchronize(s), "tune: idle");
    c.apply_tune(t);
    auto restore = [&] { check(cudaMemcpyAsync(c.arena, snapshot, c.arena_bytes, cudaMemcpyDeviceToDevice, s), "tune: restore state"); };
    restore();
    check(cudaGraphLaunch(c.exec, s), "tune: untimed step");
    SmokeB200TuneRecord r{};
    r.tune = t;
    r.ms_per_step = std::numeric_limits<float>::infinity();
    for (int rep = 0; rep < 2; ++rep) {
        restore();
        check(cudaEventRecord(ev.a, s), "tune: event");
        for (uint32_t i = 0; i < steps; ++i) check(cudaGraphLaunch(c.exec, s), "tune: timed step");
        check(cudaEventRecord(ev.b, s), "tune: event");
        check(cudaEventSynchronize(ev.b), "tune: timed steps");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, ev.a, ev.b), "tune: elapsed");
        r.ms_per_step = std::min(r.ms_per_step, ms / static_cast<float>(steps));
    }
    PcgStatusDevice st{};
    check(cudaMemcpy(&st, &c.control->status, sizeof(st), cudaMemcpyDeviceToHost), "tune: status");
    r.iterations = st.iterations;
    return r;
}

}  // namespace

extern "C" {

SmokeSimulationResult smoke_simulation_create_context_cuda(const SmokeSimulationContextCreateDesc* desc, SmokeSimulationContext* out_context) {
    nvtx3::scoped_range range("smoke_b200.create_context");
    if (desc == nullptr || out_context == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (!valid_config(desc->config)) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    *out_context = nullptr;
    std::unique_ptr<SmokeSimulationContext_t> ctx(new (std::nothrow) SmokeSimulationContext_t{});
    if (!ctx) return SMOKE_SIMULATION_RESULT_OUT_OF_MEMORY;
    const SmokeSimulationResult r = guarded([&] {
        ctx->config = desc->config;
        ctx->P = make_params(desc->config);
        ctx->stream = static_cast<cudaStream_t>(desc->stream);
        if (ctx->stream == nullptr) {
            check(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "create stream");
            ctx->owns_stream = true;
        }
        check(cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking), "create capture stream");
        check(cudaStreamCreateWithFlags(&ctx->body_stream, cudaStreamNonBlocking), "create graph body stream");
        int dev = 0, sms = 0;
        check(cudaGetDevice(&dev), "device");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        ctx->fill_blocks = sms * 4;
        check(pcg_launch_shape(&ctx->pcg_shape), "solver launch shape");
        ctx->allocate();
        cudaStream_t s = ctx->stream;
        check(cudaMemsetAsync(ctx->arena, 0, ctx->arena_bytes, s), "zero arena");
        check(launch_fill_value(ctx->density, desc->initial_density, ctx->P.n, s), "initial density");
        check(launch_fill_value(ctx->temperature, desc->initial_temperature, ctx->P.n, s), "initial temperature");
        check(launch_fill_value(ctx->solid_temperature, desc->config.ambient_temperature, ctx->P.n, s), "solid temperature");
        ctx->rebuild_occupancy_data();
        // the capture stream must not start before the arena is initialised
        check(cudaStreamSynchronize(s), "initialise context");
        ctx->capture_step_graph();
        return SMOKE_SIMULATION_RESULT_OK;
    });
    if (r != SMOKE_SIMULATION_RESULT_OK) return r;
    *out_context = ctx.release();
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_simulation_destroy_context_cuda(SmokeSimulationContext context) {
    nvtx3::scoped_range range("smoke_b200.destroy_context");
    if (context == nullptr) return SMOKE_SIMULATION_RESULT_OK;
    if (context->stream) cudaStreamSynchronize(context->stream);
    delete context;
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_simulation_update_density_cuda(SmokeSimulationContext c, const float* values) {
    nvtx3::scoped_range range("smoke_b200.update_density");
    return ok_or_fail(copy_or_zero(c->density, values, c->P.n, c->stream));
}

SmokeSimulationResult smoke_simulation_update_density_source_cuda(SmokeSimulationContext c, const float* values) {
    nvtx3::scoped_range range("smoke_b200.update_density_source");
    return ok_or_fail(copy_or_zero(c->density_source, values, c->P.n, c->stream));
}

SmokeSimulationResult smoke_simulation_update_temperature_cuda(SmokeSimulationContext c, const float* values) {
    nvtx3::scoped_range range("smoke_b200.update_temperature");
    return ok_or_fail(copy_or_zero(c->temperature, values, c->P.n, c->stream));
}

SmokeSimulationResult smoke_simulation_update_temperature_source_cuda(SmokeSimulationContext c, const float* values) {
    nvtx3::scoped_range range("smoke_b200.update_temperature_source");
    return ok_or_fail(copy_or_zero(c->temperature_source, values, c->P.n, c->stream));
}

SmokeSimulationResult smoke_simulation_update_force_cuda(SmokeSimulationContext c, const float* x, const float* y, const float* z) {
    nvtx3::scoped_range range("smoke_b200.update_force");
    if (copy_or_zero(c->force_x, x, c->P.n, c->stream) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (copy_or_zero(c->force_y, y, c->P.n, c->stream) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return ok_or_fail(copy_or_zero(c->force_z, z, c->P.n, c->stream));
}

SmokeSimulationResult smoke_simulation_update_occupancy_cuda(SmokeSimulationContext c, const uint8_t* values) {
    nvtx3::scoped_range range("smoke_b200.update_occupancy");
    return guarded([&] {
        c->materialise_views();  // derived views keep showing the state right after the last step
        if (values == nullptr) check(cudaMemsetAsync(c->occupancy, 0, c->P.n, c->stream), "clear occupancy");
        else check(cudaMemcpyAsync(c->occupancy, values, c->P.n, cudaMemcpyDeviceToDevice, c->stream), "copy occupancy");
        c->rebuild_occupancy_data();
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_simulation_update_solid_velocity_cuda(SmokeSimulationContext c, const float* x, const float* y, const float* z) {
    nvtx3::scoped_range range("smoke_b200.update_solid_velocity");
    if (copy_or_zero(c->solid_vx, x, c->P.n, c->stream) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (copy_or_zero(c->solid_vy, y, c->P.n, c->stream) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return ok_or_fail(copy_or_zero(c->solid_vz, z, c->P.n, c->stream));
}

SmokeSimulationResult smoke_simulation_update_solid_temperature_cuda(SmokeSimulationContext c, const float* values) {
    nvtx3::scoped_range range("smoke_b200.update_solid_temperature");
    if (values == nullptr) return ok_or_fail(launch_fill_value(c->solid_temperature, c->config.ambient_temperature, c->P.n, c->stream));
    return ok_or_fail(cudaMemcpyAsync(c->solid_temperature, values, c->P.n * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
}

SmokeSimulationResult smoke_simulation_step_cuda(SmokeSimulationContext c) {
    nvtx3::scoped_range range("smoke_b200.step");
    if (c == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (cudaGraphLaunch(c->exec, c->stream) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    c->views_stale = kViewsAll;
    c->stepped = true;
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_simulation_get_view_cuda(SmokeSimulationContext c, const SmokeSimulationViewRequest* request, SmokeSimulationView* out) {
    nvtx3::scoped_range range("smoke_b200.get_view");
    if (c == nullptr || request == nullptr || out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    *out = SmokeSimulationView{};
    out->layout = SMOKE_SIMULATION_VIEW_LAYOUT_F32_3D;
    out->nx = c->config.nx;
    out->ny = c->config.ny;
    out->nz = c->config.nz;
    out->row_stride_bytes = static_cast<uint64_t>(c->config.nx) * sizeof(float);
    out->slice_stride_bytes = static_cast<uint64_t>(c->config.nx) * static_cast<uint64_t>(c->config.ny) * sizeof(float);
    auto one = [&](const float* p) { out->data0 = p; };
    auto three = [&](const float* a, const float* b, const float* d) {
        out->layout = SMOKE_SIMULATION_VIEW_LAYOUT_F32_3D_SOA3;
        out->data0 = a;
        out->data1 = b;
        out->data2 = d;
    };
    const SmokeSimulationResult r = guarded([&] {
        switch (request->kind) {
        case SMOKE_SIMULATION_VIEW_DENSITY: one(c->density); break;
        case SMOKE_SIMULATION_VIEW_DENSITY_SOURCE: one(c->density_source); break;
        case SMOKE_SIMULATION_VIEW_TEMPERATURE: one(c->temperature); break;
        case SMOKE_SIMULATION_VIEW_TEMPERATURE_SOURCE: one(c->temperature_source); break;
        case SMOKE_SIMULATION_VIEW_FORCE: three(c->force_x, c->force_y, c->force_z); break;
        case SMOKE_SIMULATION_VIEW_SOLID_VELOCITY: three(c->solid_vx, c->solid_vy, c->solid_vz); break;
        case SMOKE_SIMULATION_VIEW_SOLID_TEMPERATURE: one(c->solid_temperature); break;
        case SMOKE_SIMULATION_VIEW_FLOW_VELOCITY: c->materialise_views(kViewsVelocity); three(c->cx, c->cy, c->cz); break;
        case SMOKE_SIMULATION_VIEW_FLOW_VELOCITY_MAGNITUDE: c->materialise_views(kViewsVelocity); one(c->vmag); break;
        case SMOKE_SIMULATION_VIEW_FLOW_PRESSURE: one(c->pressure); break;
        case SMOKE_SIMULATION_VIEW_FLOW_PRESSURE_RHS: one(c->rhs); break;
        case SMOKE_SIMULATION_VIEW_FLOW_DIVERGENCE: c->materialise_views(kViewsVorticity); one(c->divergence); break;
        case SMOKE_SIMULATION_VIEW_FLOW_VORTICITY: c->materialise_views(kViewsVorticity); three(c->wx, c->wy, c->wz); break;
        case SMOKE_SIMULATION_VIEW_FLOW_VORTICITY_MAGNITUDE: c->materialise_views(kViewsVorticity); one(c->wmag); break;
        case SMOKE_SIMULATION_VIEW_OCCUPANCY: one(c->occupancy_float); break;
        default: return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
        }
        return SMOKE_SIMULATION_RESULT_OK;
    });
    if (r != SMOKE_SIMULATION_RESULT_OK) return r;
    // order a foreign consumer stream after the context stream (backend-cuda.cu:2189-2205)
    if (request->consumer_stream == nullptr) return SMOKE_SIMULATION_RESULT_OK;
    auto consumer = static_cast<cudaStream_t>(request->consumer_stream);
    if (consumer == c->stream) return SMOKE_SIMULATION_RESULT_OK;
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const bool ok = cudaEventRecord(ev, c->stream) == cudaSuccess && cudaStreamWaitEvent(consumer, ev, 0) == cudaSuccess;
    cudaEventDestroy(ev);
    return ok ? SMOKE_SIMULATION_RESULT_OK : SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
}

// ---------------------------------------------------------------------------------------------- extensions
SmokeSimulationResult smoke_b200_set_solver_cuda(SmokeSimulationContext c, const SmokeB200SolverDesc* desc) {
    if (c == nullptr || desc == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (desc->mode > SMOKE_B200_SOLVER_LEARNED_FCG || desc->reduction > SMOKE_B200_REDUCTION_FP64) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (desc->mode == SMOKE_B200_SOLVER_LEARNED_FCG && !c->has_net) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (desc->warm_start > (desc->mode == SMOKE_B200_SOLVER_LEARNED_FCG ? 2u : 1u)) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (desc->mode != SMOKE_B200_SOLVER_FIXED_CG && (desc->max_iterations <= 0 || !(desc->tolerance > 0.0f))) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->solver = *desc;
        c->capture_step_graph();
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_get_solver_status_cuda(SmokeSimulationContext c, SmokeB200SolverStatus* out) {
    if (c == nullptr || out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (!c->stepped) {
        *out = SmokeB200SolverStatus{};
        out->status = SMOKE_B200_SOLVE_NOT_RUN;
        out->true_relative_residual = -1.0;
        return SMOKE_SIMULATION_RESULT_OK;
    }
    PcgStatusDevice st{};
    if (cudaMemcpyAsync(&st, &c->control->status, sizeof(st), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    std::memcpy(out, &st, sizeof(st));
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_set_face_velocity_cuda(SmokeSimulationContext c, const float* u, const float* v, const float* w) {
    if (c == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->materialise_views();
        check(copy_or_zero(c->A.u, u, c->P.nu, c->stream), "set u");
        check(copy_or_zero(c->A.v, v, c->P.nv, c->stream), "set v");
        check(copy_or_zero(c->A.w, w, c->P.nw, c->stream), "set w");
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_get_face_velocity_cuda(SmokeSimulationContext c, uint32_t which, const float** u, const float** v, const float** w) {
    if (c == nullptr || u == nullptr || v == nullptr || w == nullptr || which > 2) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const Faces& f = which == 0 ? c->A : (which == 1 ? c->C : c->B);
    *u = f.u;
    *v = f.v;
    *w = f.w;
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_step_stages_cuda(SmokeSimulationContext c, uint32_t last_stage) {
    if (c == nullptr || last_stage > SMOKE_B200_STAGE_SCALARS) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->enqueue_stages(c->stream, last_stage, false);
        c->views_stale = kViewsAll;
        c->stepped = true;
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_test_barrier_timeout_cuda(SmokeSimulationContext c, uint32_t block, uint32_t timeout_ms, SmokeB200SolverStatus* out_status) {
    if (c == nullptr || out_status == nullptr || block == 0 || timeout_ms == 0 || timeout_ms > 10000 || c->uses_mg()) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        PcgSettings S = c->pcg_settings();
        S.withhold_block = static_cast<int32_t>(block) + 1;
        S.barrier_timeout_ms = timeout_ms;
        check(launch_pcg(c->P, S, c->pcg_shape, c->codes, c->rhs, c->pressure, c->pcg, c->control, c->stream), "pressure solve with a withheld block");
        c->stepped = true;
        PcgStatusDevice st{};
        check(cudaMemcpyAsync(&st, &c->control->status, sizeof(st), cudaMemcpyDeviceToHost, c->stream), "status read-back");
        check(cudaStreamSynchronize(c->stream), "status read-back");
        std::memcpy(out_status, &st, sizeof(st));
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_solve_pressure_cuda(SmokeSimulationContext c) {
    if (c == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->enqueue_solve(c->stream, false);
        c->stepped = true;
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_batch_create_cuda(const SmokeSimulationContext* contexts, uint32_t count, void* stream, SmokeB200Batch* out_batch) {
    if (contexts == nullptr || out_batch == nullptr || count == 0) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    *out_batch = nullptr;
    for (uint32_t i = 0; i < count; ++i) {
        if (contexts[i] == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
        for (uint32_t j = 0; j < i; ++j)
            if (contexts[j] == contexts[i]) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    }
    std::unique_ptr<SmokeB200Batch_t> b(new (std::nothrow) SmokeB200Batch_t{});
    if (!b) return SMOKE_SIMULATION_RESULT_OUT_OF_MEMORY;
    const SmokeSimulationResult r = guarded([&] {
        b->contexts.assign(contexts, contexts + count);
        b->stream = static_cast<cudaStream_t>(stream);
        if (b->stream == nullptr) {
            check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch stream");
            b->owns_stream = true;
        }
        b->ready.assign(count, nullptr);
        for (cudaEvent_t& e : b->ready) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
        check(cudaMalloc(&b->stamps, (count + 1) * sizeof(unsigned long long)), "batch time stamps");
        check(cudaMemset(b->stamps, 0, (count + 1) * sizeof(unsigned long long)), "batch time stamps");
        check(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "batch event");
        for (SmokeSimulationContext_t* c : b->contexts) check(cudaStreamSynchronize(c->stream), "batch: contexts idle");
        b->build();
        return SMOKE_SIMULATION_RESULT_OK;
    });
    if (r != SMOKE_SIMULATION_RESULT_OK) return r;
    *out_batch = b.release();
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_batch_step_cuda(SmokeB200Batch batch) {
    if (batch == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        for (size_t i = 0; i < batch->contexts.size(); ++i) {
            SmokeSimulationContext_t* c = batch->contexts[i];
            check(cudaEventRecord(batch->ready[i], c->stream), "batch step: context ready");
            check(cudaStreamWaitEvent(batch->stream, batch->ready[i], 0), "batch step: wait");
        }
        check(cudaGraphLaunch(batch->exec, batch->stream), "batch step");
        check(cudaEventRecord(batch->done, batch->stream), "batch step: done");
        for (SmokeSimulationContext_t* c : batch->contexts) {
            check(cudaStreamWaitEvent(c->stream, batch->done, 0), "batch step: order the context");
            c->views_stale = kViewsAll;
            c->stepped = true;
        }
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_batch_member_times_cuda(SmokeB200Batch batch, float* ms_out) {
    if (batch == nullptr || ms_out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        check(cudaEventSynchronize(batch->done), "batch member times: wait");
        std::vector<unsigned long long> t(batch->contexts.size() + 1);
        check(cudaMemcpy(t.data(), batch->stamps, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost), "batch member times");
        for (size_t i = 0; i < batch->contexts.size(); ++i) ms_out[i] = static_cast<float>(static_cast<double>(t[i + 1] - t[0]) * 1e-6);
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_batch_destroy_cuda(SmokeB200Batch batch) {
    if (batch == nullptr) return SMOKE_SIMULATION_RESULT_OK;
    if (batch->stream) cudaStreamSynchronize(batch->stream);
    delete batch;
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_apply_operator_cuda(SmokeSimulationContext c, const float* x, float* out) {
    if (c == nullptr || x == nullptr || out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return ok_or_fail(launch_mg_apply(c->mg, x, out, c->stream));
}

SmokeSimulationResult smoke_b200_apply_multigrid_cuda(SmokeSimulationContext c, const float* r, float* z) {
    if (c == nullptr || r == nullptr || z == nullptr || r == z) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return ok_or_fail(launch_mg_vcycle(c->mg, static_cast<int>(c->tune.mg_wave), r, z, c->stream));
}

SmokeSimulationResult smoke_b200_set_learned_iterations_cuda(SmokeSimulationContext c, uint32_t count) {
    if (c == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->net_iterations = count;
        c->capture_step_graph();
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_set_preconditioner_net_cuda(SmokeSimulationContext c, SmokeB200Net net) {
    if (c == nullptr || net == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->set_net(net);
        c->capture_step_graph();
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_set_launch_tune_cuda(SmokeSimulationContext c, const SmokeB200LaunchTune* tune) {
    if (c == nullptr || tune == nullptr || !SmokeSimulationContext_t::valid_tune(*tune)) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->apply_tune(*tune);
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_get_launch_tune_cuda(SmokeSimulationContext c, SmokeB200LaunchTune* out) {
    if (c == nullptr || out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    *out = c->tune;
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_autotune_cuda(SmokeSimulationContext c, uint32_t steps, uint32_t flags, SmokeB200TuneReport* report) {
    nvtx3::scoped_range range("smoke_b200.autotune");
    if (c == nullptr || steps > 64 || (flags & ~SMOKE_B200_TUNE_FORCE) != 0) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (steps == 0) steps = 4;
    return guarded([&] {
        SmokeB200TuneReport rep{};
        const TuneKey key = tune_key(*c);
        if (!(flags & SMOKE_B200_TUNE_FORCE)) {
            std::lock_guard<std::mutex> guard(tune_lock);
            auto it = tune_cache.find(key);
            if (it != tune_cache.end()) {
                c->apply_tune(it->second);
                rep.chosen = it->second;
                rep.from_cache = 1;
                if (report) *report = rep;
                return SMOKE_SIMULATION_RESULT_OK;
            }
        }
        const cudaStream_t s = c->stream;
        check(cudaStreamSynchronize(s), "tune: idle");
        const uint32_t views_stale = c->views_stale;
        const bool stepped = c->stepped;
        const SmokeB200LaunchTune start = c->tune;
        DeviceBuffer snap;
        check(cudaMalloc(&snap.p, c->arena_bytes), "tune: state copy");
        check(cudaMemcpyAsync(snap.p, c->arena, c->arena_bytes, cudaMemcpyDeviceToDevice, s), "tune: save state");
        Events ev;
        check(cudaEventCreate(&ev.a), "tune: event");
        check(cudaEventCreate(&ev.b), "tune: event");
        auto record = [&](const SmokeB200TuneRecord& r) {
            if (rep.record_count < SMOKE_B200_TUNE_MAX_RECORDS) rep.records[rep.record_count++] = r;
        };
        try {
            SmokeB200TuneRecord best = time_candidate(*c, start, steps, snap.p, ev);
            record(best);
            rep.default_ms = best.ms_per_step;
            // a candidate replaces the best only when it is at least 1% faster (timing noise)
            auto consider = [&](SmokeB200LaunchTune t) {
                const SmokeB200TuneRecord r = time_candidate(*c, t, steps, snap.p, ev);
                record(r);
                if (r.ms_per_step < 0.99f * best.ms_per_step) best = r;
            };
            const SmokeB200LaunchTune base_tiles = best.tune;
            for (uint32_t v = 0; v < static_cast<uint32_t>(kAdvectTileCount); ++v)
                if (v != base_tiles.advect_tile) {
                    SmokeB200LaunchTune t = best.tune;
                    t.advect_tile = v;
                    consider(t);
                }
            const SmokeB200LaunchTune base_grid = best.tune;
            if (c->uses_mg()) {
                for (uint32_t v = 0; v < static_cast<uint32_t>(kMgWaveCount); ++v)
                    if (v != base_grid.mg_wave) {
                        SmokeB200LaunchTune t = best.tune;
                        t.mg_wave = v;
                        consider(t);
                    }
            } else {
                for (uint32_t v = 0; v < static_cast<uint32_t>(kPcgGridCount); ++v)
                    if (v != base_grid.pcg_grid) {
                        SmokeB200LaunchTune t = best.tune;
                        t.pcg_grid = v;
                        consider(t);
                    }
                const SmokeB200LaunchTune base_regs = best.tune;
                for (uint32_t v = 0; v < static_cast<uint32_t>(kPcgRegsCount); ++v)
                    if (v != base_regs.pcg_regs) {
                        SmokeB200LaunchTune t = best.tune;
                        t.pcg_regs = v;
                        consider(t);
                    }
            }
            check(cudaStreamSynchronize(s), "tune: idle");
            c->apply_tune(best.tune);
            rep.chosen = best.tune;
            rep.chosen_ms = best.ms_per_step;
        } catch (...) {
            // leave the context as it was: its shapes and its state
            cudaStreamSynchronize(s);
            try {
                c->apply_tune(start);
            } catch (...) {
            }
            cudaMemcpyAsync(c->arena, snap.p, c->arena_bytes, cudaMemcpyDeviceToDevice, s);
            cudaStreamSynchronize(s);
            throw;
        }
        check(cudaMemcpyAsync(c->arena, snap.p, c->arena_bytes, cudaMemcpyDeviceToDevice, s), "tune: restore state");
        check(cudaStreamSynchronize(s), "tune: restore state");
        c->views_stale = views_stale;
        c->stepped = stepped;
        {
            std::lock_guard<std::mutex> guard(tune_lock);
            tune_cache[key] = rep.chosen;
        }
        if (report) *report = rep;
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_solve_pressure_eager_cuda(SmokeSimulationContext c) {
    if (c == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        c->run_solve_eager(c->stream);
        c->stepped = true;
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

}  // extern "C"
