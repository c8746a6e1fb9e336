// Pressure solve that allocates nothing: smoke_b200_solve_pressure_noalloc_cuda.
//
// Some callers cannot call cudaMalloc while they run: a renderer or game engine that reserves all of its GPU
// memory up front and forbids allocations inside its frame loop (cudaMalloc may synchronise the device and stall
// the frame), a plug-in living inside another application's memory budget, or a process whose allocations are
// capped by a pool it does not own. For them this entry point solves the pressure system with scratch memory that
// is part of the library image itself: one file-scope device array of kNoAllocBytes bytes, sized for grids of up
// to kNoAllocMaxCells cells. Every GPU that loads the library holds that array until the process exits.
//
// The solve is the same persistent CG kernel as the context path (pcg.cu); only where its scratch lives differs.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "config_check.h"
#include "launch.h"
#include "smoke_b200_ext.h"

namespace smoke_b200 {
namespace {

constexpr uint64_t kNoAllocMaxCells = 64ull * 64ull * 64ull;
constexpr uint32_t kNoAllocMaxRefinement = 64;  // refinement passes accepted (each is one FP64 residual restart)
constexpr uint64_t align256(uint64_t v) { return (v + 255) & ~uint64_t(255); }

// Scratch layout: operator codes, anchor, occupancy (used when the caller passes none), 8 FP32 CG vectors,
// the FP64 solution accumulator, the solver control block.
constexpr uint64_t kOffCodes = 0;
constexpr uint64_t kOffAnchor = kOffCodes + align256((kNoAllocMaxCells + 2) * sizeof(uint16_t));  // codes carry 2 spare entries
constexpr uint64_t kOffOcc = kOffAnchor + 256;
constexpr uint64_t kOffVectors = kOffOcc + align256(kNoAllocMaxCells);
constexpr uint64_t kVectorBytes = align256(kNoAllocMaxCells * sizeof(float));
constexpr uint64_t kOffX64 = kOffVectors + 8 * kVectorBytes;
constexpr uint64_t kOffControl = kOffX64 + align256(kNoAllocMaxCells * sizeof(double));
constexpr uint64_t kNoAllocBytes = kOffControl + align256(sizeof(PcgControl));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

thread_local char g_last_error[256] = "";

void set_error(const char* msg) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

// Records `step` and the CUDA error text as the reason of this call's failure.
SmokeSimulationResult cuda_failure(const char* step, cudaError_t e) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s", step, cudaGetErrorString(e));
    return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
}

// Device address of the scratch array on the current device, looked up once per device.
unsigned char* scratch_for_current_device() {
    int dev = 0;
    const cudaError_t ed = cudaGetDevice(&dev);
    if (ed != cudaSuccess) {
        cuda_failure("cudaGetDevice", ed);
        return nullptr;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device ordinal beyond the 64 devices the scratch table covers");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[dev] == nullptr) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr) {
            cuda_failure("cudaGetSymbolAddress of the scratch array", e);
            return nullptr;
        }
        g_scratch_ptr[dev] = static_cast<unsigned char*>(ptr);
    }
    return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace smoke_b200

using namespace smoke_b200;

extern "C" {

SmokeSimulationResult smoke_b200_solve_pressure_noalloc_cuda(const SmokeSimulationConfig* config, const uint8_t* occupancy, const float* rhs, float* pressure, const SmokeB200SolverDesc* solver, void* stream,
                                                            SmokeB200SolverStatus* out_status) {
    g_last_error[0] = '\0';
    if (config == nullptr || rhs == nullptr || pressure == nullptr) {
        set_error("config, rhs and pressure must not be NULL");
        return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    }
    if (!valid_config(*config)) {  // the same configurations smoke_simulation_create_context_cuda refuses
        set_error("invalid configuration (extents, cell size, dt and pressure_iterations must be positive; boundary types in range; a periodic face only opposite a periodic face)");
        return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    }
    const uint64_t cells = static_cast<uint64_t>(config->nx) * config->ny * config->nz;
    if (cells > kNoAllocMaxCells) {
        std::snprintf(g_last_error, sizeof(g_last_error), "grid of %llu cells exceeds the no-allocation limit of %llu cells (64^3)", static_cast<unsigned long long>(cells),
                      static_cast<unsigned long long>(kNoAllocMaxCells));
        return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    }
    SmokeB200SolverDesc d{SMOKE_B200_SOLVER_FIXED_CG, SMOKE_B200_REDUCTION_FP32, 500, 1.0e-5f, 0, 0};
    if (solver != nullptr) d = *solver;
    if (d.mode > SMOKE_B200_SOLVER_JACOBI_PCG || d.reduction > SMOKE_B200_REDUCTION_FP64 || d.refinement > kNoAllocMaxRefinement ||
        (d.mode == SMOKE_B200_SOLVER_JACOBI_PCG && (d.max_iterations <= 0 || !(d.tolerance > 0.0f)))) {
        set_error("invalid solver description (mode FIXED_CG or JACOBI_PCG only, reduction FP32 or FP64, refinement <= 64; JACOBI_PCG needs max_iterations > 0 and tolerance > 0)");
        return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    }
    unsigned char* base = scratch_for_current_device();
    if (base == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    auto s = static_cast<cudaStream_t>(stream);
    const StepParams P = make_params(*config);

    uint16_t* codes = reinterpret_cast<uint16_t*>(base + kOffCodes);
    int32_t* anchor = reinterpret_cast<int32_t*>(base + kOffAnchor);
    const uint8_t* occ = occupancy;
    if (occ == nullptr) {  // no solids: an all-fluid occupancy in scratch
        const cudaError_t e = cudaMemsetAsync(base + kOffOcc, 0, cells, s);
        if (e != cudaSuccess) return cuda_failure("clearing the scratch occupancy", e);
        occ = base + kOffOcc;
    }
    PcgWork work{};
    float* vec[8];
    for (int i = 0; i < 8; ++i) vec[i] = reinterpret_cast<float*>(base + kOffVectors + i * kVectorBytes);
    work.r[0] = vec[0];
    work.r[1] = vec[1];
    work.s[0] = vec[2];
    work.s[1] = vec[3];
    work.w[0] = vec[4];
    work.w[1] = vec[5];
    work.p = vec[6];
    work.e = vec[7];
    work.x64 = reinterpret_cast<double*>(base + kOffX64);
    PcgControl* control = reinterpret_cast<PcgControl*>(base + kOffControl);

    PcgSettings S{};
    const bool fixed = d.mode == SMOKE_B200_SOLVER_FIXED_CG;
    S.jacobi = fixed ? 0 : 1;
    S.fp64 = d.reduction == SMOKE_B200_REDUCTION_FP64;
    S.fixed = fixed ? 1 : 0;
    S.max_iterations = fixed ? config->pressure_iterations : d.max_iterations;
    S.tolerance = d.tolerance;
    S.refinement = fixed ? 0 : static_cast<int32_t>(d.refinement);
    S.warm_start = 0;  // the scratch holds the previous call's solution, which need not belong to this problem

    PcgLaunchShape shape{};
    cudaError_t e = launch_anchor(P, occ, anchor, s);
    if (e != cudaSuccess) return cuda_failure("pressure anchor launch", e);
    if ((e = launch_stencil_codes(P, occ, anchor, codes, s)) != cudaSuccess) return cuda_failure("operator code launch", e);
    if ((e = launch_pcg(P, S, shape, codes, rhs, pressure, work, control, s)) != cudaSuccess) return cuda_failure("solver launch", e);
    if (out_status != nullptr) {
        PcgStatusDevice st{};
        if ((e = cudaMemcpyAsync(&st, &control->status, sizeof(st), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_failure("status read-back", e);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_failure("stream synchronisation", e);
        std::memcpy(out_status, &st, sizeof(st));
    }
    return SMOKE_SIMULATION_RESULT_OK;
}

const char* smoke_b200_last_error(void) { return g_last_error; }

unsigned long long smoke_b200_noalloc_max_cells(void) { return kNoAllocMaxCells; }

}  // extern "C"
