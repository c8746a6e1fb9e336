// smoke_b200_benchmark: command-line benchmark with the flags, scene and output lines of the reference's benchmark
// driver (benchmark.cu:14-245), so its numbers compare directly with the reference's own.
//
//  - scene (benchmark.cu:84-147): periodic x and z, no-slip floor, outflow top; density/temperature sources in an
//    ellipsoid at (0.5, 0.12, 0.5) of the extent with radii (0.07, 0.05, 0.07), 18 and 36 times exp(-2.2 r^2);
//  - warm-up steps, then timed steps between two CUDA events on the context stream (benchmark.cu:178-202);
//  - the density view is read back for its total and peak (benchmark.cu:204-212);
//  - the same two output lines (benchmark.cu:214-236); `--json` adds one JSON line with the solver's outcome.
// Beyond the reference's flags: --library PATH drives any library exporting the ABI (the reference's build too);
// --solver/--tolerance/--refinement/--max-iters/--warm-start select this library's solvers; --autotune runs its tuner
// first; --weights loads the learned preconditioner.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <string_view>
#include <vector>

#include "smoke_b200_ext.h"
#include "visual-simulation-of-smoke-3d.h"

namespace {

struct Options {
    int nx = 128, ny = 160, nz = 128;
    int warmup = 24, steps = 128, pressure_iters = 64;
    float cell_size = 0.01f, dt = 1.0f / 90.0f, ambient = 0.0f;
    float buoyancy_density = 0.15f, buoyancy_temperature = 1.2f, confinement = 0.22f;
    bool cubic = true;
    std::string library, solver = "fixed", weights;
    float tolerance = 1e-5f;
    int refinement = 3, max_iters = 500;
    bool autotune = false, json = false, warm_start = false;
};

// The ABI entry points, looked up in the library at run time; the extension ones may be missing.
struct Api {
    void* handle = nullptr;
    decltype(&smoke_simulation_create_context_cuda) create = nullptr;
    decltype(&smoke_simulation_destroy_context_cuda) destroy = nullptr;
    decltype(&smoke_simulation_update_density_source_cuda) density_source = nullptr;
    decltype(&smoke_simulation_update_temperature_source_cuda) temperature_source = nullptr;
    decltype(&smoke_simulation_step_cuda) step = nullptr;
    decltype(&smoke_simulation_get_view_cuda) get_view = nullptr;
    decltype(&smoke_b200_set_solver_cuda) set_solver = nullptr;
    decltype(&smoke_b200_get_solver_status_cuda) solver_status = nullptr;
    decltype(&smoke_b200_autotune_cuda) autotune = nullptr;
    decltype(&smoke_b200_net_create_cuda) net_create = nullptr;
    decltype(&smoke_b200_net_set_parameters_cuda) net_set = nullptr;
    decltype(&smoke_b200_net_parameter_count) net_count = nullptr;
    decltype(&smoke_b200_set_preconditioner_net_cuda) set_net = nullptr;
    decltype(&smoke_b200_net_destroy_cuda) net_destroy = nullptr;

    template <class F>
    bool bind(F& fn, const char* name, bool required) {
        fn = reinterpret_cast<F>(dlsym(handle, name));
        if (!fn && required) std::fprintf(stderr, "%s: symbol %s not found\n", "smoke_b200_benchmark", name);
        return fn != nullptr || !required;
    }
    bool load(const std::string& path) {
        handle = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!handle) {
            std::fprintf(stderr, "cannot load %s: %s\n", path.c_str(), dlerror());
            return false;
        }
        bool ok = bind(create, "smoke_simulation_create_context_cuda", true) && bind(destroy, "smoke_simulation_destroy_context_cuda", true) &&
                  bind(density_source, "smoke_simulation_update_density_source_cuda", true) && bind(temperature_source, "smoke_simulation_update_temperature_source_cuda", true) &&
                  bind(step, "smoke_simulation_step_cuda", true) && bind(get_view, "smoke_simulation_get_view_cuda", true);
        bind(set_solver, "smoke_b200_set_solver_cuda", false);
        bind(solver_status, "smoke_b200_get_solver_status_cuda", false);
        bind(autotune, "smoke_b200_autotune_cuda", false);
        bind(net_create, "smoke_b200_net_create_cuda", false);
        bind(net_set, "smoke_b200_net_set_parameters_cuda", false);
        bind(net_count, "smoke_b200_net_parameter_count", false);
        bind(set_net, "smoke_b200_set_preconditioner_net_cuda", false);
        bind(net_destroy, "smoke_b200_net_destroy_cuda", false);
        return ok;
    }
};

void usage() {
    std::printf(
        "smoke_b200_benchmark [--nx N] [--ny N] [--nz N] [--warmup N] [--steps N]\n"
        "                     [--pressure-iters N] [--cell-size H] [--dt DT]\n"
        "                     [--ambient-temperature T0]\n"
        "                     [--buoyancy-density A] [--buoyancy-temperature B]\n"
        "                     [--vorticity-confinement E] [--linear-advection]\n"
        "                     [--library PATH] [--solver fixed|jacobi|multigrid|learned] [--tolerance R]\n"
        "                     [--refinement N] [--max-iters N] [--weights PATH] [--warm-start] [--autotune] [--json]\n");
}

// Parses argv into `o`; returns -1 to go on, else the exit code.
int parse(int argc, char** argv, Options& o) {
    struct IntFlag {
        const char* name;
        int* v;
    };
    struct FloatFlag {
        const char* name;
        float* v;
    };
    struct TextFlag {
        const char* name;
        std::string* v;
    };
    const IntFlag ints[] = {{"--nx", &o.nx}, {"--ny", &o.ny}, {"--nz", &o.nz}, {"--warmup", &o.warmup}, {"--steps", &o.steps}, {"--pressure-iters", &o.pressure_iters}, {"--refinement", &o.refinement}, {"--max-iters", &o.max_iters}};
    const FloatFlag floats[] = {{"--cell-size", &o.cell_size}, {"--dt", &o.dt}, {"--ambient-temperature", &o.ambient}, {"--buoyancy-density", &o.buoyancy_density}, {"--buoyancy-temperature", &o.buoyancy_temperature}, {"--vorticity-confinement", &o.confinement}, {"--tolerance", &o.tolerance}};
    const TextFlag texts[] = {{"--library", &o.library}, {"--solver", &o.solver}, {"--weights", &o.weights}};
    for (int i = 1; i < argc; ++i) {
        const std::string_view a = argv[i];
        auto value = [&]() -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", argv[i]);
                return nullptr;
            }
            return argv[++i];
        };
        bool matched = false;
        for (const IntFlag& f : ints)
            if (a == f.name) {
                const char* v = value();
                if (!v) return EXIT_FAILURE;
                *f.v = std::atoi(v);
                matched = true;
            }
        for (const FloatFlag& f : floats)
            if (!matched && a == f.name) {
                const char* v = value();
                if (!v) return EXIT_FAILURE;
                *f.v = std::strtof(v, nullptr);
                matched = true;
            }
        for (const TextFlag& f : texts)
            if (!matched && a == f.name) {
                const char* v = value();
                if (!v) return EXIT_FAILURE;
                *f.v = v;
                matched = true;
            }
        if (matched) continue;
        if (a == "--linear-advection") o.cubic = false;
        else if (a == "--autotune") o.autotune = true;
        else if (a == "--warm-start") o.warm_start = true;
        else if (a == "--json") o.json = true;
        else if (a == "--help") {
            usage();
            return EXIT_SUCCESS;
        } else {
            std::fprintf(stderr, "unknown argument: %s\n", argv[i]);
            return EXIT_FAILURE;
        }
    }
    return -1;
}

SmokeSimulationConfig scene_config(const Options& o) {
    SmokeSimulationConfig c{};
    c.nx = o.nx;
    c.ny = o.ny;
    c.nz = o.nz;
    c.cell_size = o.cell_size;
    c.dt = o.dt;
    c.pressure_iterations = o.pressure_iters;
    c.ambient_temperature = o.ambient;
    c.buoyancy_density_factor = o.buoyancy_density;
    c.buoyancy_temperature_factor = o.buoyancy_temperature;
    c.vorticity_confinement = o.confinement;
    c.scalar_advection_mode = o.cubic ? SMOKE_SIMULATION_SCALAR_ADVECTION_MONOTONIC_CUBIC : SMOKE_SIMULATION_SCALAR_ADVECTION_LINEAR;
    auto flow = [](uint32_t type) {
        SmokeSimulationFlowBoundaryFaceDesc f{};
        f.type = type;
        return f;
    };
    auto scalar = [](uint32_t type, float value) {
        SmokeSimulationScalarBoundaryFaceDesc f{};
        f.type = type;
        f.value = value;
        return f;
    };
    c.flow_boundary.x_minus = c.flow_boundary.x_plus = flow(SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC);
    c.flow_boundary.z_minus = c.flow_boundary.z_plus = flow(SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC);
    c.flow_boundary.y_minus = flow(SMOKE_SIMULATION_FLOW_BOUNDARY_NO_SLIP_WALL);
    c.flow_boundary.y_plus = flow(SMOKE_SIMULATION_FLOW_BOUNDARY_OUTFLOW);
    for (auto* b : {&c.density_boundary, &c.temperature_boundary}) {
        const float v = b == &c.density_boundary ? 0.0f : o.ambient;
        b->x_minus = b->x_plus = b->z_minus = b->z_plus = scalar(SMOKE_SIMULATION_SCALAR_BOUNDARY_PERIODIC, v);
        b->y_minus = b->y_plus = scalar(SMOKE_SIMULATION_SCALAR_BOUNDARY_FIXED_VALUE, v);
    }
    return c;
}

// Density and temperature sources of the ellipsoidal plume (x fastest).
void plume_sources(const Options& o, std::vector<float>& density, std::vector<float>& temperature) {
    const size_t n = static_cast<size_t>(o.nx) * o.ny * o.nz;
    density.assign(n, 0.0f);
    temperature.assign(n, 0.0f);
    const float ex = o.nx * o.cell_size, ey = o.ny * o.cell_size, ez = o.nz * o.cell_size;
    const float cx = 0.5f * ex, cy = 0.12f * ey, cz = 0.5f * ez, rx = 0.07f * ex, ry = 0.05f * ey, rz = 0.07f * ez;
    size_t q = 0;
    for (int z = 0; z < o.nz; ++z)
        for (int y = 0; y < o.ny; ++y)
            for (int x = 0; x < o.nx; ++x, ++q) {
                const float dx = ((x + 0.5f) * o.cell_size - cx) / rx, dy = ((y + 0.5f) * o.cell_size - cy) / ry, dz = ((z + 0.5f) * o.cell_size - cz) / rz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > 1.0f) continue;
                const float g = std::exp(-2.2f * r2);
                density[q] = 18.0f * g;
                temperature[q] = 36.0f * g;
            }
}

std::string default_library(const char* argv0) {
    std::string dir = argv0;
    const size_t slash = dir.rfind('/');
    dir = slash == std::string::npos ? "." : dir.substr(0, slash);
    return dir + "/libsmoke_b200.so";
}

bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    std::fprintf(stderr, "%s failed: %s\n", what, cudaGetErrorString(e));
    return false;
}
bool smoke_ok(SmokeSimulationResult r, const char* what) {
    if (r == SMOKE_SIMULATION_RESULT_OK) return true;
    std::fprintf(stderr, "%s failed: %d\n", what, static_cast<int>(r));
    return false;
}

int run(const Options& o, Api& api) {
    const SmokeSimulationConfig cfg = scene_config(o);
    const size_t n = static_cast<size_t>(o.nx) * o.ny * o.nz;
    std::vector<float> src_d, src_t;
    plume_sources(o, src_d, src_t);
    cudaStream_t stream = nullptr;
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags")) return EXIT_FAILURE;
    SmokeSimulationContextCreateDesc desc{};
    desc.config = cfg;
    desc.stream = stream;
    desc.initial_density = 0.0f;
    desc.initial_temperature = o.ambient;
    SmokeSimulationContext ctx = nullptr;
    if (!smoke_ok(api.create(&desc, &ctx), "smoke_simulation_create_context_cuda")) return EXIT_FAILURE;
    float *dev_d = nullptr, *dev_t = nullptr;
    if (!cuda_ok(cudaMalloc(&dev_d, n * sizeof(float)), "cudaMalloc") || !cuda_ok(cudaMalloc(&dev_t, n * sizeof(float)), "cudaMalloc")) return EXIT_FAILURE;
    if (!cuda_ok(cudaMemcpyAsync(dev_d, src_d.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync") ||
        !cuda_ok(cudaMemcpyAsync(dev_t, src_t.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync"))
        return EXIT_FAILURE;
    if (!smoke_ok(api.density_source(ctx, dev_d), "update_density_source") || !smoke_ok(api.temperature_source(ctx, dev_t), "update_temperature_source")) return EXIT_FAILURE;

    SmokeB200Net net = nullptr;
    if (o.solver != "fixed") {
        if (!api.set_solver) {
            std::fprintf(stderr, "--solver %s: the library has no smoke_b200_set_solver_cuda\n", o.solver.c_str());
            return EXIT_FAILURE;
        }
        SmokeB200SolverDesc sd{};
        sd.reduction = SMOKE_B200_REDUCTION_FP64;
        sd.max_iterations = o.max_iters;
        sd.tolerance = o.tolerance;
        sd.refinement = static_cast<uint32_t>(o.refinement);
        sd.warm_start = o.warm_start ? 1u : 0u;  // each solve from the previous step's pressure (refinement >= 1)
        if (o.solver == "jacobi") sd.mode = SMOKE_B200_SOLVER_JACOBI_PCG;
        else if (o.solver == "multigrid") sd.mode = SMOKE_B200_SOLVER_MG_FCG;
        else if (o.solver == "learned") {
            sd.mode = SMOKE_B200_SOLVER_LEARNED_FCG;
            if (!api.net_create || !api.set_net || !api.net_set || !api.net_count || o.weights.empty()) {
                std::fprintf(stderr, "--solver learned needs the network entry points and --weights\n");
                return EXIT_FAILURE;
            }
            std::vector<float> w(api.net_count());
            FILE* f = std::fopen(o.weights.c_str(), "rb");
            const bool read = f && std::fread(w.data(), sizeof(float), w.size(), f) == w.size();
            if (f) std::fclose(f);
            if (!read) {
                std::fprintf(stderr, "cannot read %zu parameters from %s\n", w.size(), o.weights.c_str());
                return EXIT_FAILURE;
            }
            if (!smoke_ok(api.net_create(0, &net), "net_create") || !smoke_ok(api.net_set(net, w.data()), "net_set_parameters") || !smoke_ok(api.set_net(ctx, net), "set_preconditioner_net")) return EXIT_FAILURE;
        } else {
            std::fprintf(stderr, "unknown solver: %s\n", o.solver.c_str());
            return EXIT_FAILURE;
        }
        if (!smoke_ok(api.set_solver(ctx, &sd), "smoke_b200_set_solver_cuda")) return EXIT_FAILURE;
    }
    if (o.autotune) {
        if (!api.autotune) {
            std::fprintf(stderr, "--autotune: the library has no smoke_b200_autotune_cuda\n");
            return EXIT_FAILURE;
        }
        if (!smoke_ok(api.autotune(ctx, 0, 0, nullptr), "smoke_b200_autotune_cuda")) return EXIT_FAILURE;
    }

    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (!cuda_ok(cudaEventCreate(&t0), "cudaEventCreate") || !cuda_ok(cudaEventCreate(&t1), "cudaEventCreate")) return EXIT_FAILURE;
    for (int s = 0; s < o.warmup; ++s)
        if (!smoke_ok(api.step(ctx), "smoke_simulation_step_cuda warmup")) return EXIT_FAILURE;
    if (!cuda_ok(cudaStreamSynchronize(stream), "cudaStreamSynchronize warmup")) return EXIT_FAILURE;
    if (!cuda_ok(cudaEventRecord(t0, stream), "cudaEventRecord")) return EXIT_FAILURE;
    for (int s = 0; s < o.steps; ++s)
        if (!smoke_ok(api.step(ctx), "smoke_simulation_step_cuda")) return EXIT_FAILURE;
    float ms = 0.0f;
    if (!cuda_ok(cudaEventRecord(t1, stream), "cudaEventRecord") || !cuda_ok(cudaEventSynchronize(t1), "cudaEventSynchronize") || !cuda_ok(cudaEventElapsedTime(&ms, t0, t1), "cudaEventElapsedTime")) return EXIT_FAILURE;

    std::vector<float> density(n, 0.0f);
    SmokeSimulationViewRequest req{};
    req.kind = SMOKE_SIMULATION_VIEW_DENSITY;
    req.consumer_stream = stream;
    SmokeSimulationView view{};
    if (!smoke_ok(api.get_view(ctx, &req, &view), "smoke_simulation_get_view_cuda")) return EXIT_FAILURE;
    if (!cuda_ok(cudaMemcpyAsync(density.data(), view.data0, n * sizeof(float), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync") || !cuda_ok(cudaStreamSynchronize(stream), "cudaStreamSynchronize")) return EXIT_FAILURE;

    const double avg = o.steps > 0 ? ms / static_cast<double>(o.steps) : 0.0;
    const double mlups = ms > 0.0f ? static_cast<double>(n) * o.steps / (static_cast<double>(ms) * 1000.0) : 0.0;
    const float total = std::accumulate(density.begin(), density.end(), 0.0f);
    const float peak = density.empty() ? 0.0f : *std::max_element(density.begin(), density.end());
    std::printf("benchmark grid=%dx%dx%d warmup=%d steps=%d dt=%.6f ambient=%.3f buoyancy_density=%.3f buoyancy_temperature=%.3f vorticity_confinement=%.3f advection=%s\n", o.nx, o.ny, o.nz, o.warmup, o.steps,
                o.dt, o.ambient, o.buoyancy_density, o.buoyancy_temperature, o.confinement, o.cubic ? "monotonic_cubic" : "linear");
    std::printf("timing total_ms=%.3f avg_step_ms=%.6f mlups=%.3f total_density=%.6f peak_density=%.6f\n", static_cast<double>(ms), avg, mlups, total, peak);
    if (o.json) {
        SmokeB200SolverStatus st{};
        const bool have = api.solver_status && api.solver_status(ctx, &st) == SMOKE_SIMULATION_RESULT_OK;
        std::printf("{\"avg_step_ms\": %.6f, \"mlups\": %.3f, \"total_density\": %.6f, \"peak_density\": %.6f, \"solver\": \"%s\", \"iterations\": %d, \"status\": %d, \"true_relative_residual\": %.3e}\n", avg, mlups, total, peak,
                    o.solver.c_str(), have ? st.iterations : -1, have ? static_cast<int>(st.status) : -1, have ? st.true_relative_residual : -1.0);
    }
    cudaEventDestroy(t1);
    cudaEventDestroy(t0);
    cudaFree(dev_t);
    cudaFree(dev_d);
    api.destroy(ctx);
    if (net && api.net_destroy) api.net_destroy(net);
    cudaStreamDestroy(stream);
    return EXIT_SUCCESS;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    const int parsed = parse(argc, argv, o);
    if (parsed >= 0) return parsed;
    if (o.library.empty()) o.library = default_library(argv[0]);
    Api api;
    if (!api.load(o.library)) return EXIT_FAILURE;
    return run(o, api);
}
