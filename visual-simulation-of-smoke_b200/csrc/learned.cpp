// C ABI of the learned preconditioner (smoke_b200_ext.h): the network object (parameters, Adam state, packed
// operand images, evaluation workspace), its evaluation, gradient and training step, and the standalone 3x3x3
// convolution. Host code only; the kernels are reached through unet.h.
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "smoke_b200_ext.h"
#include "unet.h"

using namespace smoke_b200;

namespace {

struct DeviceScratch {
    void* p = nullptr;
    ~DeviceScratch() {
        if (p) cudaFree(p);
    }
};

bool valid_volume(int nx, int ny, int nz) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return false;
    const unsigned long long n = static_cast<unsigned long long>(nx) * ny * nz;
    return n < (1ull << 31);
}

struct CudaFailure : std::runtime_error {
    using std::runtime_error::runtime_error;
};
void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaFailure(std::string(what) + ": " + cudaGetErrorString(e));
}

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

// Initial parameters: He-normal weights (std sqrt(2 / fan_in)), the output layer scaled by 0.1, zero biases; normal
// deviates by Box-Muller from a splitmix64 stream of `seed`.
std::vector<float> initial_parameters(uint32_t seed) {
    std::vector<float> w(kNetParams, 0.0f);
    uint64_t state = 0x9E3779B97F4A7C15ull * (static_cast<uint64_t>(seed) + 1);
    auto next = [&] {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto uniform = [&] { return (static_cast<double>(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
    for (int L = 0; L < kNetLayers; ++L) {
        const double sd = std::sqrt(2.0 / (27.0 * kNet[L].cin)) * (L == kNetLayers - 1 ? 0.1 : 1.0);
        float* p = w.data() + net_param_offset(L);
        for (int i = 0; i < net_weight_count(L); ++i) {
            const double u1 = uniform(), u2 = uniform();
            p[i] = static_cast<float>(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
    }
    return w;
}

}  // namespace

// The network: FP32 parameters, gradient and Adam moments, packed images, and an evaluation workspace that grows to
// the largest volume seen.
struct SmokeB200Net_t {
    void* mem = nullptr;  // [params | grad | m | v | images]
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    NetImages images{};
    int adam_step = 0;
    void* work = nullptr;
    size_t work_bytes = 0;
    VolumeDims dims{};
    NetActs acts{};
    NetGrads grads{};

    ~SmokeB200Net_t() {
        if (work) cudaFree(work);
        if (mem) cudaFree(mem);
    }

    void allocate() {
        const size_t pbytes = (static_cast<size_t>(kNetParams) * sizeof(float) + 255) & ~size_t(255);
        check(cudaMalloc(&mem, 4 * pbytes + net_images_bytes()), "network parameters");
        char* p = static_cast<char*>(mem);
        params = reinterpret_cast<float*>(p);
        grad = reinterpret_cast<float*>(p + pbytes);
        m = reinterpret_cast<float*>(p + 2 * pbytes);
        v = reinterpret_cast<float*>(p + 3 * pbytes);
        net_images_bind(images, p + 4 * pbytes);
        check(cudaMemset(mem, 0, 4 * pbytes + net_images_bytes()), "network parameters");
    }

    // Workspace (activations and gradients) for a volume; reallocated when the volume changes size.
    void workspace(int nx, int ny, int nz) {
        const VolumeDims d = volume_dims(nx, ny, nz);
        const size_t need = net_acts_bytes(d) + net_grads_bytes(d);
        if (need > work_bytes) {
            if (work) check(cudaFree(work), "network workspace");
            work = nullptr;
            work_bytes = 0;
            check(cudaMalloc(&work, need), "network workspace");
            work_bytes = need;
        }
        dims = d;
        net_acts_bind(acts, work, d);
        net_grads_bind(grads, static_cast<char*>(work) + net_acts_bytes(d), d);
    }

    void check_error(cudaStream_t s) {
        unsigned err = 0;
        check(cudaMemcpyAsync(&err, acts.error, sizeof(err), cudaMemcpyDeviceToHost, s), "network status");
        check(cudaStreamSynchronize(s), "network status");
        if (err) throw CudaFailure("tensor-core completion wait ran out");
    }
};

const void* smoke_b200_net_images_block(const SmokeB200Net_t* net) { return net->images.fwd[0]; }

extern "C" {

uint32_t smoke_b200_net_parameter_count(void) { return static_cast<uint32_t>(kNetParams); }

SmokeSimulationResult smoke_b200_net_create_cuda(uint32_t seed, SmokeB200Net* out) {
    if (out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    *out = nullptr;
    std::unique_ptr<SmokeB200Net_t> net(new (std::nothrow) SmokeB200Net_t{});
    if (!net) return SMOKE_SIMULATION_RESULT_OUT_OF_MEMORY;
    const SmokeSimulationResult r = guarded([&] {
        net->allocate();
        const std::vector<float> w = initial_parameters(seed);
        check(cudaMemcpy(net->params, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice), "network parameters");
        check(net_pack(net->params, net->images, nullptr), "network images");
        check(cudaDeviceSynchronize(), "network images");
        return SMOKE_SIMULATION_RESULT_OK;
    });
    if (r != SMOKE_SIMULATION_RESULT_OK) return r;
    *out = net.release();
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_net_destroy_cuda(SmokeB200Net net) {
    if (net == nullptr) return SMOKE_SIMULATION_RESULT_OK;
    cudaDeviceSynchronize();
    delete net;
    return SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_net_get_parameters_cuda(SmokeB200Net net, float* out) {
    if (net == nullptr || out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        check(cudaDeviceSynchronize(), "network parameters");
        check(cudaMemcpy(out, net->params, static_cast<size_t>(kNetParams) * sizeof(float), cudaMemcpyDeviceToHost), "network parameters");
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_net_set_parameters_cuda(SmokeB200Net net, const float* values) {
    if (net == nullptr || values == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return guarded([&] {
        check(cudaDeviceSynchronize(), "network parameters");
        check(cudaMemcpy(net->params, values, static_cast<size_t>(kNetParams) * sizeof(float), cudaMemcpyHostToDevice), "network parameters");
        check(cudaMemset(net->m, 0, static_cast<size_t>(kNetParams) * sizeof(float)), "adam state");
        check(cudaMemset(net->v, 0, static_cast<size_t>(kNetParams) * sizeof(float)), "adam state");
        net->adam_step = 0;
        check(net_pack(net->params, net->images, nullptr), "network images");
        check(cudaDeviceSynchronize(), "network images");
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_net_apply_cuda(SmokeB200Net net, int nx, int ny, int nz, const float* rhs, const uint8_t* occupancy, float* out, void* stream) {
    if (net == nullptr || !valid_volume(nx, ny, nz) || rhs == nullptr || occupancy == nullptr || out == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return guarded([&] {
        net->workspace(nx, ny, nz);
        check(cudaMemsetAsync(net->acts.error, 0, sizeof(unsigned), s), "network status");
        check(net_forward(net->images, net->acts, rhs, nullptr, nullptr, nullptr, occupancy, s), "network forward");
        check(net_output(net->acts, nullptr, occupancy, out, s), "network output");
        net->check_error(s);
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_net_gradient_cuda(SmokeB200Net net, int nx, int ny, int nz, const float* rhs, const uint8_t* occupancy, const float* target, float* grad_out, double* loss_out, void* stream) {
    if (net == nullptr || !valid_volume(nx, ny, nz) || rhs == nullptr || occupancy == nullptr || target == nullptr) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return guarded([&] {
        net->workspace(nx, ny, nz);
        check(cudaMemsetAsync(net->acts.error, 0, sizeof(unsigned), s), "network status");
        check(cudaMemsetAsync(net->grads.sums, 0, 2 * sizeof(double), s), "network loss");
        check(net_forward(net->images, net->acts, rhs, nullptr, nullptr, nullptr, occupancy, s), "network forward");
        check(net_backward(net->images, net->acts, net->grads, nullptr, target, occupancy, net->grad, 0, s), "network backward");
        net->check_error(s);
        if (grad_out) check(cudaMemcpy(grad_out, net->grad, static_cast<size_t>(kNetParams) * sizeof(float), cudaMemcpyDeviceToHost), "network gradient");
        if (loss_out) check(cudaMemcpy(loss_out, net->grads.sums + 1, sizeof(double), cudaMemcpyDeviceToHost), "network loss");
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_net_train_cuda(SmokeB200Net net, int nx, int ny, int nz, uint32_t count, const float* rhs, const uint8_t* occupancy, const float* target, float learning_rate, double* mean_loss_out, void* stream) {
    if (net == nullptr || !valid_volume(nx, ny, nz) || count == 0 || rhs == nullptr || occupancy == nullptr || target == nullptr || !(learning_rate > 0.0f)) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return guarded([&] {
        net->workspace(nx, ny, nz);
        const size_t n = net->dims.n;
        check(cudaMemsetAsync(net->acts.error, 0, sizeof(unsigned), s), "network status");
        check(cudaMemsetAsync(net->grads.sums, 0, 2 * sizeof(double), s), "network loss");
        for (uint32_t i = 0; i < count; ++i) {
            check(net_forward(net->images, net->acts, rhs + i * n, nullptr, nullptr, nullptr, occupancy + i * n, s), "network forward");
            check(net_backward(net->images, net->acts, net->grads, nullptr, target + i * n, occupancy + i * n, net->grad, i > 0 ? 1 : 0, s), "network backward");
        }
        net->adam_step += 1;
        check(net_adam(net->params, net->grad, net->m, net->v, learning_rate, net->adam_step, 1.0f / static_cast<float>(count), net->images, s), "adam");
        net->check_error(s);
        if (mean_loss_out) {
            double loss = 0.0;
            check(cudaMemcpy(&loss, net->grads.sums + 1, sizeof(double), cudaMemcpyDeviceToHost), "network loss");
            *mean_loss_out = loss / static_cast<double>(count);
        }
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

SmokeSimulationResult smoke_b200_conv3d_cuda(int nx, int ny, int nz, int cin, int cout, const void* in, const float* weights, const float* bias, int relu, void* out, float* out_f32, void* stream) {
    const int cin_store = cin >= 1 ? net_store(cin) : 0;
    const bool cin_ok = cin_store == 8 || cin_store == 16 || cin_store == 32 || cin_store == 64 || cin_store == 128;
    if (!valid_volume(nx, ny, nz) || !cin_ok || cout < 1 || cout > 128 || in == nullptr || weights == nullptr || (out == nullptr && out_f32 == nullptr)) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int cout_store = net_store(cout), cpad = net_cout_pad(cout);
    const size_t pack_bytes = (conv_pack_bytes(cin_store, cout) + 255) & ~size_t(255);
    DeviceScratch scratch;
    // [pack | cpad bias floats | error word]
    if (cudaMalloc(&scratch.p, pack_bytes + cpad * sizeof(float) + 16) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    uint8_t* pack = static_cast<uint8_t*>(scratch.p);
    float* bpad = reinterpret_cast<float*>(pack + pack_bytes);
    unsigned* error = reinterpret_cast<unsigned*>(bpad + cpad);
    if (cudaMemsetAsync(bpad, 0, cpad * sizeof(float) + 16, s) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (bias && cudaMemcpyAsync(bpad, bias, cout * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    if (launch_pack_conv(weights, cin, cout, 0, cin_store, pack, s) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const VolumeDims d = volume_dims(nx, ny, nz);
    if (launch_conv3(d, cin_store, cout, static_cast<const __nv_bfloat16*>(in), pack, bpad, relu, nullptr, static_cast<__nv_bfloat16*>(out), cout_store, out_f32, error, s, nullptr) != cudaSuccess)
        return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    unsigned err = 0;
    if (cudaMemcpyAsync(&err, error, sizeof(err), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    return err ? SMOKE_SIMULATION_RESULT_BACKEND_FAILURE : SMOKE_SIMULATION_RESULT_OK;
}

SmokeSimulationResult smoke_b200_test_conv_wait_timeout_cuda(int nx, int ny, int nz, unsigned long long wait_cycles, unsigned* error_out, void* stream) {
    if (!valid_volume(nx, ny, nz) || error_out == nullptr || wait_cycles == 0 || wait_cycles > 4000000000ull) return SMOKE_SIMULATION_RESULT_BACKEND_FAILURE;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return guarded([&] {
        const VolumeDims d = volume_dims(nx, ny, nz);
        const size_t in_bytes = (static_cast<size_t>(d.n) * 16 * 2 + 255) & ~size_t(255);
        const size_t pack_bytes = (conv_pack_bytes(16, 16) + 255) & ~size_t(255);
        DeviceScratch scratch;
        check(cudaMalloc(&scratch.p, in_bytes + pack_bytes + 256), "scratch");
        auto* in = static_cast<__nv_bfloat16*>(scratch.p);
        auto* pack = static_cast<uint8_t*>(scratch.p) + in_bytes;
        auto* error = reinterpret_cast<unsigned*>(pack + pack_bytes);
        check(cudaMemsetAsync(scratch.p, 0, in_bytes + pack_bytes + 256, s), "scratch");
        // the loads of every tile are expected but never issued: each block's first wait must run out
        check(launch_conv3(d, 16, 16, in, pack, nullptr, 0, nullptr, nullptr, 16, nullptr, error, s, nullptr, static_cast<long long>(wait_cycles), 1), "convolution");
        check(cudaMemcpyAsync(error_out, error, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "error word");
        check(cudaStreamSynchronize(s), "error word");
        return SMOKE_SIMULATION_RESULT_OK;
    });
}

}  // extern "C"
