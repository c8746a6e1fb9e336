// Learned preconditioner: a 3-D U-Net of four levels (16, 32, 64 and 128 channels) on channels-last BF16 volumes,
// its 3x3x3 convolutions as implicit GEMMs on the tcgen05 tensor cores (forward, backward-data, backward-weight),
// and the glue kernels between them. Host launchers only; the kernels are in unet.cu.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace smoke_b200 {

// ------------------------------------------------------------------------------------------ network shape
// Four levels (level l halves the extents of level l - 1, rounding up). Layers, in execution order:
//   a: level 0, [r * s, fluid] (2) -> e0 (16), ReLU      b: level 1, pool(e0) (16) -> e1 (32), ReLU
//   c: level 2, pool(e1) (32) -> e2 (64), ReLU           d: level 3, pool(e2) (64) -> e3 (128), ReLU
//   m: level 3, e3 (128) -> m3 (64), ReLU                e: level 2, up(m3) + e2 (64) -> u2 (32), ReLU
//   f: level 1, up(u2) + e1 (32) -> u1 (16), ReLU        g: level 0, up(u1) + e0 (16) -> y (1), linear
// Every convolution is 3x3x3 with zero padding; pool = mean of the existing children of a coarse cell; up = copy
// of the parent. The input scale s = sqrt(n) / ||r|| makes the network positively homogeneous: the output is y / s.
constexpr int kNetLevels = 4;
constexpr int kNetLayers = 8;
struct NetLayer {
    int cin, cout;  // real channel counts
    int level;
};
constexpr NetLayer kNet[kNetLayers] = {{2, 16, 0}, {16, 32, 1}, {32, 64, 2}, {64, 128, 3}, {128, 64, 3}, {64, 32, 2}, {32, 16, 1}, {16, 1, 0}};
// Stored channels of an activation with c real channels: 8 for the 2-channel input, else c (a multiple of 16).
__host__ __device__ constexpr int net_store(int c) { return c <= 8 ? 8 : ((c + 15) / 16) * 16; }
// Output columns of a convolution with c output channels: a multiple of 16 (the tensor core's N step).
__host__ __device__ constexpr int net_cout_pad(int c) { return ((c + 15) / 16) * 16; }
// Stored channels of the gradient with respect to a layer's output (the backward convolution's input).
__host__ __device__ constexpr int net_grad_store(int c) { return c <= 16 ? 16 : net_store(c); }
// FP32 parameters of layer L: weights [27][cin][cout] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)), then bias [cout].
constexpr int net_weight_count(int L) { return 27 * kNet[L].cin * kNet[L].cout; }
constexpr int net_param_count(int L) { return net_weight_count(L) + kNet[L].cout; }
constexpr int net_param_offset(int L) { return L == 0 ? 0 : net_param_offset(L - 1) + net_param_count(L - 1); }
constexpr int kNetParams = net_param_offset(kNetLayers);

// Implicit-GEMM shape of a convolution whose input has `cin_store` stored channels and `cout` output channels: the
// output columns computed per block (N of one MMA; it divides net_cout_pad(cout)).
__host__ __device__ constexpr int conv_nc(int cin_store, int cout) {
    return cin_store == 8 || cin_store == 128 || net_cout_pad(cout) % 32 != 0 ? 16 : 32;
}
__host__ __device__ constexpr int conv_taps(int cin_store) { return cin_store == 8 ? 28 : 27; }
// Bytes of the packed BF16 weight image (K-major B operand, one image of conv_nc columns per output chunk).
__host__ __device__ constexpr uint32_t conv_pack_bytes(int cin_store, int cout) {
    return static_cast<uint32_t>(conv_taps(cin_store) * cin_store) * static_cast<uint32_t>(net_cout_pad(cout)) * 2u;
}

// ------------------------------------------------------------------------------------------ launchers
struct VolumeDims {
    int nx, ny, nz;
    uint32_t n;
};
inline VolumeDims volume_dims(int nx, int ny, int nz) { return {nx, ny, nz, static_cast<uint32_t>(nx) * ny * nz}; }
inline VolumeDims coarse_dims(const VolumeDims& d) { return volume_dims((d.nx + 1) / 2, (d.ny + 1) / 2, (d.nz + 1) / 2); }

// 3x3x3 convolution of `in` ([n][cin_store] BF16, cin_store in {8, 16, 32, 64, 128}) with the packed weights `wpack`
// (launch_pack_conv, `cout` output channels): out = act(conv + bias), act = ReLU when `relu`, then zeroed where
// `gate` ([n][cout_store] BF16, optional) is not positive. Writes `out` ([n][cout_store] BF16, optional) and/or
// `out_f32` (channel 0, [n] FP32, optional). bias: net_cout_pad(cout) floats or null. `error` (device word) gets
// bit 0 when a tensor-core or TMA completion wait ran out. With `skip` (device word, optional) nonzero when the
// kernel starts, it does nothing. `wait_cycles` bounds every wait (0: about 2 s); `drop_loads` (test only) makes the
// producer expect its loads without issuing them.
cudaError_t launch_conv3(const VolumeDims& d, int cin_store, int cout, const __nv_bfloat16* in, const uint8_t* wpack, const float* bias, int relu, const __nv_bfloat16* gate, __nv_bfloat16* out,
                         int cout_store, float* out_f32, unsigned* error, cudaStream_t s, const uint32_t* skip = nullptr, long long wait_cycles = 0, int drop_loads = 0);

// Packs layer weights W [27][cin][cout] (FP32) into the operand image of the forward convolution (input stored
// channels cin_store = net_store(cin)), or with `transpose` of the backward-data convolution (input = the output
// gradient, cin_store = net_grad_store(cout); output = cin channels; taps mirrored).
cudaError_t launch_pack_conv(const float* w, int cin, int cout, int transpose, int cin_store, uint8_t* pack, cudaStream_t s);

// ------------------------------------------------------------------------------------------ whole network
// Device images of the network's parameters the kernels read: packed BF16 operand images of every forward
// convolution and of the backward-data convolutions of layers 1..7, and the biases padded to net_cout_pad.
struct NetImages {
    uint8_t* fwd[kNetLayers];
    uint8_t* bwd[kNetLayers];  // bwd[0] unused
    float* bias[kNetLayers];
    uint8_t* band;             // the last (single-output) layer's banded image for its forward (unet.cu)
};
// Bytes of NetImages storage and the binding of its pointers inside one buffer.
size_t net_images_bytes();
void net_images_bind(NetImages& I, void* base);
// Rebuilds the packed images and padded biases from the FP32 parameters w (kNetParams floats).
cudaError_t net_pack(const float* w, const NetImages& I, cudaStream_t s);

// Activations of one evaluation on a level-0 volume d[0] (level l + 1 is coarse_dims of level l).
struct NetActs {
    VolumeDims d[kNetLevels];
    __nv_bfloat16* x0;                 // level 0, 8 channels: the input
    __nv_bfloat16 *e0, *s0;            // level 0, 16
    __nv_bfloat16 *p1, *u1;            // level 1, 16
    __nv_bfloat16 *e1, *s1;            // level 1, 32
    __nv_bfloat16 *p2, *u2;            // level 2, 32
    __nv_bfloat16 *e2, *s2;            // level 2, 64
    __nv_bfloat16 *p3, *m3;            // level 3, 64
    __nv_bfloat16* e3;                 // level 3, 128
    float* y;                          // level 0, network output (before the 1 / s scale)
    double* norm2;                     // ||input||^2 when the caller does not supply it
    unsigned* error;                   // tensor-core wait timeouts (bit 0)
};
size_t net_acts_bytes(const VolumeDims& d0);
void net_acts_bind(NetActs& A, void* base, const VolumeDims& d0);

// Gradient scratch of one evaluation (same volume as the NetActs it belongs to).
struct NetGrads {
    __nv_bfloat16 *gy, *gs0, *ge0;     // level 0, 16
    __nv_bfloat16 *gu1, *gp1;          // level 1, 16
    __nv_bfloat16 *gs1, *ge1;          // level 1, 32
    __nv_bfloat16 *gu2, *gp2;          // level 2, 32
    __nv_bfloat16 *gs2, *ge2;          // level 2, 64
    __nv_bfloat16 *gm3, *gp3;          // level 3, 64
    __nv_bfloat16* ge3;                // level 3, 128
    float* partial;                    // weight-gradient partial sums
    float* tmask;                      // masked target
    double* sums;                      // [0] target norm^2, [1] loss
};
size_t net_grads_bytes(const VolumeDims& d0);
void net_grads_bind(NetGrads& G, void* base, const VolumeDims& d0);

// Forward pass on the input r (r1 and *parity pick the buffer on the device when parity is given); norm2 is ||r||^2
// on the device, or null to compute it into A.norm2. Leaves the network output in A.y. Every kernel of the pass does
// nothing when `skip` (device word, optional) is nonzero.
cudaError_t net_forward(const NetImages& I, const NetActs& A, const float* r0, const float* r1, const int* parity, const double* norm2, const uint8_t* occ, cudaStream_t s, const uint32_t* skip = nullptr);
// out = fluid ? A.y / s : 0 (the preconditioned vector with the input's scale restored).
cudaError_t net_output(const NetActs& A, const double* norm2, const uint8_t* occ, float* out, cudaStream_t s);
// Loss of the last forward pass against `target` and the parameter gradient: grad (kNetParams floats) is
// overwritten, or accumulated into when `accumulate`; the loss is added into G.sums[1].
cudaError_t net_backward(const NetImages& I, const NetActs& A, const NetGrads& G, const double* norm2, const float* target, const uint8_t* occ, float* grad, int accumulate, cudaStream_t s);
// One Adam step on w with moments m, v (step >= 1), gradient scaled by gscale; then the images are repacked.
cudaError_t net_adam(float* w, const float* grad, float* m, float* v, float lr, int step, float gscale, const NetImages& I, cudaStream_t s);

// What a solve with the learned preconditioner needs. The network runs on the multigrid hierarchy's level 1 (every
// extent of the grid halved, rounding up): its images, an activation workspace on that volume, the level's solid mask
// (1 = no fluid child; the fluid-mask input channel), and a level-0 array for the prolonged correction.
struct LearnedSolve {
    NetImages images;
    NetActs acts;
    uint8_t* occupancy;
    float* fine;
};

}  // namespace smoke_b200

// The device block of a network's packed images (net_images_bytes() long), for copies into a context.
struct SmokeB200Net_t;
const void* smoke_b200_net_images_block(const SmokeB200Net_t* net);
