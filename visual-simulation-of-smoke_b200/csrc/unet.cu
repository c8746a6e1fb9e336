// Kernels of the learned preconditioner (unet.h): tcgen05 implicit-GEMM 3x3x3 convolutions on channels-last BF16
// volumes with FP32 accumulation in tensor memory, and the glue between the U-Net's layers.
//
// Convolution as a GEMM: D[cell][co] = sum over k = (tap, ci) of A[cell][k] * B[co][k], with A[cell][(tap, ci)] =
// in[cell + offset(tap)][ci] (0 outside the volume). One block of 128 threads computes tiles of M = 128 consecutive
// cells, N = 16 output channels: every thread gathers its cell's 27 neighbour channel vectors (16 or 32 bytes each)
// straight into the core-matrix layout of the A operand in shared memory, then one thread issues the K/16 MMAs, whose
// accumulators stay in tensor memory until the epilogue (bias, ReLU, gate) reads them back.
#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "tcgen05.cuh"
#include "unet.h"

namespace smoke_b200 {
namespace {

constexpr int kConvThreads = 128;
constexpr long long kSpinCycles = 4000000000ll;  // ~2 s: bound of every tensor-core completion wait

// Tiles of 8 x 16 x 1 cells (M = 128 rows, row m = cell (m % 8, m / 8) of the tile). A tile's input is its halo box
// of 10 x 18 x 3 cells, brought into shared memory by one TMA load per 8-channel plane (zeros outside the volume):
// cell (x, y, z) of the box at byte ((z * 18 + y) * 10 + x) * 16 of its plane. The A operand of tap (dx, dy, dz) is
// that box read from offset ((1 + dz) * 18 + 1 + dy) * 160 + (1 + dx) * 16: every 8 cells of a tile row are 8
// consecutive 16-byte rows of the box, i.e. one core matrix, and the next tile row starts one box row (160 bytes) on
// (SBO). So no im2col copy exists: each MMA reads its two K columns (two taps of an 8-channel input, or the two
// planes of one tap of a 16-channel input; LBO = their distance) straight from the box.
template <int CIN>
struct ConvShape {
    static constexpr int kTX = 8, kTY = 16;
    static constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = 3;
    static constexpr uint32_t kRow = kHX * 16;                               // bytes of one box row (SBO)
    static constexpr uint32_t kBox = kHX * kHY * kHZ * 16;                   // 8640 bytes per plane
    static constexpr uint32_t kPlane = 8704;                                 // plane pitch: box + zero slack, 128-aligned
    static constexpr int kPlanes = CIN / 8;
    static constexpr uint32_t kStage = (kPlanes * kPlane + 1023u) & ~1023u;  // one pipeline stage
    static constexpr int kKSteps = conv_taps(CIN) * CIN / 16;                // MMAs per tile (K = 16 each)
    static constexpr uint32_t kBBytes = conv_pack_bytes(CIN);
    static constexpr uint32_t kSmem = 2 * kStage + kBBytes;
};
__host__ __device__ constexpr uint32_t tap_offset(int tap) {
    return ((tap / 9) * 18 + (tap / 3) % 3) * 160u + (tap % 3) * 16u;  // (dz + 1, dy + 1, dx + 1) of the tap
}
// the padding tap's K column (tap 26's rows, 16 bytes on) stays inside the plane's zero slack
static_assert(tap_offset(26) + 16 + 15 * ConvShape<8>::kRow + 128 <= ConvShape<8>::kPlane, "zero slack");
static_assert(tap_offset(26) + 15 * ConvShape<8>::kRow + 128 <= ConvShape<8>::kBox, "box");

struct ConvArgs {
    const __nv_bfloat16* in;
    const uint8_t* wpack;
    const float* bias;
    const __nv_bfloat16* gate;
    __nv_bfloat16* out;
    float* out_f32;
    unsigned* error;
    const uint32_t* skip;  // optional: the launch does nothing when *skip is nonzero
    int relu, cout_store;
    int nx, ny, nz;
    uint32_t n;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// Persistent over tiles with two pipeline stages: while the tensor core works on tile j (stage j % 2, accumulator
// j % 2 in tensor memory), the TMA load of tile j + 1 fills the other stage. Thread 0 issues the loads and the MMAs;
// all 128 threads run the epilogue (tensor memory -> bias, ReLU, gate -> BF16/FP32 stores).
template <int CIN>
__global__ void __launch_bounds__(kConvThreads) conv3_kernel(const __grid_constant__ ConvArgs a, const __grid_constant__ CUtensorMap map) {
    using S = ConvShape<CIN>;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* Bs = smem + 2 * S::kStage;
    __shared__ uint64_t full[2], done[2];
    __shared__ uint32_t tmem_slot;
    if (a.skip && *a.skip) return;  // uniform: every block reads the same word
    const int t = threadIdx.x, warp = t >> 5;
    const uint4* wsrc = reinterpret_cast<const uint4*>(a.wpack);
    for (uint32_t i = t; i < S::kBBytes / 16u; i += kConvThreads) reinterpret_cast<uint4*>(Bs)[i] = wsrc[i];
    for (int st = 0; st < 2; ++st)  // the slack after each box stays zero (read by the padding tap, times zero weights)
        for (int p = 0; p < S::kPlanes; ++p)
            for (uint32_t i = t; i < (S::kPlane - S::kBox) / 16u; i += kConvThreads) reinterpret_cast<uint4*>(smem + st * S::kStage + p * S::kPlane + S::kBox)[i] = make_uint4(0, 0, 0, 0);
    if (t == 0) {
        for (int st = 0; st < 2; ++st) {
            tc::mbar_init(&full[st], 1);
            tc::mbar_init(&done[st], 1);
        }
    }
    if (warp == 0) tc::tmem_alloc(&tmem_slot, 32);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 16, false, false);
    const uint32_t b_base = tc::smem_addr(Bs);
    const int ntx = (a.nx + S::kTX - 1) / S::kTX, nty = (a.ny + S::kTY - 1) / S::kTY;
    const uint32_t tiles = static_cast<uint32_t>(ntx) * nty * a.nz;
    auto load = [&](uint32_t tile, int st) {
        const int tx = static_cast<int>(tile % ntx), rest = static_cast<int>(tile / ntx);
        const int ty = rest % nty, tz = rest / nty;
        tc::mbar_arrive_expect_tx(&full[st], S::kPlanes * S::kBox);
        for (int p = 0; p < S::kPlanes; ++p) tc::tma_load_4d(smem + st * S::kStage + p * S::kPlane, &map, 8 * p, tx * S::kTX - 1, ty * S::kTY - 1, tz - 1, &full[st]);
    };
    float bias[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) bias[c] = a.bias ? __ldg(a.bias + c) : 0.0f;
    if (t == 0 && blockIdx.x < tiles) load(blockIdx.x, 0);
    uint32_t j = 0;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++j) {
        const int st = static_cast<int>(j & 1u);
        const uint32_t parity = (j >> 1) & 1u;
        if (t == 0) {
            // the other stage was last read by the MMAs of tile j - 1, which completed before that tile's epilogue
            if (tile + gridDim.x < tiles) load(tile + gridDim.x, st ^ 1);
            if (tc::mbar_wait(&full[st], parity, kSpinCycles)) {
                tc::fence_after_sync();
                const uint32_t a_base = tc::smem_addr(smem + st * S::kStage);
#pragma unroll 1
                for (int k = 0; k < S::kKSteps; ++k) {
                    uint32_t start, lbo;
                    if constexpr (CIN == 8) {  // taps 2k and 2k + 1 (tap 27: zero weights, any finite A)
                        start = a_base + tap_offset(2 * k);
                        lbo = 2 * k + 1 < 27 ? tap_offset(2 * k + 1) - tap_offset(2 * k) : 16u;
                    } else {  // tap k, channel planes 0 and 1
                        start = a_base + tap_offset(k);
                        lbo = S::kPlane;
                    }
                    tc::mma_bf16(tmem + st * 16, tc::smem_desc(start, lbo, S::kRow), tc::smem_desc(b_base + k * 512u, 256u, 128u), idesc, k > 0 ? 1u : 0u);
                }
                tc::commit(&done[st]);
            } else {
                atomicOr(a.error, 1u);
            }
        }
        __syncwarp();
        const bool ok = __syncthreads_and(tc::mbar_wait(&done[st], parity, kSpinCycles) ? 1 : 0) != 0;
        if (!ok) {
            if (t == 0) atomicOr(a.error, 1u);
            break;
        }
        tc::fence_after_sync();
        float acc[16];
        tc::tmem_load16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + st * 16, acc);
        const int tx = static_cast<int>(tile % ntx), rest = static_cast<int>(tile / ntx);
        const int x = tx * S::kTX + (t & 7), y = (rest % nty) * S::kTY + (t >> 3), z = rest / nty;
        if (x < a.nx && y < a.ny) {
            const uint32_t q = (static_cast<uint32_t>(z) * a.ny + y) * a.nx + x;
            float v[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                v[c] = acc[c] + bias[c];
                if (a.relu) v[c] = fmaxf(v[c], 0.0f);
            }
            if (a.gate) {
                const uint4* g = reinterpret_cast<const uint4*>(a.gate) + static_cast<size_t>(q) * (a.cout_store / 8);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (h * 8 >= a.cout_store) break;
                    const uint4 gv = __ldg(g + h);
                    const __nv_bfloat16* gb = reinterpret_cast<const __nv_bfloat16*>(&gv);
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        if (!(__bfloat162float(gb[c]) > 0.0f)) v[h * 8 + c] = 0.0f;
                }
            }
            if (a.out_f32) a.out_f32[q] = v[0];
            if (a.out) {
                uint4* o = reinterpret_cast<uint4*>(a.out) + static_cast<size_t>(q) * (a.cout_store / 8);
                o[0] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]), pack_bf16x2(v[6], v[7]));
                if (a.cout_store == 16) o[1] = make_uint4(pack_bf16x2(v[8], v[9]), pack_bf16x2(v[10], v[11]), pack_bf16x2(v[12], v[13]), pack_bf16x2(v[14], v[15]));
            }
        }
        tc::fence_before_sync();
        __syncthreads();  // this accumulator is read out before tile j + 2's MMAs overwrite it
        tc::fence_after_sync();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, 32);
}

// Operand image of B (N = 16 rows = output channels, K = taps x stored input channels), K-major core matrices:
// element (co, k) at byte ((k / 8) * 2 + co / 8) * 128 + (co % 8) * 16 + (k % 8) * 2.
__global__ void pack_conv_kernel(const float* __restrict__ w, int cin, int cout, int transpose, uint8_t* __restrict__ pack) {
    const int in_ch = transpose ? cout : cin, out_ch = transpose ? cin : cout;
    const int store = net_store(in_ch);
    const int K = conv_taps(store) * store;
    const int total = K * 16;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int k = i / 16, co = i % 16;
        const int tap = k / store, ci = k % store;
        float v = 0.0f;
        if (tap < 27 && ci < in_ch && co < out_ch) {
            // forward: W[tap][ci][co]; backward-data: input channel = forward output, mirrored tap
            v = transpose ? w[(static_cast<size_t>(26 - tap) * cin + co) * cout + ci] : w[(static_cast<size_t>(tap) * cin + ci) * cout + co];
        }
        const size_t off = static_cast<size_t>((k / 8) * 2 + co / 8) * 128 + (co % 8) * 16 + (k % 8) * 2;
        *reinterpret_cast<__nv_bfloat16*>(pack + off) = __float2bfloat16_rn(v);
    }
}

// Resident blocks of a kernel that uses `smem` bytes of dynamic shared memory (per SM x SMs): the shared memory of
// an SM over what one block takes (its dynamic bytes, 1 KB of static data and the 1 KB the system reserves per
// block), at most 6 (tensor memory: 6 x 64 columns at most of 512). These kernels' 128 threads and < 64 registers
// never bind first. Cached per kernel and device.
int resident_blocks(const void* kernel, size_t smem) {
    static std::mutex lock;
    static std::map<std::pair<const void*, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> guard(lock);
    auto it = cache.find({kernel, dev});
    if (it != cache.end()) return it->second;
    int sms = 1, smem_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    const int per_sm = std::min(6, std::max(1, smem_sm / static_cast<int>(smem + 2048)));
    const int r = std::max(1, sms * per_sm);
    cache.emplace(std::make_pair(kernel, dev), r);
    return r;
}

// cuTensorMapEncodeTiled from the driver, found once through the runtime (no link against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map of a channels-last BF16 volume with `cin` stored channels: dimensions (channel, x, y, z), boxes of
// 8 channels x the halo of one tile, zeros outside.
template <int CIN>
cudaError_t halo_map(CUtensorMap* map, const ConvArgs& a) {
    using S = ConvShape<CIN>;
    const auto encode = tensor_map_encoder();
    if (encode == nullptr) return cudaErrorNotSupported;
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(CIN), static_cast<cuuint64_t>(a.nx), static_cast<cuuint64_t>(a.ny), static_cast<cuuint64_t>(a.nz)};
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(CIN) * 2, static_cast<cuuint64_t>(a.nx) * CIN * 2, static_cast<cuuint64_t>(a.nx) * a.ny * CIN * 2};
    const cuuint32_t box[4] = {8, S::kHX, S::kHY, S::kHZ};
    const cuuint32_t step[4] = {1, 1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(a.in), dims, strides, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int CIN>
cudaError_t conv_typed(const VolumeDims& d, const ConvArgs& a, cudaStream_t s) {
    using S = ConvShape<CIN>;
    static bool configured = false;
    if (!configured) {  // all of the unified L1 as shared memory, so that several blocks fit on an SM
        cudaError_t e = cudaFuncSetAttribute(conv3_kernel<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::kSmem));
        if (e == cudaSuccess) e = cudaFuncSetAttribute(conv3_kernel<CIN>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if ((reinterpret_cast<uintptr_t>(a.in) & 15u) != 0) return cudaErrorMisalignedAddress;
    CUtensorMap map;
    const cudaError_t e = halo_map<CIN>(&map, a);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = static_cast<uint64_t>((d.nx + S::kTX - 1) / S::kTX) * ((d.ny + S::kTY - 1) / S::kTY) * d.nz;
    const int grid = static_cast<int>(std::min<uint64_t>(tiles, static_cast<uint64_t>(resident_blocks(reinterpret_cast<const void*>(conv3_kernel<CIN>), S::kSmem))));
    conv3_kernel<CIN><<<grid, kConvThreads, S::kSmem, s>>>(a, map);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------ weight gradient
// dW[tap][ci][co] = sum over cells q of in[q + offset(tap)][ci] * g[q][co], as a GEMM with M = (tap, ci) (taps padded
// to 32: M-tiles of 128 rows), N = 16 (co), K = cells. Both operands are MN-major in shared memory: a core matrix is
// 8 cells (K) x 16 bytes = 8 consecutive channels, so every 16-byte channel vector lands as one core-matrix row.
// Row (tap 27, channel 0) of A is 1 for every cell, which makes D[27 * CIN][co] the bias gradient sum_q g[q][co].
// Every block accumulates its share of the cells in tensor memory and writes its partial D; wgrad_reduce sums them.
constexpr int kWgradCells = 64;  // cells (K) per gather round: 8 core-matrix groups, 4 MMA K-steps

template <int CIN>
struct WgradShape {
    static constexpr int kMPad = 32 * CIN;                 // 256 or 512 rows
    static constexpr int kMTiles = kMPad / 128;            // 2 or 4
    static constexpr int kMGroups = kMPad / 8;             // core matrices along M
    static constexpr uint32_t kABytes = (kWgradCells / 8) * kMGroups * 128u;
    static constexpr uint32_t kARegion = kABytes;
    static constexpr uint32_t kBBytes = (kWgradCells / 8) * 2u * 128u;
    static constexpr uint32_t kBRegion = kBBytes;
    static constexpr uint32_t kSmem = kARegion + kBRegion;
    static constexpr uint32_t kTmemCols = kMTiles * 16 <= 32 ? 32u : 64u;
};

struct WgradArgs {
    const __nv_bfloat16* in;  // [n][CIN]
    const __nv_bfloat16* g;   // [n][gc]
    float* partial;           // [gridDim.x][kMPad][16]
    unsigned* error;
    int gc;                   // stored channels of g (8 or 16)
    int nx, ny, nz;
    uint32_t n;
};

template <int CIN>
__global__ void __launch_bounds__(kConvThreads) wgrad_kernel(const __grid_constant__ WgradArgs a) {
    using S = WgradShape<CIN>;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* As = smem;
    uint8_t* Bs = smem + S::kARegion;
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5;
    constexpr int kCg = CIN / 8;
    // rows of taps 27..31 are constant: zero, except channel 0 of tap 27, which is 1 (bias gradient)
    for (int i = t; i < (kWgradCells / 8) * (S::kMGroups - 27 * kCg) * 8; i += kConvThreads) {
        const int row = i % 8, rest = i / 8;
        const int kg = rest % (kWgradCells / 8), mg = 27 * kCg + rest / (kWgradCells / 8);
        const uint32_t one = mg == 27 * kCg ? 0x3F80u : 0u;  // BF16 1.0 in channel 0
        *reinterpret_cast<uint4*>(As + (kg * S::kMGroups + mg) * 128 + row * 16) = make_uint4(one, 0, 0, 0);
    }
    for (int i = t; i < static_cast<int>(S::kBBytes / 16u); i += kConvThreads) reinterpret_cast<uint4*>(Bs)[i] = make_uint4(0, 0, 0, 0);
    if (t == 0) tc::mbar_init(&bar, 1);
    if (warp == 0) tc::tmem_alloc(&tmem_slot, S::kTmemCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 16, true, true);
    const uint32_t a_base = tc::smem_addr(As), b_base = tc::smem_addr(Bs);
    const uint32_t chunks = (a.n + kWgradCells - 1) / kWgradCells;
    uint32_t phase = 0;
    bool any = false, ok = true;
    for (uint32_t chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x) {
        const uint32_t q0 = chunk * kWgradCells;
        for (int i = t; i < kWgradCells * 27 * kCg; i += kConvThreads) {
            const int cell = i % kWgradCells, rest = i / kWgradCells;
            const int tap = rest / kCg, cg = rest % kCg;
            const uint32_t q = q0 + cell;
            bool inside = q < a.n;
            uint32_t nq = 0;
            if (inside) {
                const uint32_t row = q / a.nx;
                const int x = static_cast<int>(q - row * a.nx) + tap % 3 - 1;
                const uint32_t zr = row / a.ny;
                const int y = static_cast<int>(row - zr * a.ny) + (tap / 3) % 3 - 1, z = static_cast<int>(zr) + tap / 9 - 1;
                inside = x >= 0 && x < a.nx && y >= 0 && y < a.ny && z >= 0 && z < a.nz;
                nq = inside ? (static_cast<uint32_t>(z) * a.ny + y) * a.nx + x : 0u;
            }
            const uint4 v = inside ? __ldg(reinterpret_cast<const uint4*>(a.in) + static_cast<size_t>(nq) * kCg + cg) : make_uint4(0, 0, 0, 0);
            const int mg = tap * kCg + cg, kg = cell / 8;
            *reinterpret_cast<uint4*>(As + (kg * S::kMGroups + mg) * 128 + (cell % 8) * 16) = v;
        }
        for (int i = t; i < kWgradCells * (a.gc / 8); i += kConvThreads) {
            const int cell = i % kWgradCells, ng = i / kWgradCells;
            const uint32_t q = q0 + cell;
            const uint4 v = q < a.n ? __ldg(reinterpret_cast<const uint4*>(a.g) + static_cast<size_t>(q) * (a.gc / 8) + ng) : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4*>(Bs + ((cell / 8) * 2 + ng) * 128 + (cell % 8) * 16) = v;
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) {
#pragma unroll 1
            for (int mt = 0; mt < S::kMTiles; ++mt)
#pragma unroll 1
                for (int k = 0; k < kWgradCells / 16; ++k) {
                    // K step k: cell groups 2k, 2k + 1 (LBO: next cell group); SBO: next 8 rows of M (or N)
                    const uint64_t ad = tc::smem_desc(a_base + (2 * k * S::kMGroups + mt * 16) * 128u, S::kMGroups * 128u, 128u);
                    const uint64_t bd = tc::smem_desc(b_base + (2 * k * 2) * 128u, 256u, 128u);
                    tc::mma_bf16(tmem + mt * 16, ad, bd, idesc, (any || k > 0) ? 1u : 0u);
                }
            tc::commit(&bar);
        }
        __syncwarp();
        ok = __syncthreads_and(tc::mbar_wait(&bar, phase, kSpinCycles) ? 1 : 0) != 0;
        phase ^= 1u;
        any = true;
        if (!ok) {
            if (t == 0) atomicOr(a.error, 1u);
            break;
        }
        tc::fence_after_sync();
    }
    float* out = a.partial + static_cast<size_t>(blockIdx.x) * S::kMPad * 16;
    for (int mt = 0; mt < S::kMTiles; ++mt) {
        float v[16];
        if (any && ok) {
            tc::tmem_load16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + mt * 16, v);
        } else {
#pragma unroll
            for (int c = 0; c < 16; ++c) v[c] = 0.0f;
        }
        float4* o = reinterpret_cast<float4*>(out + static_cast<size_t>(mt * 128 + t) * 16);
#pragma unroll
        for (int c = 0; c < 4; ++c) o[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, S::kTmemCols);
}

// grad[w(tap, ci, co)] (+)= sum over blocks of partial[b][tap * cin_store + ci][co]; grad[bias co] likewise from
// row 27 * cin_store.
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, int blocks, int m_pad, int cin_store, int cin, int cout, int accumulate, float* __restrict__ grad) {
    const int wcount = 27 * cin * cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < wcount + cout; i += gridDim.x * blockDim.x) {
        int row, co;
        if (i < wcount) {
            co = i % cout;
            const int ci = (i / cout) % cin, tap = i / (cout * cin);
            row = tap * cin_store + ci;
        } else {
            co = i - wcount;
            row = 27 * cin_store;
        }
        float sum = 0.0f;
        for (int b = 0; b < blocks; ++b) sum += partial[(static_cast<size_t>(b) * m_pad + row) * 16 + co];
        grad[i] = accumulate ? grad[i] + sum : sum;
    }
}

// ------------------------------------------------------------------------------------------ glue
__device__ __forceinline__ void load_bf16x8(const __nv_bfloat16* p, float v[8]) {
    const uint4 u = __ldg(reinterpret_cast<const uint4*>(p));
    const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(&u);
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = __bfloat162float(b[c]);
}
__device__ __forceinline__ void store_bf16x8(__nv_bfloat16* p, const float v[8]) {
    *reinterpret_cast<uint4*>(p) = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]), pack_bf16x2(v[6], v[7]));
}
__device__ __forceinline__ void cell_of(const VolumeDims& d, uint32_t q, int& x, int& y, int& z) {
    const uint32_t row = q / d.nx;
    x = static_cast<int>(q - row * d.nx);
    z = static_cast<int>(row / d.ny);
    y = static_cast<int>(row - static_cast<uint32_t>(z) * d.ny);
}
__device__ __forceinline__ uint32_t cell_at(const VolumeDims& d, int x, int y, int z) { return (static_cast<uint32_t>(z) * d.ny + y) * d.nx + x; }

// sum of squares into *out (FP64)
__global__ void sumsq_kernel(const float* __restrict__ v, uint32_t n, double* __restrict__ out) {
    double s = 0.0;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) s += static_cast<double>(v[q]) * v[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(out, s);
}

// X0[q] = (r[q] * s, fluid, 0, ...), s = sqrt(n / ||r||^2) (0 when r = 0); r = r_sel[*parity] when parity is given.
__global__ void net_input_kernel(VolumeDims d, const float* __restrict__ r0, const float* __restrict__ r1, const int* __restrict__ parity, const double* __restrict__ norm2, const uint8_t* __restrict__ occ, __nv_bfloat16* __restrict__ x0, const uint32_t* __restrict__ skip) {
    if (skip && *skip) return;
    const float* r = (parity && *parity) ? r1 : r0;
    const double nn = *norm2;
    const float s = nn > 0.0 ? static_cast<float>(sqrt(static_cast<double>(d.n) / nn)) : 0.0f;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < d.n; q += gridDim.x * blockDim.x) {
        float v[8] = {r[q] * s, occ[q] == 0 ? 1.0f : 0.0f, 0, 0, 0, 0, 0, 0};
        store_bf16x8(x0 + static_cast<size_t>(q) * 8, v);
    }
}

// coarse[Q][c] = mean of the existing children fine[q][c]
template <int C>
__global__ void pool_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ fine, __nv_bfloat16* __restrict__ coarse, const uint32_t* __restrict__ skip) {
    if (skip && *skip) return;
    for (uint32_t Q = blockIdx.x * blockDim.x + threadIdx.x; Q < c.n; Q += gridDim.x * blockDim.x) {
        int X, Y, Z;
        cell_of(c, Q, X, Y, Z);
        float acc[C] = {};
        int count = 0;
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                    if (x >= f.nx || y >= f.ny || z >= f.nz) continue;
                    ++count;
                    const __nv_bfloat16* p = fine + static_cast<size_t>(cell_at(f, x, y, z)) * C;
#pragma unroll
                    for (int h = 0; h < C / 8; ++h) {
                        float v[8];
                        load_bf16x8(p + 8 * h, v);
#pragma unroll
                        for (int k = 0; k < 8; ++k) acc[8 * h + k] += v[k];
                    }
                }
        const float inv = 1.0f / static_cast<float>(count);
#pragma unroll
        for (int h = 0; h < C / 8; ++h) {
            float v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = acc[8 * h + k] * inv;
            store_bf16x8(coarse + static_cast<size_t>(Q) * C + 8 * h, v);
        }
    }
}

// out[q][c] = coarse[parent(q)][c] + skip[q][c]
template <int C>
__global__ void up_add_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip, __nv_bfloat16* __restrict__ out, const uint32_t* __restrict__ off) {
    if (off && *off) return;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < f.n; q += gridDim.x * blockDim.x) {
        int x, y, z;
        cell_of(f, q, x, y, z);
        const uint32_t Q = cell_at(c, x / 2, y / 2, z / 2);
#pragma unroll
        for (int h = 0; h < C / 8; ++h) {
            float a[8], b[8];
            load_bf16x8(coarse + static_cast<size_t>(Q) * C + 8 * h, a);
            load_bf16x8(skip + static_cast<size_t>(q) * C + 8 * h, b);
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] += b[k];
            store_bf16x8(out + static_cast<size_t>(q) * C + 8 * h, a);
        }
    }
}

// Backward of up (sum over the children), then the ReLU gate of the coarse activation: dc[Q] = (sum df[q]) * [act > 0]
template <int C>
__global__ void up_bwd_relu_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ dfine, const __nv_bfloat16* __restrict__ act, __nv_bfloat16* __restrict__ dcoarse) {
    for (uint32_t Q = blockIdx.x * blockDim.x + threadIdx.x; Q < c.n; Q += gridDim.x * blockDim.x) {
        int X, Y, Z;
        cell_of(c, Q, X, Y, Z);
        float acc[C] = {};
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                    if (x >= f.nx || y >= f.ny || z >= f.nz) continue;
                    const __nv_bfloat16* p = dfine + static_cast<size_t>(cell_at(f, x, y, z)) * C;
#pragma unroll
                    for (int h = 0; h < C / 8; ++h) {
                        float v[8];
                        load_bf16x8(p + 8 * h, v);
#pragma unroll
                        for (int k = 0; k < 8; ++k) acc[8 * h + k] += v[k];
                    }
                }
#pragma unroll
        for (int h = 0; h < C / 8; ++h) {
            float g[8], v[8];
            load_bf16x8(act + static_cast<size_t>(Q) * C + 8 * h, g);
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = g[k] > 0.0f ? acc[8 * h + k] : 0.0f;
            store_bf16x8(dcoarse + static_cast<size_t>(Q) * C + 8 * h, v);
        }
    }
}

// Backward of pool (each child gets its parent's gradient / children count) plus the skip gradient, then the ReLU
// gate of the fine activation: df[q] = (skip[q] + dc[parent] / count) * [act > 0]
template <int C>
__global__ void pool_bwd_add_relu_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ skip, const __nv_bfloat16* __restrict__ dcoarse, const __nv_bfloat16* __restrict__ act, __nv_bfloat16* __restrict__ dfine) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < f.n; q += gridDim.x * blockDim.x) {
        int x, y, z;
        cell_of(f, q, x, y, z);
        const int X = x / 2, Y = y / 2, Z = z / 2;
        const int cx = min(2, f.nx - 2 * X), cy = min(2, f.ny - 2 * Y), cz = min(2, f.nz - 2 * Z);
        const float inv = 1.0f / static_cast<float>(cx * cy * cz);
        const uint32_t Q = cell_at(c, X, Y, Z);
#pragma unroll
        for (int h = 0; h < C / 8; ++h) {
            float s[8], d[8], g[8];
            load_bf16x8(skip + static_cast<size_t>(q) * C + 8 * h, s);
            load_bf16x8(dcoarse + static_cast<size_t>(Q) * C + 8 * h, d);
            load_bf16x8(act + static_cast<size_t>(q) * C + 8 * h, g);
#pragma unroll
            for (int k = 0; k < 8; ++k) s[k] = g[k] > 0.0f ? s[k] + d[k] * inv : 0.0f;
            store_bf16x8(dfine + static_cast<size_t>(q) * C + 8 * h, s);
        }
    }
}

// out[q] = fluid ? y[q] / s : 0 with s the input scale of net_input_kernel.
__global__ void net_output_kernel(VolumeDims d, const float* __restrict__ y, const double* __restrict__ norm2, const uint8_t* __restrict__ occ, float* __restrict__ out) {
    const double nn = *norm2;
    const float inv_s = nn > 0.0 ? static_cast<float>(sqrt(nn / static_cast<double>(d.n))) : 0.0f;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < d.n; q += gridDim.x * blockDim.x) out[q] = occ[q] == 0 ? y[q] * inv_s : 0.0f;
}

// Loss of one sample: L = sum_fluid (y - s t)^2 / sum_fluid (s t)^2 (s the input scale); dy = dL/dy into channel 0 of
// gy ([n][8] BF16), L added into *loss. tt = sum_fluid t^2 (from sumsq of the masked target).
__global__ void net_loss_kernel(VolumeDims d, const float* __restrict__ y, const float* __restrict__ target, const uint8_t* __restrict__ occ, const double* __restrict__ norm2, const double* __restrict__ tt, __nv_bfloat16* __restrict__ gy, double* __restrict__ loss) {
    const double nn = *norm2;
    const double s = nn > 0.0 ? sqrt(static_cast<double>(d.n) / nn) : 0.0;
    const double denom = s * s * *tt;
    const float scale = denom > 0.0 ? static_cast<float>(2.0 / denom) : 0.0f;
    double l = 0.0;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < d.n; q += gridDim.x * blockDim.x) {
        const bool fluid = occ[q] == 0;
        const float e = fluid ? y[q] - static_cast<float>(s) * target[q] : 0.0f;
        l += static_cast<double>(e) * e;
        float v[8] = {scale * e, 0, 0, 0, 0, 0, 0, 0};
        store_bf16x8(gy + static_cast<size_t>(q) * 8, v);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && denom > 0.0) atomicAdd(loss, l / denom);
}

// masked copy for the target norm: out[q] = fluid ? t[q] : 0
__global__ void mask_fluid_kernel(uint32_t n, const float* __restrict__ t, const uint8_t* __restrict__ occ, float* __restrict__ out) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) out[q] = occ[q] == 0 ? t[q] : 0.0f;
}

// Adam on the FP32 parameters: m, v moments, bias-corrected step (step >= 1); grad scaled by `gscale`.
__global__ void adam_kernel(int count, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps, int step, float gscale) {
    const float c1 = 1.0f / (1.0f - powf(b1, static_cast<float>(step))), c2 = 1.0f / (1.0f - powf(b2, static_cast<float>(step)));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float gi = g[i] * gscale;
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// bias16[c] = bias[c] for c < cout, else 0
__global__ void bias16_kernel(const float* __restrict__ bias, int cout, float* __restrict__ out) {
    const int c = threadIdx.x;
    if (c < 16) out[c] = c < cout ? bias[c] : 0.0f;
}

}  // namespace

cudaError_t launch_conv3(const VolumeDims& d, int cin_store, const __nv_bfloat16* in, const uint8_t* wpack, const float* bias, int relu, const __nv_bfloat16* gate, __nv_bfloat16* out, int cout_store, float* out_f32, unsigned* error, cudaStream_t s, const uint32_t* skip) {
    if (d.n == 0) return cudaSuccess;
    if ((cin_store != 8 && cin_store != 16) || (cout_store != 8 && cout_store != 16) || error == nullptr) return cudaErrorInvalidValue;
    ConvArgs a{};
    a.in = in;
    a.wpack = wpack;
    a.bias = bias;
    a.gate = gate;
    a.out = out;
    a.out_f32 = out_f32;
    a.error = error;
    a.skip = skip;
    a.relu = relu;
    a.cout_store = cout_store;
    a.nx = d.nx;
    a.ny = d.ny;
    a.nz = d.nz;
    a.n = d.n;
    return cin_store == 8 ? conv_typed<8>(d, a, s) : conv_typed<16>(d, a, s);
}

cudaError_t launch_pack_conv(const float* w, int cin, int cout, int transpose, uint8_t* pack, cudaStream_t s) {
    pack_conv_kernel<<<32, 256, 0, s>>>(w, cin, cout, transpose, pack);
    return cudaGetLastError();
}


// ------------------------------------------------------------------------------------------ orchestration
namespace {

constexpr int kGlueThreads = 256;
unsigned glue_blocks(uint32_t n) { return std::max(1u, std::min<uint32_t>((n + kGlueThreads - 1) / kGlueThreads, 148u * 8u)); }

template <int CIN>
cudaError_t wgrad_typed(const VolumeDims& d, const WgradArgs& a, int blocks, cudaStream_t s) {
    using S = WgradShape<CIN>;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(wgrad_kernel<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::kSmem));
        if (e == cudaSuccess) e = cudaFuncSetAttribute(wgrad_kernel<CIN>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    wgrad_kernel<CIN><<<blocks, kConvThreads, S::kSmem, s>>>(a);
    return cudaGetLastError();
}

// Blocks of the weight-gradient kernel for a volume of n cells (at most one per SM: the partials buffer holds
// kWgradMaxBlocks of them).
constexpr int kWgradMaxBlocks = 160;
int wgrad_blocks(uint32_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t chunks = (n + kWgradCells - 1) / kWgradCells;
    return static_cast<int>(std::max<uint32_t>(1u, std::min<uint32_t>({chunks, static_cast<uint32_t>(sms), static_cast<uint32_t>(kWgradMaxBlocks)})));
}

// Layer L's weight and bias gradient from its input `in` and its output-side gradient `g` (pre-activation).
cudaError_t layer_wgrad(int L, const VolumeDims& d, const __nv_bfloat16* in, const __nv_bfloat16* g, const NetGrads& G, float* grad, int accumulate, unsigned* error, cudaStream_t s) {
    const int cs = net_store(kNet[L].cin), gs = net_store(kNet[L].cout);
    WgradArgs a{};
    a.in = in;
    a.g = g;
    a.partial = G.partial;
    a.error = error;
    a.gc = gs;
    a.nx = d.nx;
    a.ny = d.ny;
    a.nz = d.nz;
    a.n = d.n;
    const int blocks = wgrad_blocks(d.n);
    cudaError_t e = cs == 8 ? wgrad_typed<8>(d, a, blocks, s) : wgrad_typed<16>(d, a, blocks, s);
    if (e != cudaSuccess) return e;
    wgrad_reduce_kernel<<<16, 256, 0, s>>>(G.partial, blocks, 32 * cs, cs, kNet[L].cin, kNet[L].cout, accumulate, grad + net_param_offset(L));
    return cudaGetLastError();
}

cudaError_t conv_layer(int L, const VolumeDims& d, const NetImages& I, const __nv_bfloat16* in, __nv_bfloat16* out, float* out_f32, unsigned* error, cudaStream_t s, const uint32_t* skip = nullptr) {
    const int relu = L < kNetLayers - 1;
    return launch_conv3(d, net_store(kNet[L].cin), in, I.fwd[L], I.bias16[L], relu, nullptr, out, net_store(kNet[L].cout), out_f32, error, s, skip);
}
// Gradient through layer L's convolution: gin = conv^T(g), gated by `gate` (the layer's input activation when it is
// a ReLU output consumed only by this layer).
cudaError_t conv_layer_bwd(int L, const VolumeDims& d, const NetImages& I, const __nv_bfloat16* g, const __nv_bfloat16* gate, __nv_bfloat16* gin, unsigned* error, cudaStream_t s) {
    return launch_conv3(d, net_store(kNet[L].cout), g, I.bwd[L], nullptr, 0, gate, gin, net_store(kNet[L].cin), nullptr, error, s, nullptr);
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

size_t net_images_bytes() {
    size_t b = 0;
    for (int L = 0; L < kNetLayers; ++L) {
        b += align256(conv_pack_bytes(net_store(kNet[L].cin)));
        if (L > 0) b += align256(conv_pack_bytes(net_store(kNet[L].cout)));
        b += align256(16 * sizeof(float));
    }
    return b;
}

void net_images_bind(NetImages& I, void* base) {
    char* p = static_cast<char*>(base);
    for (int L = 0; L < kNetLayers; ++L) {
        I.fwd[L] = reinterpret_cast<uint8_t*>(p);
        p += align256(conv_pack_bytes(net_store(kNet[L].cin)));
        I.bwd[L] = nullptr;
        if (L > 0) {
            I.bwd[L] = reinterpret_cast<uint8_t*>(p);
            p += align256(conv_pack_bytes(net_store(kNet[L].cout)));
        }
        I.bias16[L] = reinterpret_cast<float*>(p);
        p += align256(16 * sizeof(float));
    }
}

cudaError_t net_pack(const float* w, const NetImages& I, cudaStream_t s) {
    for (int L = 0; L < kNetLayers; ++L) {
        const float* wl = w + net_param_offset(L);
        cudaError_t e = launch_pack_conv(wl, kNet[L].cin, kNet[L].cout, 0, I.fwd[L], s);
        if (e == cudaSuccess && L > 0) e = launch_pack_conv(wl, kNet[L].cin, kNet[L].cout, 1, I.bwd[L], s);
        if (e != cudaSuccess) return e;
        bias16_kernel<<<1, 32, 0, s>>>(wl + net_weight_count(L), kNet[L].cout, I.bias16[L]);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

namespace {
// Buffers of a NetActs / NetGrads, in binding order: (level, channels) per BF16 volume.
struct Slot {
    int level, channels;
};
constexpr Slot kActSlots[] = {{0, 8}, {0, 8}, {0, 8}, {0, 8}, {1, 8}, {1, 8}, {1, 16}, {1, 16}, {2, 16}, {2, 16}};
constexpr Slot kGradSlots[] = {{0, 8}, {0, 8}, {0, 8}, {0, 8}, {1, 8}, {1, 8}, {1, 16}, {1, 16}, {2, 16}, {2, 16}};
void levels_of(const VolumeDims& d0, VolumeDims d[3]) {
    d[0] = d0;
    d[1] = coarse_dims(d[0]);
    d[2] = coarse_dims(d[1]);
}
}  // namespace

size_t net_acts_bytes(const VolumeDims& d0) {
    VolumeDims d[3];
    levels_of(d0, d);
    size_t b = 0;
    for (const Slot& sl : kActSlots) b += align256(static_cast<size_t>(d[sl.level].n) * sl.channels * 2);
    return b + align256(static_cast<size_t>(d0.n) * 4) + align256(16) + align256(16);
}

void net_acts_bind(NetActs& A, void* base, const VolumeDims& d0) {
    levels_of(d0, A.d);
    char* p = static_cast<char*>(base);
    __nv_bfloat16** v[] = {&A.x0, &A.e0, &A.s0, &A.d0, &A.p1, &A.d1, &A.e1, &A.s1, &A.p2, &A.e2};
    for (int i = 0; i < 10; ++i) {
        *v[i] = reinterpret_cast<__nv_bfloat16*>(p);
        p += align256(static_cast<size_t>(A.d[kActSlots[i].level].n) * kActSlots[i].channels * 2);
    }
    A.y = reinterpret_cast<float*>(p);
    p += align256(static_cast<size_t>(d0.n) * 4);
    A.norm2 = reinterpret_cast<double*>(p);
    p += align256(16);
    A.error = reinterpret_cast<unsigned*>(p);
}

size_t net_grads_bytes(const VolumeDims& d0) {
    VolumeDims d[3];
    levels_of(d0, d);
    size_t b = 0;
    for (const Slot& sl : kGradSlots) b += align256(static_cast<size_t>(d[sl.level].n) * sl.channels * 2);
    return b + align256(static_cast<size_t>(kWgradMaxBlocks) * 512 * 16 * 4) + align256(static_cast<size_t>(d0.n) * 4) + align256(16);
}

void net_grads_bind(NetGrads& G, void* base, const VolumeDims& d0) {
    VolumeDims d[3];
    levels_of(d0, d);
    char* p = static_cast<char*>(base);
    __nv_bfloat16** v[] = {&G.gy, &G.ge, &G.gs0, &G.ga, &G.gd, &G.gp1, &G.gs1, &G.gb, &G.gc, &G.gp2};
    for (int i = 0; i < 10; ++i) {
        *v[i] = reinterpret_cast<__nv_bfloat16*>(p);
        p += align256(static_cast<size_t>(d[kGradSlots[i].level].n) * kGradSlots[i].channels * 2);
    }
    G.partial = reinterpret_cast<float*>(p);
    p += align256(static_cast<size_t>(kWgradMaxBlocks) * 512 * 16 * 4);
    G.tmask = reinterpret_cast<float*>(p);
    p += align256(static_cast<size_t>(d0.n) * 4);
    G.sums = reinterpret_cast<double*>(p);
}

cudaError_t net_forward(const NetImages& I, const NetActs& A, const float* r0, const float* r1, const int* parity, const double* norm2, const uint8_t* occ, cudaStream_t s, const uint32_t* skip) {
    const VolumeDims *d = A.d;
    cudaError_t e;
    if (norm2 == nullptr) {
        if ((e = cudaMemsetAsync(A.norm2, 0, sizeof(double), s)) != cudaSuccess) return e;
        sumsq_kernel<<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(r0, d[0].n, A.norm2);
        norm2 = A.norm2;
    }
    net_input_kernel<<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(d[0], r0, r1, parity, norm2, occ, A.x0, skip);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = conv_layer(0, d[0], I, A.x0, A.e0, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    pool_kernel<8><<<glue_blocks(d[1].n), kGlueThreads, 0, s>>>(d[0], d[1], A.e0, A.p1, skip);
    if ((e = conv_layer(1, d[1], I, A.p1, A.e1, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    pool_kernel<16><<<glue_blocks(d[2].n), kGlueThreads, 0, s>>>(d[1], d[2], A.e1, A.p2, skip);
    if ((e = conv_layer(2, d[2], I, A.p2, A.e2, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    up_add_kernel<16><<<glue_blocks(d[1].n), kGlueThreads, 0, s>>>(d[1], d[2], A.e2, A.e1, A.s1, skip);
    if ((e = conv_layer(3, d[1], I, A.s1, A.d1, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    up_add_kernel<8><<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(d[0], d[1], A.d1, A.e0, A.s0, skip);
    if ((e = conv_layer(4, d[0], I, A.s0, A.d0, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    return conv_layer(5, d[0], I, A.d0, nullptr, A.y, A.error, s, skip);
}

cudaError_t net_output(const NetActs& A, const double* norm2, const uint8_t* occ, float* out, cudaStream_t s) {
    net_output_kernel<<<glue_blocks(A.d[0].n), kGlueThreads, 0, s>>>(A.d[0], A.y, norm2 ? norm2 : A.norm2, occ, out);
    return cudaGetLastError();
}

cudaError_t net_backward(const NetImages& I, const NetActs& A, const NetGrads& G, const double* norm2, const float* target, const uint8_t* occ, float* grad, int accumulate, cudaStream_t s) {
    const VolumeDims* d = A.d;
    if (norm2 == nullptr) norm2 = A.norm2;
    cudaError_t e = cudaMemsetAsync(G.sums, 0, sizeof(double), s);  // target norm^2 (the loss accumulates)
    if (e != cudaSuccess) return e;
    mask_fluid_kernel<<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(d[0].n, target, occ, G.tmask);
    sumsq_kernel<<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(G.tmask, d[0].n, G.sums);
    net_loss_kernel<<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(d[0], A.y, target, occ, norm2, G.sums, G.gy, G.sums + 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // f: y = conv(d0); e: d0 = relu(conv(s0))
    if ((e = layer_wgrad(5, d[0], A.d0, G.gy, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(5, d[0], I, G.gy, A.d0, G.ge, A.error, s)) != cudaSuccess) return e;
    if ((e = layer_wgrad(4, d[0], A.s0, G.ge, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(4, d[0], I, G.ge, nullptr, G.gs0, A.error, s)) != cudaSuccess) return e;
    // s0 = up(d1) + e0; d1 = relu(conv_d(s1))
    up_bwd_relu_kernel<8><<<glue_blocks(d[1].n), kGlueThreads, 0, s>>>(d[0], d[1], G.gs0, A.d1, G.gd);
    if ((e = layer_wgrad(3, d[1], A.s1, G.gd, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(3, d[1], I, G.gd, nullptr, G.gs1, A.error, s)) != cudaSuccess) return e;
    // s1 = up(e2) + e1; e2 = relu(conv_c(p2))
    up_bwd_relu_kernel<16><<<glue_blocks(d[2].n), kGlueThreads, 0, s>>>(d[1], d[2], G.gs1, A.e2, G.gc);
    if ((e = layer_wgrad(2, d[2], A.p2, G.gc, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(2, d[2], I, G.gc, nullptr, G.gp2, A.error, s)) != cudaSuccess) return e;
    // p2 = pool(e1); e1 = relu(conv_b(p1))
    pool_bwd_add_relu_kernel<16><<<glue_blocks(d[1].n), kGlueThreads, 0, s>>>(d[1], d[2], G.gs1, G.gp2, A.e1, G.gb);
    if ((e = layer_wgrad(1, d[1], A.p1, G.gb, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(1, d[1], I, G.gb, nullptr, G.gp1, A.error, s)) != cudaSuccess) return e;
    // p1 = pool(e0); e0 = relu(conv_a(x0))
    pool_bwd_add_relu_kernel<8><<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(d[0], d[1], G.gs0, G.gp1, A.e0, G.ga);
    return layer_wgrad(0, d[0], A.x0, G.ga, G, grad, accumulate, A.error, s);
}

cudaError_t net_adam(float* w, const float* grad, float* m, float* v, float lr, int step, float gscale, const NetImages& I, cudaStream_t s) {
    adam_kernel<<<(kNetParams + 255) / 256, 256, 0, s>>>(kNetParams, w, grad, m, v, lr, 0.9f, 0.999f, 1e-8f, step, gscale);
    const cudaError_t e = cudaGetLastError();
    return e != cudaSuccess ? e : net_pack(w, I, s);
}

}  // namespace smoke_b200
