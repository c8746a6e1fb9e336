// Kernels of the learned preconditioner (unet.h): tcgen05 implicit-GEMM 3x3x3 convolutions on channels-last BF16
// volumes with FP32 accumulation in tensor memory, their weight gradients, and the glue between the U-Net's layers.
//
// Convolution as a GEMM: D[cell][co] = sum over k = (tap, ci) of A[cell][k] * B[co][k], with A[cell][(tap, ci)] =
// in[cell + offset(tap)][ci] (0 outside the volume). A block computes tiles of M = 128 cells and N = NC output
// channels (one chunk of the output; gridDim.y chunks cover all of them) with its chunk of the weights resident in
// shared memory. A producer warp streams each tile's input halo box into shared memory with TMA and issues the
// MMAs into one of two tensor-memory accumulators; four epilogue warps read the other accumulator back (bias,
// ReLU, gate) and store, so a tile's epilogue overlaps the next tile's loads and MMAs.
#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "tcgen05.cuh"
#include "pdl.cuh"
#include "unet.h"

namespace smoke_b200 {
namespace {

constexpr int kEpiThreads = 128;                  // epilogue warps 0-3: thread t owns tensor-memory lane t
constexpr int kConvThreads = kEpiThreads + 32;    // + warp 4: TMA producer and MMA issuer (lane 0)
constexpr long long kSpinCycles = 4000000000ll;   // ~2 s: default bound of every completion wait

// Tiles of 8 x 16 x 1 cells (M = 128 rows, row m = cell (m % 8, m / 8) of the tile). A tile's input is its halo box
// of 10 x 18 x 3 cells, brought into shared memory by one TMA load per 8-channel plane (zeros outside the volume):
// cell (x, y, z) of the box at byte ((z * 18 + y) * 10 + x) * 16 of its plane. The A operand of tap (dx, dy, dz) is
// that box read from offset ((1 + dz) * 18 + 1 + dy) * 160 + (1 + dx) * 16: every 8 cells of a tile row are 8
// consecutive 16-byte rows of the box, i.e. one core matrix, and the next tile row starts one box row (160 bytes) on
// (SBO). So no im2col copy exists: each MMA reads its two K columns (two taps of an 8-channel input, or two channel
// planes of one tap) straight from the boxes.
constexpr int kTX = 8, kTY = 16;
constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = 3;
constexpr uint32_t kRow = kHX * 16;                 // bytes of one box row (SBO)
constexpr uint32_t kBox = kHX * kHY * kHZ * 16;     // 8640 bytes per plane
constexpr uint32_t kPlane = 8704;                   // plane pitch: box + zero slack, 128-aligned
__host__ __device__ constexpr uint32_t tap_offset(int tap) {
    return ((tap / 9) * 18 + (tap / 3) % 3) * 160u + (tap % 3) * 16u;  // (dz + 1, dy + 1, dx + 1) of the tap
}
// the padding tap's K column (tap 26's rows, 16 bytes on) stays inside the plane's zero slack
static_assert(tap_offset(26) + 16 + 15 * kRow + 128 <= kPlane, "zero slack");
static_assert(tap_offset(26) + 15 * kRow + 128 <= kBox, "box");

// CS stored input channels, NC output channels per block. A K group is one plane (CS = 8: its 27 taps paired into
// 14 MMAs, the 28th tap zero) or two planes (16 channels: one MMA per tap); a tile has CS / 16 groups.
template <int CS, int NC>
struct ConvShape {
    static constexpr int kGP = CS == 8 ? 1 : 2;      // planes per group (one TMA stage)
    static constexpr int kGroups = CS / (8 * kGP);
    static constexpr int kStages = 3;
    static constexpr uint32_t kStage = kGP * kPlane;
    static constexpr int kMmas = CS == 8 ? 14 : 27;  // MMAs of one group (K = 16 each)
    static constexpr uint32_t kBChunk = static_cast<uint32_t>(conv_taps(CS) * CS * NC * 2);
    static_assert(kBChunk % 16 == 0, "bulk copy size");
    static constexpr uint32_t kSmem = kStages * kStage + kBChunk;
    static constexpr uint32_t kTmemCols = 2 * NC < 32 ? 32u : static_cast<uint32_t>(2 * NC);  // two accumulators
    static_assert(NC == 16 || NC == 32, "N per block");
    static_assert(kSmem <= 200 * 1024, "shared memory");
};

struct ConvArgs {
    const __nv_bfloat16* in;
    const uint8_t* wpack;
    const float* bias;
    const __nv_bfloat16* gate;
    __nv_bfloat16* out;
    float* out_f32;
    unsigned* error;
    const uint32_t* skip;  // optional: the launch does nothing when *skip is nonzero
    long long wait_cycles; // bound of every wait
    int drop_loads;        // test only: the producer expects its loads but never issues them
    int relu, cout_store;
    int nx, ny, nz;
    uint32_t n;
};


__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

template <int CS, int NC>
__global__ void __launch_bounds__(kConvThreads) conv3_kernel(const __grid_constant__ ConvArgs a, const __grid_constant__ CUtensorMap map) {
    using S = ConvShape<CS, NC>;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* Bs = smem + S::kStages * S::kStage;
    __shared__ uint64_t full[S::kStages], freed[S::kStages], done[2], drained[2], wbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    pdl_trigger();
    const int t = threadIdx.x, warp = t >> 5;
    const int chunk = blockIdx.y;
    for (int st = 0; st < S::kStages; ++st)  // the slack after each box stays zero (read by the padding tap, times zero weights)
        for (int p = 0; p < S::kGP; ++p)
            for (uint32_t i = t; i < (kPlane - kBox) / 16u; i += kConvThreads) reinterpret_cast<uint4*>(smem + st * S::kStage + p * kPlane + kBox)[i] = make_uint4(0, 0, 0, 0);
    if (t == 0) {
        for (int st = 0; st < S::kStages; ++st) {
            tc::mbar_init(&full[st], 1);
            tc::mbar_init(&freed[st], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&done[b], 1);
            tc::mbar_init(&drained[b], kEpiThreads);
        }
        tc::mbar_init(&wbar, 1);
        abort_flag = 0;
    }
    if (warp == 0) tc::tmem_alloc(&tmem_slot, S::kTmemCols);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    pdl_wait();  // the set-up above overlaps the previous kernel's tail
    if (a.skip && *a.skip) {  // uniform: every block reads the same word
        if (warp == 0) tc::tmem_free(tmem, S::kTmemCols);
        return;
    }
    const long long wait = a.wait_cycles > 0 ? a.wait_cycles : kSpinCycles;
    volatile int* abort = &abort_flag;
    const int ntx = (a.nx + kTX - 1) / kTX, nty = (a.ny + kTY - 1) / kTY;
    const uint32_t tiles = static_cast<uint32_t>(ntx) * nty * a.nz;
    const uint32_t my_tiles = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0u;

    if (warp == 4) {
        if ((t & 31) == 0) {
            // ---------------------------------------------------------------- producer and MMA issuer
            const uint32_t items = my_tiles * S::kGroups;  // (tile, K group) pairs in order
            constexpr uint32_t idesc = tc::idesc_bf16_f32(128, NC, false, false);
            const uint32_t b_base = tc::smem_addr(Bs);
            uint32_t loaded = 0, consumed = 0, issued = 0;  // items whose TMA was issued / whose box arrived / whose MMAs were issued
            bool ok = true;
            // this block's chunk of the packed weights: bulk copies into shared memory, overlapping the first boxes
            bool weights_ready = false;
            {
                const uint8_t* wsrc = a.wpack + static_cast<size_t>(chunk) * S::kBChunk;
                tc::mbar_arrive_expect_tx(&wbar, S::kBChunk);
                for (uint32_t off = 0; off < S::kBChunk; off += 16384u) tc::bulk_copy_g2s(Bs + off, wsrc + off, min(16384u, S::kBChunk - off), &wbar);
            }
            auto issue_load = [&](uint32_t k) -> bool {
                const int st = static_cast<int>(k % S::kStages);
                // stage st last held item k - kStages: its MMAs must have completed before the box is overwritten
                if (k >= static_cast<uint32_t>(S::kStages) && !tc::mbar_wait_or_abort(&freed[st], ((k / S::kStages) - 1u) & 1u, wait, abort)) return false;
                const uint32_t tile = blockIdx.x + (k / S::kGroups) * gridDim.x;
                const int g = static_cast<int>(k % S::kGroups);
                const int tx = static_cast<int>(tile % ntx), rest = static_cast<int>(tile / ntx);
                const int ty = rest % nty, tz = rest / nty;
                tc::mbar_arrive_expect_tx(&full[st], S::kGP * kBox);
                if (!a.drop_loads) {
                    for (int p = 0; p < S::kGP; ++p) tc::tma_load_4d(smem + st * S::kStage + p * kPlane, &map, 8 * (g * S::kGP + p), tx * kTX - 1, ty * kTY - 1, tz - 1, &full[st]);
                    loaded = k + 1;
                }
                return true;
            };
            for (uint32_t k = 0; k < static_cast<uint32_t>(S::kStages - 1) && k < items && ok; ++k) ok = issue_load(k);
            for (uint32_t i = 0; ok && i < items; ++i) {
                const uint32_t jl = i / S::kGroups;
                const int g = static_cast<int>(i % S::kGroups), b = static_cast<int>(jl & 1u), st = static_cast<int>(i % S::kStages);
                // accumulator b last held tile jl - 2: its epilogue must have read it out
                if (g == 0 && jl >= 2 && !tc::mbar_wait_or_abort(&drained[b], ((jl >> 1) - 1u) & 1u, wait, abort)) {
                    ok = false;
                    break;
                }
                if (!tc::mbar_wait_or_abort(&full[st], (i / S::kStages) & 1u, wait, abort)) {
                    ok = false;
                    break;
                }
                consumed = i + 1;
                if (!weights_ready) {
                    if (!tc::mbar_wait_or_abort(&wbar, 0, wait, abort)) {
                        ok = false;
                        break;
                    }
                    weights_ready = true;
                }
                tc::fence_after_sync();
                const uint32_t a_base = tc::smem_addr(smem + st * S::kStage);
#pragma unroll 1
                for (int k = 0; k < S::kMmas; ++k) {
                    uint32_t start, lbo, k0;
                    if constexpr (CS == 8) {  // taps 2k and 2k + 1 (tap 27: zero weights, any finite A)
                        start = a_base + tap_offset(2 * k);
                        lbo = 2 * k + 1 < 27 ? tap_offset(2 * k + 1) - tap_offset(2 * k) : 16u;
                        k0 = 16u * k;
                    } else {  // tap k, channel planes 2g and 2g + 1
                        start = a_base + tap_offset(k);
                        lbo = kPlane;
                        k0 = static_cast<uint32_t>(k * CS + 16 * g);
                    }
                    const uint64_t bd = tc::smem_desc(b_base + (k0 / 8u) * (NC / 8) * 128u, (NC / 8) * 128u, 128u);
                    tc::mma_bf16(tmem + static_cast<uint32_t>(b * NC), tc::smem_desc(start, lbo, kRow), bd, idesc, (g > 0 || k > 0) ? 1u : 0u);
                }
                tc::commit(&freed[st]);
                if (g == S::kGroups - 1) tc::commit(&done[b]);
                issued = i + 1;
                if (i + S::kStages - 1 < items && !issue_load(i + S::kStages - 1)) ok = false;
            }
            if (!ok) {
                atomicOr(a.error, 1u);
                *abort = 1;
            }
            // nothing may still write this block's shared or tensor memory when it exits: every issued box must have
            // landed and the last MMAs completed (bounded waits again)
            for (uint32_t k = consumed; k < loaded; ++k) tc::mbar_wait(&full[k % S::kStages], (k / S::kStages) & 1u, wait);
            if (!weights_ready) tc::mbar_wait(&wbar, 0, wait);
            if (issued > 0) tc::mbar_wait(&freed[(issued - 1) % S::kStages], ((issued - 1) / S::kStages) & 1u, wait);
        }
    } else {
        // -------------------------------------------------------------------- epilogue (threads 0-127)
        float bias[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) bias[c] = a.bias ? __ldg(a.bias + chunk * NC + c) : 0.0f;
        const int n0 = chunk * NC;
        const int stored = min(NC, a.cout_store - n0);  // output channels this chunk stores (fewer than NC for cout <= 8)
        for (uint32_t jl = 0; jl < my_tiles; ++jl) {
            const int b = static_cast<int>(jl & 1u);
            // warp-uniform outcome: the accumulator loads below are warp-collective
            const bool ready = __all_sync(0xffffffffu, tc::mbar_wait_or_abort(&done[b], (jl >> 1) & 1u, wait, abort) ? 1 : 0) != 0;
            if (!ready) {
                if (t == 0) atomicOr(a.error, 1u);
                *abort = 1;
                break;
            }
            tc::fence_after_sync();
            float acc[NC];
#pragma unroll
            for (int c = 0; c < NC; c += 16) tc::tmem_load16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(b * NC + c), acc + c);
            tc::fence_before_sync();
            tc::mbar_arrive(&drained[b]);
            const uint32_t tile = blockIdx.x + jl * gridDim.x;
            const int tx = static_cast<int>(tile % ntx), rest = static_cast<int>(tile / ntx);
            const int x = tx * kTX + (t & 7), y = (rest % nty) * kTY + (t >> 3), z = rest / nty;
            if (x < a.nx && y < a.ny) {
                const uint32_t q = (static_cast<uint32_t>(z) * a.ny + y) * a.nx + x;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    acc[c] += bias[c];
                    if (a.relu) acc[c] = fmaxf(acc[c], 0.0f);
                }
                if (a.gate) {
                    const uint4* g = reinterpret_cast<const uint4*>(a.gate + static_cast<size_t>(q) * a.cout_store + n0);
#pragma unroll
                    for (int h = 0; h < NC / 8; ++h) {
                        if (8 * h >= stored) break;
                        const uint4 gv = __ldg(g + h);
                        const __nv_bfloat16* gb = reinterpret_cast<const __nv_bfloat16*>(&gv);
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            if (!(__bfloat162float(gb[c]) > 0.0f)) acc[h * 8 + c] = 0.0f;
                    }
                }
                if (a.out_f32 && chunk == 0) a.out_f32[q] = acc[0];
                if (a.out) {
                    uint4* o = reinterpret_cast<uint4*>(a.out + static_cast<size_t>(q) * a.cout_store + n0);
#pragma unroll
                    for (int h = 0; h < NC / 8; ++h)
                        if (8 * h < stored)
                            o[h] = make_uint4(pack_bf16x2(acc[8 * h], acc[8 * h + 1]), pack_bf16x2(acc[8 * h + 2], acc[8 * h + 3]), pack_bf16x2(acc[8 * h + 4], acc[8 * h + 5]),
                                          pack_bf16x2(acc[8 * h + 6], acc[8 * h + 7]));
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, S::kTmemCols);
}

// ------------------------------------------------------------------------------------------ single-output layer
// The network's last convolution has one output channel (16 -> 1). Padding it to N = 16 output channels runs 16x the
// MMAs it needs, each reading a 4 KB A operand. Here the N = 16 accumulator columns are 16 output z-planes instead: a
// tile is 8 x 16 cells x kBandZ planes (z0 .. z0 + 15), its inputs are the 18 planes z0 - 1 .. z0 + 16 (six 3-deep halo
// boxes), and input plane j (z' = z0 - 1 + j) contributes through each in-plane tap (dx, dy) with the banded matrix
// B[j][tap][n][ci] = w[dz][dy][dx][ci] for dz = j - 1 - n in {-1, 0, 1}, else 0. So a tile costs 18 x 9 MMAs
// instead of 16 x 27, and every A operand (the box at the tap's offset) is read once per input plane.
// The 18 banded matrices of a tap are windows of one tall matrix: rows i = 0 .. 32 (16 bytes = 8 channels each, in
// two K column blocks of kBandRows rows) hold dz = 16 - i (zero but for i = 15, 16, 17), and the matrix of input plane
// j is rows 17 - j .. 32 - j (a descriptor starting 16 (17 - j) bytes in, SBO 128 bytes, LBO one column block). 9.5 KB
// of weights instead of 83 KB, so three blocks fit on an SM.
constexpr int kBandZ = 16;                                                // output planes per tile (N)
constexpr int kBandJ = kBandZ + 2;                                        // input planes per tile
constexpr int kBandRows = kBandZ + kBandJ - 1;                            // rows of a tap's tall matrix
constexpr uint32_t kBandBlock = static_cast<uint32_t>(kBandRows) * 16u;   // one K column block (LBO)
constexpr uint32_t kBandTap = 2u * kBandBlock;                            // a tap's two column blocks (16 channels)
constexpr uint32_t kBandBytes = 9u * kBandTap;                            // 9504
static_assert(kBandBytes % 16 == 0, "bulk copy size");
constexpr int kBandStages = 3;
constexpr uint32_t kBandStage = 2 * kPlane;                               // one 3-deep box of both 8-channel planes
constexpr uint32_t kBandSmem = kBandStages * kBandStage + kBandBytes;
constexpr int kBandItems = kBandJ / 3;                                    // boxes per tile
static_assert(kBandJ % 3 == 0, "whole boxes");

__global__ void __launch_bounds__(kConvThreads) conv3_band_kernel(const __grid_constant__ ConvArgs a, const __grid_constant__ CUtensorMap map) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* Bs = smem + kBandStages * kBandStage;
    __shared__ uint64_t full[kBandStages], freed[kBandStages], done[2], drained[2], wbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    constexpr uint32_t kCols = 32;  // two 16-column accumulators
    pdl_trigger();
    const int t = threadIdx.x, warp = t >> 5;
    if (t == 0) {
        for (int st = 0; st < kBandStages; ++st) {
            tc::mbar_init(&full[st], 1);
            tc::mbar_init(&freed[st], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&done[b], 1);
            tc::mbar_init(&drained[b], kEpiThreads);
        }
        tc::mbar_init(&wbar, 1);
        abort_flag = 0;
    }
    if (warp == 0) tc::tmem_alloc(&tmem_slot, kCols);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    pdl_wait();  // the set-up above overlaps the previous kernel's tail
    if (a.skip && *a.skip) {  // uniform: every block reads the same word
        if (warp == 0) tc::tmem_free(tmem, kCols);
        return;
    }
    const long long wait = a.wait_cycles > 0 ? a.wait_cycles : kSpinCycles;
    volatile int* abort = &abort_flag;
    const int ntx = (a.nx + kTX - 1) / kTX, nty = (a.ny + kTY - 1) / kTY, ntz = (a.nz + kBandZ - 1) / kBandZ;
    const uint32_t tiles = static_cast<uint32_t>(ntx) * nty * ntz;
    const uint32_t my_tiles = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0u;

    if (warp == 4) {
        if ((t & 31) == 0) {
            // ---------------------------------------------------------------- producer and MMA issuer
            const uint32_t items = my_tiles * kBandItems;  // (tile, box) pairs in order
            constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 16, false, false);
            const uint32_t b_base = tc::smem_addr(Bs);
            uint32_t loaded = 0, consumed = 0, issued = 0;
            bool ok = true;
            bool weights_ready = false;
            tc::mbar_arrive_expect_tx(&wbar, kBandBytes);
            for (uint32_t off = 0; off < kBandBytes; off += 16384u) tc::bulk_copy_g2s(Bs + off, a.wpack + off, min(16384u, kBandBytes - off), &wbar);
            auto issue_load = [&](uint32_t k) -> bool {
                const int st = static_cast<int>(k % kBandStages);
                if (k >= static_cast<uint32_t>(kBandStages) && !tc::mbar_wait_or_abort(&freed[st], ((k / kBandStages) - 1u) & 1u, wait, abort)) return false;
                const uint32_t tile = blockIdx.x + (k / kBandItems) * gridDim.x;
                const int box = static_cast<int>(k % kBandItems);
                const int tx = static_cast<int>(tile % ntx), rest = static_cast<int>(tile / ntx);
                const int ty = rest % nty, tz = rest / nty;
                tc::mbar_arrive_expect_tx(&full[st], 2 * kBox);
                if (!a.drop_loads) {
                    for (int p = 0; p < 2; ++p) tc::tma_load_4d(smem + st * kBandStage + p * kPlane, &map, 8 * p, tx * kTX - 1, ty * kTY - 1, tz * kBandZ - 1 + 3 * box, &full[st]);
                    loaded = k + 1;
                }
                return true;
            };
            for (uint32_t k = 0; k < static_cast<uint32_t>(kBandStages - 1) && k < items && ok; ++k) ok = issue_load(k);
            for (uint32_t i = 0; ok && i < items; ++i) {
                const uint32_t jl = i / kBandItems;
                const int box = static_cast<int>(i % kBandItems), b = static_cast<int>(jl & 1u), st = static_cast<int>(i % kBandStages);
                if (box == 0 && jl >= 2 && !tc::mbar_wait_or_abort(&drained[b], ((jl >> 1) - 1u) & 1u, wait, abort)) {
                    ok = false;
                    break;
                }
                if (!tc::mbar_wait_or_abort(&full[st], (i / kBandStages) & 1u, wait, abort)) {
                    ok = false;
                    break;
                }
                consumed = i + 1;
                if (!weights_ready) {
                    if (!tc::mbar_wait_or_abort(&wbar, 0, wait, abort)) {
                        ok = false;
                        break;
                    }
                    weights_ready = true;
                }
                tc::fence_after_sync();
                const uint32_t a_base = tc::smem_addr(smem + st * kBandStage);
#pragma unroll 1
                for (int k = 0; k < 27; ++k) {  // box plane zz = k / 9 (input plane j = 3 box + zz), in-plane tap k % 9
                    const int j = 3 * box + k / 9, tap = k % 9;
                    const uint64_t bd = tc::smem_desc(b_base + static_cast<uint32_t>(tap) * kBandTap + static_cast<uint32_t>(kBandJ - 1 - j) * 16u, kBandBlock, 128u);
                    tc::mma_bf16(tmem + static_cast<uint32_t>(b * 16), tc::smem_desc(a_base + tap_offset(k), kPlane, kRow), bd, idesc, (box > 0 || k > 0) ? 1u : 0u);
                }
                tc::commit(&freed[st]);
                if (box == kBandItems - 1) tc::commit(&done[b]);
                issued = i + 1;
                if (i + kBandStages - 1 < items && !issue_load(i + kBandStages - 1)) ok = false;
            }
            if (!ok) {
                atomicOr(a.error, 1u);
                *abort = 1;
            }
            // nothing may still write this block's shared or tensor memory when it exits (bounded waits again)
            for (uint32_t k = consumed; k < loaded; ++k) tc::mbar_wait(&full[k % kBandStages], (k / kBandStages) & 1u, wait);
            if (!weights_ready) tc::mbar_wait(&wbar, 0, wait);
            if (issued > 0) tc::mbar_wait(&freed[(issued - 1) % kBandStages], ((issued - 1) / kBandStages) & 1u, wait);
        }
    } else {
        // -------------------------------------------------------------------- epilogue (threads 0-127)
        const float bias = a.bias ? __ldg(a.bias) : 0.0f;
        const uint32_t slab = static_cast<uint32_t>(a.nx) * a.ny;
        for (uint32_t jl = 0; jl < my_tiles; ++jl) {
            const int b = static_cast<int>(jl & 1u);
            const bool ready = __all_sync(0xffffffffu, tc::mbar_wait_or_abort(&done[b], (jl >> 1) & 1u, wait, abort) ? 1 : 0) != 0;
            if (!ready) {
                if (t == 0) atomicOr(a.error, 1u);
                *abort = 1;
                break;
            }
            tc::fence_after_sync();
            float acc[16];
            tc::tmem_load16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(b * 16), acc);
            tc::fence_before_sync();
            tc::mbar_arrive(&drained[b]);
            const uint32_t tile = blockIdx.x + jl * gridDim.x;
            const int tx = static_cast<int>(tile % ntx), rest = static_cast<int>(tile / ntx);
            const int x = tx * kTX + (t & 7), y = (rest % nty) * kTY + (t >> 3), z0 = (rest / nty) * kBandZ;
            if (x < a.nx && y < a.ny) {
                const uint32_t q0 = static_cast<uint32_t>(y) * a.nx + x;
#pragma unroll
                for (int n = 0; n < kBandZ; ++n)
                    if (z0 + n < a.nz) a.out_f32[static_cast<uint32_t>(z0 + n) * slab + q0] = acc[n] + bias;
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, kCols);
}

// Banded operand image of the single-output layer (w: W[tap][ci][0], tap = (dz + 1) * 9 + (dy + 1) * 3 + dx + 1, 16
// input channels): for in-plane tap t and column block c, row i holds channels 8c .. 8c + 7 of the weight of
// dz = 16 - i (0 outside [-1, 1]), at byte t * kBandTap + c * kBandBlock + i * 16 + (k % 8) * 2.
__global__ void pack_band_kernel(const float* __restrict__ w, int cin, uint8_t* __restrict__ band) {
    const int total = 9 * 2 * kBandRows * 8;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int kk = e % 8, i = (e / 8) % kBandRows, c = (e / (8 * kBandRows)) % 2, tap = e / (16 * kBandRows);
        const int k = 8 * c + kk, dz = kBandJ - 2 - i;
        float v = 0.0f;
        if (dz >= -1 && dz <= 1 && k < cin) v = w[static_cast<size_t>((dz + 1) * 9 + tap) * cin + k];
        const size_t off = static_cast<size_t>(tap) * kBandTap + static_cast<size_t>(c) * kBandBlock + static_cast<size_t>(i) * 16 + kk * 2;
        *reinterpret_cast<__nv_bfloat16*>(band + off) = __float2bfloat16_rn(v);
    }
}

// Operand image of B for a convolution whose input has `cs` stored channels: K = taps x cs rows (tap-major), N =
// the output channels in chunks of nc; K-major core matrices, element (co, k) of chunk co / nc at byte
// ((k / 8) * (nc / 8) + (co % nc) / 8) * 128 + (co % 8) * 16 + (k % 8) * 2 of that chunk's image.
__global__ void pack_conv_kernel(const float* __restrict__ w, int cin, int cout, int transpose, int cs, uint8_t* __restrict__ pack) {
    const int in_ch = transpose ? cout : cin, out_ch = transpose ? cin : cout;
    const int nc = conv_nc(cs, out_ch), cpad = net_cout_pad(out_ch);
    const int K = conv_taps(cs) * cs;
    const size_t chunk_bytes = static_cast<size_t>(K) * nc * 2;
    const int total = K * cpad;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int k = i / cpad, co = i % cpad;
        const int tap = k / cs, ci = k % cs;
        float v = 0.0f;
        if (tap < 27 && ci < in_ch && co < out_ch) {
            // forward: W[tap][ci][co]; backward-data: input channel = forward output, mirrored tap
            v = transpose ? w[(static_cast<size_t>(26 - tap) * cin + co) * cout + ci] : w[(static_cast<size_t>(tap) * cin + ci) * cout + co];
        }
        const int cl = co % nc;
        const size_t off = (co / nc) * chunk_bytes + static_cast<size_t>((k / 8) * (nc / 8) + cl / 8) * 128 + (cl % 8) * 16 + (k % 8) * 2;
        *reinterpret_cast<__nv_bfloat16*>(pack + off) = __float2bfloat16_rn(v);
    }
}

// Resident blocks of a kernel per device: by shared memory (its dynamic bytes plus about 2 KB of static data and
// the per-block reservation), by tensor memory (512 columns per SM) and by threads; at most 8 per SM. Cached.
int resident_blocks(const void* kernel, size_t smem, uint32_t tmem_cols, int threads) {
    static std::mutex lock;
    static std::map<std::pair<const void*, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> guard(lock);
    auto it = cache.find({kernel, dev});
    if (it != cache.end()) return it->second;
    int sms = 1, smem_sm = 0, threads_sm = 2048;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    int per_sm = std::max(1, smem_sm / static_cast<int>(smem + 2048));
    if (tmem_cols > 0) per_sm = std::min(per_sm, static_cast<int>(512u / tmem_cols));
    per_sm = std::min({per_sm, threads_sm / threads, 8});
    const int r = std::max(1, sms * std::max(1, per_sm));
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

// Tensor map of a channels-last BF16 volume with `cs` stored channels: dimensions (channel, x, y, z), boxes of
// 8 channels x the halo of one tile, zeros outside. Every box starts at a channel coordinate that is a multiple of
// 8 (16 bytes).
cudaError_t halo_map(CUtensorMap* map, int cs, const ConvArgs& a) {
    const auto encode = tensor_map_encoder();
    if (encode == nullptr) return cudaErrorNotSupported;
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(cs), static_cast<cuuint64_t>(a.nx), static_cast<cuuint64_t>(a.ny), static_cast<cuuint64_t>(a.nz)};
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(cs) * 2, static_cast<cuuint64_t>(a.nx) * cs * 2, static_cast<cuuint64_t>(a.nx) * a.ny * cs * 2};
    const cuuint32_t box[4] = {8, kHX, kHY, kHZ};
    const cuuint32_t step[4] = {1, 1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(a.in), dims, strides, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}


template <int CS, int NC>
cudaError_t conv_typed(const VolumeDims& d, int chunks, const ConvArgs& a, cudaStream_t s) {
    using S = ConvShape<CS, NC>;
    static std::once_flag once;
    static cudaError_t configured = cudaSuccess;
    std::call_once(once, [] {  // all of the unified L1 as shared memory, so that several blocks fit on an SM
        configured = cudaFuncSetAttribute(conv3_kernel<CS, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::kSmem));
        if (configured == cudaSuccess) configured = cudaFuncSetAttribute(conv3_kernel<CS, NC>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    });
    if (configured != cudaSuccess) return configured;
    if ((reinterpret_cast<uintptr_t>(a.in) & 15u) != 0) return cudaErrorMisalignedAddress;
    CUtensorMap map;
    const cudaError_t e = halo_map(&map, CS, a);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = static_cast<uint64_t>((d.nx + kTX - 1) / kTX) * ((d.ny + kTY - 1) / kTY) * d.nz;
    const int resident = resident_blocks(reinterpret_cast<const void*>(conv3_kernel<CS, NC>), S::kSmem, S::kTmemCols, kConvThreads);
    const int gx = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(tiles, static_cast<uint64_t>(std::max(1, resident / chunks)))));
    launch_pdl(conv3_kernel<CS, NC>, dim3(gx, chunks), dim3(kConvThreads), S::kSmem, s, a, map);
    return cudaGetLastError();
}

// The single-output layer's forward (conv3_band_kernel): FP32 output only, 16 stored input channels.
cudaError_t conv_band(const VolumeDims& d, const ConvArgs& a, cudaStream_t s) {
    static std::once_flag once;
    static cudaError_t configured = cudaSuccess;
    std::call_once(once, [] {
        configured = cudaFuncSetAttribute(conv3_band_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kBandSmem));
        if (configured == cudaSuccess) configured = cudaFuncSetAttribute(conv3_band_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    });
    if (configured != cudaSuccess) return configured;
    if ((reinterpret_cast<uintptr_t>(a.in) & 15u) != 0 || a.out_f32 == nullptr || a.error == nullptr) return cudaErrorInvalidValue;
    CUtensorMap map;
    const cudaError_t e = halo_map(&map, 16, a);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = static_cast<uint64_t>((d.nx + kTX - 1) / kTX) * ((d.ny + kTY - 1) / kTY) * ((d.nz + kBandZ - 1) / kBandZ);
    const int resident = resident_blocks(reinterpret_cast<const void*>(conv3_band_kernel), kBandSmem, 32, kConvThreads);
    const int gx = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(tiles, static_cast<uint64_t>(resident))));
    launch_pdl(conv3_band_kernel, dim3(gx), dim3(kConvThreads), kBandSmem, s, a, map);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------ weight gradient
// dW[tap][ci][co] = sum over cells q of in[q + offset(tap)][ci] * g[q][co], as a GEMM with M = (tap, ci) rows
// (row tap * CS + ci; row 27 * CS is 1 for every cell, which makes its D row the bias gradient sum_q g[q][co]; M
// padded to a multiple of 128), N = GN gradient channels, K = cells. Both operands are MN-major in shared memory: a
// core matrix is 8 cells (K) x 16 bytes = 8 consecutive channels, so every 16-byte channel vector lands as one
// core-matrix row. A block owns MT M-tiles (blockIdx.y picks which) and a share of the cells (blockIdx.x), keeps
// its D in tensor memory and writes it as a partial sum; wgrad_reduce adds the partials.
constexpr int kWgradCells = 64;  // cells (K) per gather round: 8 core-matrix groups, 4 MMA K-steps
constexpr int kWgradMaxBlocksX = 296;

__host__ __device__ constexpr int wgrad_mpad(int cs) { return ((27 * cs + 1 + 127) / 128) * 128; }
__host__ __device__ constexpr int wgrad_mt(int gn) { return gn >= 128 ? 2 : 4; }

template <int CS, int GN>
struct WgradShape {
    static constexpr int kMPad = wgrad_mpad(CS);
    static constexpr int kMT = wgrad_mt(GN);             // M-tiles per block
    static constexpr int kMGroups = kMT * 16;            // core matrices along M per block
    static constexpr uint32_t kABytes = (kWgradCells / 8) * kMGroups * 128u;
    static constexpr uint32_t kBBytes = (kWgradCells / 8) * (GN / 8) * 128u;
    static constexpr uint32_t kSmem = kABytes + kBBytes;
    static constexpr uint32_t kTmemCols = kMT * GN;      // 64..256
    static_assert(kTmemCols >= 32 && kTmemCols <= 256 && (kTmemCols & (kTmemCols - 1)) == 0, "tensor memory columns");
    // dynamic shared memory requested at launch: blocks of 256 tensor-memory columns ask for enough that at most two
    // fit on an SM (2 x 256 = all 512 columns), so no block's allocation waits for another's
    static constexpr uint32_t kSmemLaunch = kTmemCols >= 256 && kSmem < 80u * 1024u ? 80u * 1024u : kSmem;
};

struct WgradArgs {
    const __nv_bfloat16* in;  // [n][CS]
    const __nv_bfloat16* g;   // [n][GN]
    float* partial;           // [gridDim.x][kMPad][GN]
    unsigned* error;
    int nx, ny, nz;
    uint32_t n;
};

template <int CS, int GN>
__global__ void __launch_bounds__(kEpiThreads) wgrad_kernel(const __grid_constant__ WgradArgs a) {
    using S = WgradShape<CS, GN>;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* As = smem;
    uint8_t* Bs = smem + S::kABytes;
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5;
    constexpr int kCg = CS / 8;
    constexpr int kRealGroups = 27 * kCg;                        // row groups read from the input
    const int g0 = blockIdx.y * S::kMGroups;                     // first row group of this block
    const int m_tiles = min(S::kMT, S::kMPad / 128 - static_cast<int>(blockIdx.y) * S::kMT);
    // constant row groups (bias row, padding): 1 in channel 0 of group 27 * kCg, zero elsewhere
    for (int i = t; i < (kWgradCells / 8) * S::kMGroups * 8; i += kEpiThreads) {
        const int row = i % 8, rest = i / 8;
        const int kg = rest % (kWgradCells / 8), mg = rest / (kWgradCells / 8);
        if (g0 + mg < kRealGroups) continue;
        const uint32_t one = g0 + mg == kRealGroups ? 0x3F80u : 0u;  // BF16 1.0 in channel 0
        *reinterpret_cast<uint4*>(As + (kg * S::kMGroups + mg) * 128 + row * 16) = make_uint4(one, 0, 0, 0);
    }
    if (t == 0) tc::mbar_init(&bar, 1);
    if (warp == 0) tc::tmem_alloc(&tmem_slot, S::kTmemCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, GN, true, true);
    const uint32_t a_base = tc::smem_addr(As), b_base = tc::smem_addr(Bs);
    const uint32_t chunks = (a.n + kWgradCells - 1) / kWgradCells;
    const int real_here = max(0, min(S::kMGroups, kRealGroups - g0));  // input row groups of this block
    uint32_t phase = 0;
    bool any = false, ok = true;
    for (uint32_t chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x) {
        const uint32_t q0 = chunk * kWgradCells;
        for (int i = t; i < kWgradCells * real_here; i += kEpiThreads) {
            const int cell = i % kWgradCells, mg = i / kWgradCells;
            const int G = g0 + mg, tap = G / kCg, cg = G % kCg;
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
            *reinterpret_cast<uint4*>(As + ((cell / 8) * S::kMGroups + mg) * 128 + (cell % 8) * 16) = v;
        }
        for (int i = t; i < kWgradCells * (GN / 8); i += kEpiThreads) {
            const int cell = i % kWgradCells, ng = i / kWgradCells;
            const uint32_t q = q0 + cell;
            const uint4 v = q < a.n ? __ldg(reinterpret_cast<const uint4*>(a.g) + static_cast<size_t>(q) * (GN / 8) + ng) : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4*>(Bs + ((cell / 8) * (GN / 8) + ng) * 128 + (cell % 8) * 16) = v;
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) {
#pragma unroll 1
            for (int mt = 0; mt < m_tiles; ++mt)
#pragma unroll 1
                for (int k = 0; k < kWgradCells / 16; ++k) {
                    // K step k: cell groups 2k, 2k + 1 (LBO: next cell group); SBO: next 8 rows of M (or N)
                    const uint64_t ad = tc::smem_desc(a_base + (2 * k * S::kMGroups + mt * 16) * 128u, S::kMGroups * 128u, 128u);
                    const uint64_t bd = tc::smem_desc(b_base + (2 * k * (GN / 8)) * 128u, (GN / 8) * 128u, 128u);
                    tc::mma_bf16(tmem + static_cast<uint32_t>(mt * GN), ad, bd, idesc, (any || k > 0) ? 1u : 0u);
                }
            tc::commit(&bar);
        }
        __syncwarp();
        ok = __syncthreads_and(tc::mbar_wait(&bar, phase, kSpinCycles) ? 1 : 0) != 0;
        phase ^= 1u;
        any = true;
        if (!ok) {
            if (t == 0) {
                atomicOr(a.error, 1u);
                tc::mbar_wait(&bar, phase ^ 1u, kSpinCycles);  // once more, so no MMA is left running at exit
            }
            break;
        }
        tc::fence_after_sync();
    }
    float* out = a.partial + static_cast<size_t>(blockIdx.x) * S::kMPad * GN;
    for (int mt = 0; mt < m_tiles; ++mt) {
        const int row = (blockIdx.y * S::kMT + mt) * 128 + t;
        for (int c = 0; c < GN; c += 16) {
            float v[16];
            if (any && ok) {
                tc::tmem_load16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(mt * GN + c), v);
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.0f;
            }
            float4* o = reinterpret_cast<float4*>(out + static_cast<size_t>(row) * GN + c);
#pragma unroll
            for (int i = 0; i < 4; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, S::kTmemCols);
}

// grad[w(tap, ci, co)] (+)= sum over blocks of partial[b][tap * cs + ci][co]; grad[bias co] likewise from row
// 27 * cs.
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, int blocks, int m_pad, int gn, int cs, int cin, int cout, int accumulate, float* __restrict__ grad) {
    const int wcount = 27 * cin * cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < wcount + cout; i += gridDim.x * blockDim.x) {
        int row, co;
        if (i < wcount) {
            co = i % cout;
            const int ci = (i / cout) % cin, tap = i / (cout * cin);
            row = tap * cs + ci;
        } else {
            co = i - wcount;
            row = 27 * cs;
        }
        float sum = 0.0f;
        for (int b = 0; b < blocks; ++b) sum += partial[(static_cast<size_t>(b) * m_pad + row) * gn + co];
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
    pdl_trigger();
    pdl_wait();
    if (skip && *skip) return;
    const float* r = (parity && *parity) ? r1 : r0;
    const double nn = *norm2;
    const float s = nn > 0.0 ? static_cast<float>(sqrt(static_cast<double>(d.n) / nn)) : 0.0f;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < d.n; q += gridDim.x * blockDim.x) {
        float v[8] = {r[q] * s, occ[q] == 0 ? 1.0f : 0.0f, 0, 0, 0, 0, 0, 0};
        store_bf16x8(x0 + static_cast<size_t>(q) * 8, v);
    }
}

// The glue kernels run one thread per (cell, group of 8 channels): work item i is cell i / (C / 8), channels
// 8 * (i % (C / 8)) .. +7, so consecutive threads read consecutive 16-byte channel groups.

// coarse[Q][c] = mean of the existing children fine[q][c]
template <int C>
__global__ void pool_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ fine, __nv_bfloat16* __restrict__ coarse, const uint32_t* __restrict__ skip) {
    pdl_trigger();
    pdl_wait();
    if (skip && *skip) return;
    constexpr int G = C / 8;
    const uint64_t items = static_cast<uint64_t>(c.n) * G;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < items; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t Q = static_cast<uint32_t>(i / G);
        const int h = static_cast<int>(i % G);
        int X, Y, Z;
        cell_of(c, Q, X, Y, Z);
        float acc[8] = {};
        int count = 0;
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                    if (x >= f.nx || y >= f.ny || z >= f.nz) continue;
                    ++count;
                    float v[8];
                    load_bf16x8(fine + static_cast<size_t>(cell_at(f, x, y, z)) * C + 8 * h, v);
#pragma unroll
                    for (int k = 0; k < 8; ++k) acc[k] += v[k];
                }
        const float inv = 1.0f / static_cast<float>(count);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] *= inv;
        store_bf16x8(coarse + static_cast<size_t>(Q) * C + 8 * h, acc);
    }
}

// out[q][c] = coarse[parent(q)][c] + skip[q][c]
template <int C>
__global__ void up_add_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip, __nv_bfloat16* __restrict__ out, const uint32_t* __restrict__ off) {
    pdl_trigger();
    pdl_wait();
    if (off && *off) return;
    constexpr int G = C / 8;
    const uint64_t items = static_cast<uint64_t>(f.n) * G;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < items; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t q = static_cast<uint32_t>(i / G);
        const int h = static_cast<int>(i % G);
        int x, y, z;
        cell_of(f, q, x, y, z);
        const uint32_t Q = cell_at(c, x / 2, y / 2, z / 2);
        float a[8], b[8];
        load_bf16x8(coarse + static_cast<size_t>(Q) * C + 8 * h, a);
        load_bf16x8(skip + static_cast<size_t>(q) * C + 8 * h, b);
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] += b[k];
        store_bf16x8(out + static_cast<size_t>(q) * C + 8 * h, a);
    }
}

// Backward of up (sum over the children), then the ReLU gate of the coarse activation: dc[Q] = (sum df[q]) * [act > 0]
template <int C>
__global__ void up_bwd_relu_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ dfine, const __nv_bfloat16* __restrict__ act, __nv_bfloat16* __restrict__ dcoarse) {
    constexpr int G = C / 8;
    const uint64_t items = static_cast<uint64_t>(c.n) * G;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < items; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t Q = static_cast<uint32_t>(i / G);
        const int h = static_cast<int>(i % G);
        int X, Y, Z;
        cell_of(c, Q, X, Y, Z);
        float acc[8] = {};
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                    if (x >= f.nx || y >= f.ny || z >= f.nz) continue;
                    float v[8];
                    load_bf16x8(dfine + static_cast<size_t>(cell_at(f, x, y, z)) * C + 8 * h, v);
#pragma unroll
                    for (int k = 0; k < 8; ++k) acc[k] += v[k];
                }
        float g[8];
        load_bf16x8(act + static_cast<size_t>(Q) * C + 8 * h, g);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = g[k] > 0.0f ? acc[k] : 0.0f;
        store_bf16x8(dcoarse + static_cast<size_t>(Q) * C + 8 * h, acc);
    }
}

// Backward of pool (each child gets its parent's gradient / children count) plus the skip gradient, then the ReLU
// gate of the fine activation: df[q] = (skip[q] + dc[parent] / count) * [act > 0]
template <int C>
__global__ void pool_bwd_add_relu_kernel(VolumeDims f, VolumeDims c, const __nv_bfloat16* __restrict__ skip, const __nv_bfloat16* __restrict__ dcoarse, const __nv_bfloat16* __restrict__ act, __nv_bfloat16* __restrict__ dfine) {
    constexpr int G = C / 8;
    const uint64_t items = static_cast<uint64_t>(f.n) * G;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < items; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t q = static_cast<uint32_t>(i / G);
        const int h = static_cast<int>(i % G);
        int x, y, z;
        cell_of(f, q, x, y, z);
        const int X = x / 2, Y = y / 2, Z = z / 2;
        const int cx = min(2, f.nx - 2 * X), cy = min(2, f.ny - 2 * Y), cz = min(2, f.nz - 2 * Z);
        const float inv = 1.0f / static_cast<float>(cx * cy * cz);
        const uint32_t Q = cell_at(c, X, Y, Z);
        float s[8], d[8], g[8];
        load_bf16x8(skip + static_cast<size_t>(q) * C + 8 * h, s);
        load_bf16x8(dcoarse + static_cast<size_t>(Q) * C + 8 * h, d);
        load_bf16x8(act + static_cast<size_t>(q) * C + 8 * h, g);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = g[k] > 0.0f ? s[k] + d[k] * inv : 0.0f;
        store_bf16x8(dfine + static_cast<size_t>(q) * C + 8 * h, s);
    }
}

// out[q] = fluid ? y[q] / s : 0 with s the input scale of net_input_kernel.
__global__ void net_output_kernel(VolumeDims d, const float* __restrict__ y, const double* __restrict__ norm2, const uint8_t* __restrict__ occ, float* __restrict__ out) {
    const double nn = *norm2;
    const float inv_s = nn > 0.0 ? static_cast<float>(sqrt(nn / static_cast<double>(d.n))) : 0.0f;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < d.n; q += gridDim.x * blockDim.x) out[q] = occ[q] == 0 ? y[q] * inv_s : 0.0f;
}

// Loss of one sample: L = sum_fluid (y - s t)^2 / sum_fluid (s t)^2 (s the input scale); dy = dL/dy into channel 0 of
// gy ([n][16] BF16, the other channels 0), L added into *loss. tt = sum_fluid t^2 (from sumsq of the masked target).
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
        const float v[8] = {scale * e, 0, 0, 0, 0, 0, 0, 0};
        const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        store_bf16x8(gy + static_cast<size_t>(q) * 16, v);
        store_bf16x8(gy + static_cast<size_t>(q) * 16 + 8, z);
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

// padded bias: out[c] = bias[c] for c < cout, else 0 (cpad entries)
__global__ void bias_pad_kernel(const float* __restrict__ bias, int cout, int cpad, float* __restrict__ out) {
    for (int c = threadIdx.x; c < cpad; c += blockDim.x) out[c] = c < cout ? bias[c] : 0.0f;
}

}  // namespace

cudaError_t launch_conv3(const VolumeDims& d, int cin_store, int cout, const __nv_bfloat16* in, const uint8_t* wpack, const float* bias, int relu, const __nv_bfloat16* gate, __nv_bfloat16* out,
                         int cout_store, float* out_f32, unsigned* error, cudaStream_t s, const uint32_t* skip, long long wait_cycles, int drop_loads) {
    if (d.n == 0) return cudaSuccess;
    const int nc = conv_nc(cin_store, cout), cpad = net_cout_pad(cout);
    // stored output channels: all padded columns, or (cout <= 8) the 8 channels of a narrow output
    const bool stores_ok = cout_store % 8 == 0 && (cout_store >= cpad || (cout <= 8 && cout_store == 8));
    if (error == nullptr || cout < 1 || cout > 128 || ((out != nullptr || gate != nullptr) && !stores_ok)) return cudaErrorInvalidValue;
    ConvArgs a{};
    a.in = in;
    a.wpack = wpack;
    a.bias = bias;
    a.gate = gate;
    a.out = out;
    a.out_f32 = out_f32;
    a.error = error;
    a.skip = skip;
    a.wait_cycles = wait_cycles;
    a.drop_loads = drop_loads;
    a.relu = relu;
    a.cout_store = cout_store;
    a.nx = d.nx;
    a.ny = d.ny;
    a.nz = d.nz;
    a.n = d.n;
    const int chunks = cpad / nc;
    switch (cin_store * 1000 + nc) {
        case 8016: return conv_typed<8, 16>(d, chunks, a, s);
        case 16016: return conv_typed<16, 16>(d, chunks, a, s);
        case 16032: return conv_typed<16, 32>(d, chunks, a, s);
        case 32016: return conv_typed<32, 16>(d, chunks, a, s);
        case 32032: return conv_typed<32, 32>(d, chunks, a, s);
        case 64016: return conv_typed<64, 16>(d, chunks, a, s);
        case 64032: return conv_typed<64, 32>(d, chunks, a, s);
        case 128016: return conv_typed<128, 16>(d, chunks, a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pack_conv(const float* w, int cin, int cout, int transpose, int cin_store, uint8_t* pack, cudaStream_t s) {
    pack_conv_kernel<<<64, 256, 0, s>>>(w, cin, cout, transpose, cin_store, pack);
    return cudaGetLastError();
}


// ------------------------------------------------------------------------------------------ orchestration
namespace {

constexpr int kGlueThreads = 256;
unsigned glue_blocks(uint64_t n) { return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n + kGlueThreads - 1) / kGlueThreads, 148u * 8u))); }
// Blocks of a per-(cell, 8-channel group) glue kernel over n cells of C channels.
unsigned glue_blocks_c(uint32_t n, int c) { return glue_blocks(static_cast<uint64_t>(n) * (c / 8)); }

// Blocks of the weight-gradient kernel along the cells for a volume of n cells and gy M-chunks.
int wgrad_blocks_x(uint32_t n, int gy) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t chunks = (n + kWgradCells - 1) / kWgradCells;
    const uint32_t want = static_cast<uint32_t>(std::max(1, 2 * sms / gy));
    return static_cast<int>(std::max<uint32_t>(1u, std::min<uint32_t>({chunks, want, static_cast<uint32_t>(kWgradMaxBlocksX)})));
}
int wgrad_gy(int cs, int gn) { return (wgrad_mpad(cs) / 128 + wgrad_mt(gn) - 1) / wgrad_mt(gn); }

template <int CS, int GN>
cudaError_t wgrad_typed(const WgradArgs& a, int bx, cudaStream_t s) {
    using S = WgradShape<CS, GN>;
    static std::once_flag once;
    static cudaError_t configured = cudaSuccess;
    std::call_once(once, [] {
        configured = cudaFuncSetAttribute(wgrad_kernel<CS, GN>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::kSmemLaunch));
        if (configured == cudaSuccess) configured = cudaFuncSetAttribute(wgrad_kernel<CS, GN>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    });
    if (configured != cudaSuccess) return configured;
    wgrad_kernel<CS, GN><<<dim3(bx, wgrad_gy(CS, GN)), kEpiThreads, S::kSmemLaunch, s>>>(a);
    return cudaGetLastError();
}

// Layer L's weight and bias gradient from its input `in` and its output-side gradient `g` (pre-activation).
cudaError_t layer_wgrad(int L, const VolumeDims& d, const __nv_bfloat16* in, const __nv_bfloat16* g, const NetGrads& G, float* grad, int accumulate, unsigned* error, cudaStream_t s) {
    const int cs = net_store(kNet[L].cin), gn = net_grad_store(kNet[L].cout);
    WgradArgs a{};
    a.in = in;
    a.g = g;
    a.partial = G.partial;
    a.error = error;
    a.nx = d.nx;
    a.ny = d.ny;
    a.nz = d.nz;
    a.n = d.n;
    const int bx = wgrad_blocks_x(d.n, wgrad_gy(cs, gn));
    cudaError_t e;
    switch (cs * 1000 + gn) {
        case 8016: e = wgrad_typed<8, 16>(a, bx, s); break;
        case 16032: e = wgrad_typed<16, 32>(a, bx, s); break;
        case 32064: e = wgrad_typed<32, 64>(a, bx, s); break;
        case 64128: e = wgrad_typed<64, 128>(a, bx, s); break;
        case 128064: e = wgrad_typed<128, 64>(a, bx, s); break;
        case 64032: e = wgrad_typed<64, 32>(a, bx, s); break;
        case 32016: e = wgrad_typed<32, 16>(a, bx, s); break;
        case 16016: e = wgrad_typed<16, 16>(a, bx, s); break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    wgrad_reduce_kernel<<<64, 256, 0, s>>>(G.partial, bx, wgrad_mpad(cs), gn, cs, kNet[L].cin, kNet[L].cout, accumulate, grad + net_param_offset(L));
    return cudaGetLastError();
}

// Largest partial-sum buffer (floats) any layer's weight gradient needs on a level-0 volume d0: blocks along the
// cells (at most one per 64 cells of the layer's level, at most kWgradMaxBlocksX) x padded rows x columns.
size_t wgrad_partial_floats(const VolumeDims& d0) {
    VolumeDims d = d0;
    size_t most = 0;
    for (int level = 0; level < kNetLevels; ++level) {
        const size_t bx = std::min<size_t>((d.n + kWgradCells - 1) / kWgradCells, kWgradMaxBlocksX);
        for (int L = 0; L < kNetLayers; ++L) {
            if (kNet[L].level != level) continue;
            const int cs = net_store(kNet[L].cin), gn = net_grad_store(kNet[L].cout);
            most = std::max(most, std::max<size_t>(bx, 1) * wgrad_mpad(cs) * gn);
        }
        d = coarse_dims(d);
    }
    return most;
}

cudaError_t conv_layer(int L, const VolumeDims& d, const NetImages& I, const __nv_bfloat16* in, __nv_bfloat16* out, float* out_f32, unsigned* error, cudaStream_t s, const uint32_t* skip = nullptr) {
    const int relu = L < kNetLayers - 1;
    if (L == kNetLayers - 1 && out == nullptr && out_f32 != nullptr && d.n > 0) {  // the single-output layer: banded
        ConvArgs a{};
        a.in = in;
        a.wpack = I.band;
        a.bias = I.bias[L];
        a.out_f32 = out_f32;
        a.error = error;
        a.skip = skip;
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.n = d.n;
        return conv_band(d, a, s);
    }
    return launch_conv3(d, net_store(kNet[L].cin), kNet[L].cout, in, I.fwd[L], I.bias[L], relu, nullptr, out, net_store(kNet[L].cout), out_f32, error, s, skip);
}
// Gradient through layer L's convolution: gin = conv^T(g), gated by `gate` (the layer's input activation when it is
// a ReLU output consumed only by this layer).
cudaError_t conv_layer_bwd(int L, const VolumeDims& d, const NetImages& I, const __nv_bfloat16* g, const __nv_bfloat16* gate, __nv_bfloat16* gin, unsigned* error, cudaStream_t s) {
    return launch_conv3(d, net_grad_store(kNet[L].cout), kNet[L].cin, g, I.bwd[L], nullptr, 0, gate, gin, net_store(kNet[L].cin), nullptr, error, s, nullptr);
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

size_t net_images_bytes() {
    size_t b = 0;
    for (int L = 0; L < kNetLayers; ++L) {
        b += align256(conv_pack_bytes(net_store(kNet[L].cin), kNet[L].cout));
        if (L > 0) b += align256(conv_pack_bytes(net_grad_store(kNet[L].cout), kNet[L].cin));
        b += align256(net_cout_pad(kNet[L].cout) * sizeof(float));
    }
    return b + align256(kBandBytes);
}

void net_images_bind(NetImages& I, void* base) {
    char* p = static_cast<char*>(base);
    for (int L = 0; L < kNetLayers; ++L) {
        I.fwd[L] = reinterpret_cast<uint8_t*>(p);
        p += align256(conv_pack_bytes(net_store(kNet[L].cin), kNet[L].cout));
        I.bwd[L] = nullptr;
        if (L > 0) {
            I.bwd[L] = reinterpret_cast<uint8_t*>(p);
            p += align256(conv_pack_bytes(net_grad_store(kNet[L].cout), kNet[L].cin));
        }
        I.bias[L] = reinterpret_cast<float*>(p);
        p += align256(net_cout_pad(kNet[L].cout) * sizeof(float));
    }
    I.band = reinterpret_cast<uint8_t*>(p);
}

cudaError_t net_pack(const float* w, const NetImages& I, cudaStream_t s) {
    for (int L = 0; L < kNetLayers; ++L) {
        const float* wl = w + net_param_offset(L);
        cudaError_t e = launch_pack_conv(wl, kNet[L].cin, kNet[L].cout, 0, net_store(kNet[L].cin), I.fwd[L], s);
        if (e == cudaSuccess && L > 0) e = launch_pack_conv(wl, kNet[L].cin, kNet[L].cout, 1, net_grad_store(kNet[L].cout), I.bwd[L], s);
        if (e != cudaSuccess) return e;
        bias_pad_kernel<<<1, 128, 0, s>>>(wl + net_weight_count(L), kNet[L].cout, net_cout_pad(kNet[L].cout), I.bias[L]);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    static_assert(kNet[kNetLayers - 1].cout == 1 && kNet[kNetLayers - 1].cin == 16 && kNet[kNetLayers - 1].level == 0, "the banded layer is 16 -> 1 on level 0");
    pack_band_kernel<<<64, 256, 0, s>>>(w + net_param_offset(kNetLayers - 1), kNet[kNetLayers - 1].cin, I.band);
    return cudaGetLastError();
}

namespace {
// Buffers of a NetActs / NetGrads, in binding order: (level, channels) per BF16 volume.
struct Slot {
    int level, channels;
};
constexpr Slot kActSlots[] = {{0, 8}, {0, 16}, {0, 16}, {1, 16}, {1, 16}, {1, 32}, {1, 32}, {2, 32}, {2, 32}, {2, 64}, {2, 64}, {3, 64}, {3, 64}, {3, 128}};
constexpr Slot kGradSlots[] = {{0, 16}, {0, 16}, {0, 16}, {1, 16}, {1, 16}, {1, 32}, {1, 32}, {2, 32}, {2, 32}, {2, 64}, {2, 64}, {3, 64}, {3, 64}, {3, 128}};
constexpr int kActCount = sizeof(kActSlots) / sizeof(kActSlots[0]);
constexpr int kGradCount = sizeof(kGradSlots) / sizeof(kGradSlots[0]);
void levels_of(const VolumeDims& d0, VolumeDims d[kNetLevels]) {
    d[0] = d0;
    for (int l = 1; l < kNetLevels; ++l) d[l] = coarse_dims(d[l - 1]);
}
}  // namespace

size_t net_acts_bytes(const VolumeDims& d0) {
    VolumeDims d[kNetLevels];
    levels_of(d0, d);
    size_t b = 0;
    for (const Slot& sl : kActSlots) b += align256(static_cast<size_t>(d[sl.level].n) * sl.channels * 2);
    return b + align256(static_cast<size_t>(d0.n) * 4) + align256(16) + align256(16);
}

void net_acts_bind(NetActs& A, void* base, const VolumeDims& d0) {
    levels_of(d0, A.d);
    char* p = static_cast<char*>(base);
    __nv_bfloat16** v[kActCount] = {&A.x0, &A.e0, &A.s0, &A.p1, &A.u1, &A.e1, &A.s1, &A.p2, &A.u2, &A.e2, &A.s2, &A.p3, &A.m3, &A.e3};
    for (int i = 0; i < kActCount; ++i) {
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
    VolumeDims d[kNetLevels];
    levels_of(d0, d);
    size_t b = 0;
    for (const Slot& sl : kGradSlots) b += align256(static_cast<size_t>(d[sl.level].n) * sl.channels * 2);
    return b + align256(wgrad_partial_floats(d0) * 4) + align256(static_cast<size_t>(d0.n) * 4) + align256(16);
}

void net_grads_bind(NetGrads& G, void* base, const VolumeDims& d0) {
    VolumeDims d[kNetLevels];
    levels_of(d0, d);
    char* p = static_cast<char*>(base);
    __nv_bfloat16** v[kGradCount] = {&G.gy, &G.gs0, &G.ge0, &G.gu1, &G.gp1, &G.gs1, &G.ge1, &G.gu2, &G.gp2, &G.gs2, &G.ge2, &G.gm3, &G.gp3, &G.ge3};
    for (int i = 0; i < kGradCount; ++i) {
        *v[i] = reinterpret_cast<__nv_bfloat16*>(p);
        p += align256(static_cast<size_t>(d[kGradSlots[i].level].n) * kGradSlots[i].channels * 2);
    }
    G.partial = reinterpret_cast<float*>(p);
    p += align256(wgrad_partial_floats(d0) * 4);
    G.tmask = reinterpret_cast<float*>(p);
    p += align256(static_cast<size_t>(d0.n) * 4);
    G.sums = reinterpret_cast<double*>(p);
}

cudaError_t net_forward(const NetImages& I, const NetActs& A, const float* r0, const float* r1, const int* parity, const double* norm2, const uint8_t* occ, cudaStream_t s, const uint32_t* skip) {
    const VolumeDims* d = A.d;
    cudaError_t e;
    if (norm2 == nullptr) {
        if ((e = cudaMemsetAsync(A.norm2, 0, sizeof(double), s)) != cudaSuccess) return e;
        sumsq_kernel<<<glue_blocks(d[0].n), kGlueThreads, 0, s>>>(r0, d[0].n, A.norm2);
        norm2 = A.norm2;
    }
    launch_pdl(net_input_kernel, dim3(glue_blocks(d[0].n)), dim3(kGlueThreads), 0, s, d[0], r0, r1, parity, norm2, occ, A.x0, skip);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // encoder
    if ((e = conv_layer(0, d[0], I, A.x0, A.e0, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    launch_pdl(pool_kernel<16>, dim3(glue_blocks_c(d[1].n, 16)), dim3(kGlueThreads), 0, s, d[0], d[1], A.e0, A.p1, skip);
    if ((e = conv_layer(1, d[1], I, A.p1, A.e1, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    launch_pdl(pool_kernel<32>, dim3(glue_blocks_c(d[2].n, 32)), dim3(kGlueThreads), 0, s, d[1], d[2], A.e1, A.p2, skip);
    if ((e = conv_layer(2, d[2], I, A.p2, A.e2, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    launch_pdl(pool_kernel<64>, dim3(glue_blocks_c(d[3].n, 64)), dim3(kGlueThreads), 0, s, d[2], d[3], A.e2, A.p3, skip);
    if ((e = conv_layer(3, d[3], I, A.p3, A.e3, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    // bottom and decoder
    if ((e = conv_layer(4, d[3], I, A.e3, A.m3, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    launch_pdl(up_add_kernel<64>, dim3(glue_blocks_c(d[2].n, 64)), dim3(kGlueThreads), 0, s, d[2], d[3], A.m3, A.e2, A.s2, skip);
    if ((e = conv_layer(5, d[2], I, A.s2, A.u2, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    launch_pdl(up_add_kernel<32>, dim3(glue_blocks_c(d[1].n, 32)), dim3(kGlueThreads), 0, s, d[1], d[2], A.u2, A.e1, A.s1, skip);
    if ((e = conv_layer(6, d[1], I, A.s1, A.u1, nullptr, A.error, s, skip)) != cudaSuccess) return e;
    launch_pdl(up_add_kernel<16>, dim3(glue_blocks_c(d[0].n, 16)), dim3(kGlueThreads), 0, s, d[0], d[1], A.u1, A.e0, A.s0, skip);
    return conv_layer(7, d[0], I, A.s0, nullptr, A.y, A.error, s, skip);
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
    // g: y = conv_g(s0); s0 = up(u1) + e0
    if ((e = layer_wgrad(7, d[0], A.s0, G.gy, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(7, d[0], I, G.gy, nullptr, G.gs0, A.error, s)) != cudaSuccess) return e;
    // f: u1 = relu(conv_f(s1)); s1 = up(u2) + e1
    up_bwd_relu_kernel<16><<<glue_blocks_c(d[1].n, 16), kGlueThreads, 0, s>>>(d[0], d[1], G.gs0, A.u1, G.gu1);
    if ((e = layer_wgrad(6, d[1], A.s1, G.gu1, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(6, d[1], I, G.gu1, nullptr, G.gs1, A.error, s)) != cudaSuccess) return e;
    // e: u2 = relu(conv_e(s2)); s2 = up(m3) + e2
    up_bwd_relu_kernel<32><<<glue_blocks_c(d[2].n, 32), kGlueThreads, 0, s>>>(d[1], d[2], G.gs1, A.u2, G.gu2);
    if ((e = layer_wgrad(5, d[2], A.s2, G.gu2, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(5, d[2], I, G.gu2, nullptr, G.gs2, A.error, s)) != cudaSuccess) return e;
    // m: m3 = relu(conv_m(e3)); e3 = relu(conv_d(p3)) feeds m only, so its ReLU gate goes into m's backward
    up_bwd_relu_kernel<64><<<glue_blocks_c(d[3].n, 64), kGlueThreads, 0, s>>>(d[2], d[3], G.gs2, A.m3, G.gm3);
    if ((e = layer_wgrad(4, d[3], A.e3, G.gm3, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(4, d[3], I, G.gm3, A.e3, G.ge3, A.error, s)) != cudaSuccess) return e;
    // d: e3 = relu(conv_d(p3)); p3 = pool(e2)
    if ((e = layer_wgrad(3, d[3], A.p3, G.ge3, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(3, d[3], I, G.ge3, nullptr, G.gp3, A.error, s)) != cudaSuccess) return e;
    // c: e2 = relu(conv_c(p2)) feeds p3 and s2
    pool_bwd_add_relu_kernel<64><<<glue_blocks_c(d[2].n, 64), kGlueThreads, 0, s>>>(d[2], d[3], G.gs2, G.gp3, A.e2, G.ge2);
    if ((e = layer_wgrad(2, d[2], A.p2, G.ge2, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(2, d[2], I, G.ge2, nullptr, G.gp2, A.error, s)) != cudaSuccess) return e;
    // b: e1 = relu(conv_b(p1)) feeds p2 and s1
    pool_bwd_add_relu_kernel<32><<<glue_blocks_c(d[1].n, 32), kGlueThreads, 0, s>>>(d[1], d[2], G.gs1, G.gp2, A.e1, G.ge1);
    if ((e = layer_wgrad(1, d[1], A.p1, G.ge1, G, grad, accumulate, A.error, s)) != cudaSuccess) return e;
    if ((e = conv_layer_bwd(1, d[1], I, G.ge1, nullptr, G.gp1, A.error, s)) != cudaSuccess) return e;
    // a: e0 = relu(conv_a(x0)) feeds p1 and s0
    pool_bwd_add_relu_kernel<16><<<glue_blocks_c(d[0].n, 16), kGlueThreads, 0, s>>>(d[0], d[1], G.gs0, G.gp1, A.e0, G.ge0);
    return layer_wgrad(0, d[0], A.x0, G.ge0, G, grad, accumulate, A.error, s);
}

cudaError_t net_adam(float* w, const float* grad, float* m, float* v, float lr, int step, float gscale, const NetImages& I, cudaStream_t s) {
    adam_kernel<<<(kNetParams + 255) / 256, 256, 0, s>>>(kNetParams, w, grad, m, v, lr, 0.9f, 0.999f, 1e-8f, step, gscale);
    const cudaError_t e = cudaGetLastError();
    return e != cudaSuccess ? e : net_pack(w, I, s);
}

}  // namespace smoke_b200
