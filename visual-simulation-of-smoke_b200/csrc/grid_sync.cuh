// Grid-wide synchronisation for the persistent cooperative solver kernels (pcg.cu): a bounded-wait grid
// barrier fused with an all-reduce of four sums, and block-level helpers. THREADS is the kernel's block size.
#pragma once

#include "launch.h"

namespace smoke_b200 {
namespace gsync {

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s: the default bound of a barrier wait
constexpr unsigned kBarrierMaxSpins = 1u << 26;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of 4 values in a fixed order; the result is valid in thread 0.
template <int THREADS, typename T>
__device__ void block_sum4(T v[4], T (*scratch)[THREADS / 32]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) scratch[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = warp_sum(lane < THREADS / 32 ? scratch[k][lane] : T(0));
    }
    __syncthreads();
}

// Grid barrier number `phase` fused with an all-reduce of 4 sums.
//  - arrival: one atomic add per block on `bar`; block 0 adds 2^31 - (blocks - 1), every other block adds 1, so the
//    top bit of `bar` flips exactly when the last block arrives, whatever the order (the counter is never reset);
//  - sums: block b adds its partials (FP64 atomics) into copy b % kPcgSumCopies of ring slot phase % 3; after the
//    barrier every block adds the copies in copy order. Once past barrier k, block 0 clears slot (k + 2) % 3, which
//    no block reads again and none writes before barrier k + 2.
// Every wait is bounded (timeout_ns of globaltimer, or kBarrierMaxSpins polls); returns false if the solve was
// aborted.
template <int THREADS, typename T>
__device__ bool barrier_allreduce(PcgControl* ctl, unsigned& phase, T local[4], T out[4], bool reduce = true, unsigned long long timeout_ns = kBarrierTimeoutNs) {
    __shared__ T scratch[4][THREADS / 32];
    __shared__ int s_ok;
    if (reduce) block_sum4<THREADS>(local, scratch);  // its __syncthreads orders the block's earlier writes
    else __syncthreads();
    const int slot = static_cast<int>(phase % 3u);
    if (threadIdx.x == 0) {
        if (reduce) {
            double* tot = ctl->totals[slot][blockIdx.x % kPcgSumCopies];
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicAdd(tot + k, static_cast<double>(local[k]));
        }
        const unsigned add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1u) : 1u;
        __threadfence();
        const unsigned before = atomicAdd(&ctl->bar, add);
        volatile unsigned* vbar = &ctl->bar;
        volatile int* vabort = &ctl->abort;
        int ok = 1;
        const unsigned long long t0 = global_ns();
        unsigned spins = 0;
        while (((before ^ *vbar) & 0x80000000u) == 0u) {
            if (*vabort) {
                ok = 0;
                break;
            }
            ++spins;
            if (spins >= kBarrierMaxSpins || ((spins & 63u) == 0 && global_ns() - t0 > timeout_ns)) {
                atomicExch(&ctl->abort, 1);
                ok = 0;
                break;
            }
        }
        __threadfence();
        if (*vabort) ok = 0;
        s_ok = ok;
        if (blockIdx.x == 0) {  // every barrier, reducing or not, frees the slot two ahead
            double* z = &ctl->totals[(phase + 2u) % 3u][0][0];
            for (int k = 0; k < kPcgSumCopies * 16; ++k) z[k] = 0.0;
        }
    }
    __syncthreads();
    if (reduce) {
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = T(0);
#pragma unroll
        for (int c = 0; c < kPcgSumCopies; ++c) {
            const double* tot = ctl->totals[slot][c];
#pragma unroll
            for (int k = 0; k < 4; ++k) out[k] += static_cast<T>(__ldcg(tot + k));
        }
    }
    const bool ok = s_ok != 0;
    __syncthreads();
    ++phase;
    return ok;
}

}  // namespace gsync
}  // namespace smoke_b200
