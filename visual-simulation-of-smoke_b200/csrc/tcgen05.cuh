// Blackwell (sm_100a) tensor-core primitives in inline PTX: tensor-memory allocation, shared-memory matrix
// descriptors, the BF16 MMA with FP32 accumulation in tensor memory, its completion barrier and the accumulator
// loads. Used by the convolution kernels of the learned preconditioner (unet.cu).
//
// Operand layout: no swizzle; a matrix in shared memory is a grid of "core matrices" of 8 rows x 16 bytes
// (8 BF16 values per row), each stored as 128 contiguous bytes. A descriptor gives the start address and two
// strides in bytes: LBO between core matrices adjacent along K (K-major operands) or along K-row groups
// (MN-major operands), SBO between core matrices adjacent along M/N. Encoding (sm100 descriptor): bits 0-13
// start >> 4, 16-29 LBO >> 4, 32-45 SBO >> 4, 46-47 version = 1, 49-51 base offset 0, 52 LBO mode 0, 61-63
// layout 0 (no swizzle).
#pragma once

#include <cstdint>

namespace smoke_b200 {
namespace tc {

// Instruction descriptor of tcgen05.mma kind::f16 with BF16 A and B and an FP32 accumulator: bits 4-5 D format
// (1 = F32), 7-9 A format (1 = BF16), 10-12 B format (1 = BF16), 15/16 A/B major (0 = K, 1 = MN), 17-22 N >> 3,
// 24-28 M >> 4.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n, bool a_mn_major, bool b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

#if defined(__CUDACC__)

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) | (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// D (tensor memory) (+)= A (shared) x B (shared); issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// The mbarrier at `bar` receives one arrival when every MMA issued so far by this thread has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy writes to shared memory become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits until the phase of parity `parity` of the mbarrier completed, for at most `max_cycles` clock cycles.
// Returns false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long max_cycles) {
    const uint32_t a = smem_addr(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > max_cycles) return false;
    }
}

// The same wait that also gives up as soon as the block-wide flag *abort (shared memory) is nonzero.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, long long max_cycles, const volatile int* abort) {
    const uint32_t a = smem_addr(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (*abort) return false;
        if (clock64() - t0 > max_cycles) return false;
    }
}

// One plain arrival on the mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Tensor-memory allocation of `cols` columns (a power of two >= 32) by one whole warp; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t addr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(addr), "r"(cols) : "memory");
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane (warp w of the block reads lanes 32w..32w+31):
// the warp-wide load, then the wait for it.
__device__ __forceinline__ void tmem_load16(uint32_t addr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// One arrival on the mbarrier that also expects `bytes` of asynchronous (TMA) transfer before its phase completes.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// TMA: the box of the 4-D tensor map at coordinates (c0, c1, c2, c3) into shared memory at `dst`, completing
// `bytes` on the mbarrier. Out-of-range elements (negative coordinates included) read as zero. No multicast.
__device__ __forceinline__ void tma_load_4d(void* dst, const void* map, int c0, int c1, int c2, int c3, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// Bulk (non-tensor) asynchronous copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global to
// shared memory, completing on the mbarrier (which must expect the bytes). No multicast.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes),
                 "r"(smem_addr(bar))
                 : "memory");
}

#endif  // __CUDACC__

}  // namespace tc
}  // namespace smoke_b200
