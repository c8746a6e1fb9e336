// Persistent matrix-free conjugate-gradient pressure solver for the B200 smoke library.
//
// Replaces the reference's CSR matrix + cuSPARSE SpMV + 11 cuBLAS/scalar graph nodes per iteration
// (backend-cuda.cu:1343-1412, 1788-1824) by ONE cooperative launch that runs every iteration:
//  - the operator is the masked 7-point stencil encoded per cell in a 16-bit code (neighbour bits + diagonal),
//    with the reference's matrix values (stencil_code_kernel in step_kernels.cu);
//  - work is split into 32x8-cell columns marched in z ("2.5D" stencil): every thread owns one (x, y) cell of a
//    column, so a plane step costs one address add; the +-z neighbours stay in registers and only the thin in-plane
//    halo goes through a three-plane ring in shared memory. Loads of plane z+2 are issued before plane z is
//    computed. Each block owns a fixed, balanced range of column-planes;
//  - the iteration is the Chronopoulos-Gear form of (P)CG: both dot products of an iteration are reduced together,
//    so there is ONE grid barrier per iteration. r, s and w are double-buffered: a block recomputes its halo's new
//    residuals from the old buffers while other blocks write the new ones;
//  - the barrier (grid_sync.cuh) is one atomic per block on a flip-bit counter; its all-reduce adds FP64 partials
//    atomically into copies spread over cache lines, so every block reads the same totals and takes the same scalar
//    decisions (the summation order of the block partials is not fixed);
//  - FIXED mode reproduces the reference: M = I, x0 = 0, exactly N iterations, alpha/beta = 0 when the denominator
//    magnitude is <= 1e-20. Tolerance mode stops at ||r|| <= tol ||b||. With refinement, the solution is accumulated
//    in FP64 (x64 += e after each FP32 inner solve of A e = r) and r = b - A x64 is recomputed in FP64, so the
//    residual can go below the FP32 floor of the pressure itself;
//  - every grid barrier waits at most kBarrierTimeoutNs, then raises an abort flag that makes all blocks leave; the
//    host reads the outcome from the status block.
#include <map>
#include <mutex>

#include "grid_sync.cuh"
#include "march.cuh"
#include "launch.h"
#include "smoke_b200_ext.h"

namespace smoke_b200 {

namespace {

using zmarch::kThreads;
using zmarch::CX;
using zmarch::CY;
using zmarch::PX;
using zmarch::kPlane;
using zmarch::Columns;
using zmarch::MarchGeom;
using zmarch::march;
using gsync::global_ns;
using gsync::warp_sum;

template <typename T>
__device__ __forceinline__ bool barrier_allreduce(const PcgSettings& S, PcgControl* ctl, unsigned& phase, T local[4], T out[4], bool reduce = true) {
    const unsigned long long timeout_ns = S.barrier_timeout_ms ? static_cast<unsigned long long>(S.barrier_timeout_ms) * 1000000ull : gsync::kBarrierTimeoutNs;
    return gsync::barrier_allreduce<kThreads, T>(ctl, phase, local, out, reduce, timeout_ns);
}

template <bool JACOBI>
__device__ __forceinline__ float inv_diag(uint16_t code) {
    if constexpr (JACOBI) return code ? __frcp_rn(static_cast<float>((code >> 8) & 7u)) : 0.0f;
    else return 1.0f;
}
__device__ __forceinline__ float diag_of(uint16_t code) { return static_cast<float>((code >> 8) & 7u); }

// diag * u0 - active neighbours; in-plane ones from the ring plane, -z/+z from registers.
template <typename V>
__device__ __forceinline__ V stencil(uint16_t code, V u0, V um1, V u1, const V* plane, int slot) {
    V acc = static_cast<V>(diag_of(code)) * u0;
    if (code & 1u) acc -= plane[slot - 1];
    if (code & 2u) acc -= plane[slot + 1];
    if (code & 4u) acc -= plane[slot - PX];
    if (code & 8u) acc -= plane[slot + PX];
    if (code & 16u) acc -= um1;
    if (code & 32u) acc -= u1;
    return acc;
}

struct IterData {
    float r, s, w, p, e;
    uint16_t code;
};
struct SrcData {
    float v;
    uint16_t code;
};
struct X64Data {
    double v;
    uint16_t code;
};

template <typename T>
__device__ __forceinline__ bool finite_all(T a, T b, T c) { return isfinite(a) && isfinite(b) && isfinite(c); }

// MINB: blocks per SM the register allocation must allow (1: unconstrained, about 125 registers and 2 blocks per SM;
// 4: at most 64 registers, a few spills, twice the loads in flight; the autotuner picks per grid).
template <bool JACOBI, typename T, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) pcg_kernel(const __grid_constant__ StepParams P, const PcgSettings S, const Columns C, const uint16_t* __restrict__ codes, const float* __restrict__ b, float* x, PcgWork W, PcgControl* ctl) {
    __shared__ __align__(16) double ring_raw[3][kPlane];
    // test hook: this block never arrives at a barrier, so the others' bounded waits run out and abort the solve
    if (S.withhold_block > 0 && static_cast<int>(blockIdx.x) == S.withhold_block - 1) return;
    const MarchGeom G = zmarch::geom_of(P.nx, P.ny, P.nz, P.fper);
    float(*ring_f)[kPlane] = reinterpret_cast<float(*)[kPlane]>(ring_raw);
    double(*ring_d)[kPlane] = ring_raw;
    const bool ir = !S.fixed && S.refinement > 0;  // FP64 accumulation + true-residual passes
    float* e = ir ? W.e : x;                         // the FP32 iterate
    const T guard = static_cast<T>(1.0e-20);
    unsigned phase = 0;
    int cur = 0;
    uint32_t status = SMOKE_B200_SOLVE_ITERATION_CAP;
    double true_rel = -1.0;
    int it = 0, passes = 1;
    bool aborted = false;

    auto sync_sums = [&](T local[4], T out[4]) -> bool {
        const bool ok = barrier_allreduce<T>(S, ctl, phase, local, out);
        if (!ok) aborted = true;
        return ok;
    };

    // ------------------------------------------------------------ pass start: R[cur] = src, W[cur] = A M src
    auto start_pass = [&](const float* src, bool zero_e, T sums[4]) -> bool {
        T loc[4] = {0, 0, 0, 0};
        float* Rc = W.r[cur];
        float* Wc = W.w[cur];
        float* Sc = W.s[cur];
        march<float, SrcData>(
            G, C, ring_f,
            [&](bool ok, uint32_t q, bool, int, int, int) {
                SrcData d{0.0f, 0};
                if (ok) {
                    d.v = __ldcg(src + q);
                    d.code = __ldg(codes + q);
                }
                return d;
            },
            [&](const SrcData& d) { return d.v * inv_diag<JACOBI>(d.code); },
            [&](uint32_t q, const SrcData& d, float um1, float u0, float u1, const float* plane, int slot, int, int, int) {
                const float w = stencil(d.code, u0, um1, u1, plane, slot);
                Rc[q] = d.v;
                Wc[q] = w;
                Sc[q] = 0.0f;
                W.p[q] = 0.0f;
                if (zero_e) e[q] = 0.0f;
                const float bv = __ldg(b + q);
                loc[0] += static_cast<T>(d.v) * static_cast<T>(u0);
                loc[1] += static_cast<T>(w) * static_cast<T>(u0);
                loc[2] += static_cast<T>(d.v) * static_cast<T>(d.v);
                loc[3] += static_cast<T>(bv) * static_cast<T>(bv);
            });
        return sync_sums(loc, sums);
    };

    // ------------------------------------------------------------ one C-G iteration: buffers cur -> cur^1
    auto iterate = [&](float fa, float fb, T sums[4]) -> bool {
        const float* Rc = W.r[cur];
        const float* Sc = W.s[cur];
        const float* Wc = W.w[cur];
        float* Rn = W.r[cur ^ 1];
        float* Sn = W.s[cur ^ 1];
        float* Wn = W.w[cur ^ 1];
        T loc[4] = {0, 0, 0, 0};
        march<float, IterData>(
            G, C, ring_f,
            [&](bool ok, uint32_t q, bool own, int, int, int) {
                IterData d{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0};
                if (ok) {
                    d.r = __ldcg(Rc + q);
                    d.s = __ldcg(Sc + q);
                    d.w = __ldcg(Wc + q);
                    d.code = __ldg(codes + q);
                    if (own) {
                        d.p = __ldcg(W.p + q);
                        d.e = __ldcg(e + q);
                    }
                }
                return d;
            },
            [&](const IterData& d) {
                const float sn = d.w + fb * d.s;  // s_i
                const float rn = d.r - fa * sn;   // r_{i+1}
                return rn * inv_diag<JACOBI>(d.code);  // u_{i+1} = M r_{i+1}
            },
            [&](uint32_t q, const IterData& d, float um1, float u0, float u1, const float* plane, int slot, int, int, int) {
                const float pv = d.r * inv_diag<JACOBI>(d.code) + fb * d.p;  // p_i = u_i + beta p_{i-1}
                const float sn = d.w + fb * d.s;
                const float rn = d.r - fa * sn;
                const float wn = stencil(d.code, u0, um1, u1, plane, slot);  // w_{i+1} = A u_{i+1}
                W.p[q] = pv;
                e[q] = d.e + fa * pv;
                Rn[q] = rn;
                Sn[q] = sn;
                Wn[q] = wn;
                loc[0] += static_cast<T>(rn) * static_cast<T>(u0);
                loc[1] += static_cast<T>(wn) * static_cast<T>(u0);
                loc[2] += static_cast<T>(rn) * static_cast<T>(rn);
            });
        const bool ok = sync_sums(loc, sums);
        cur ^= 1;
        return ok;
    };

    // ------------------------------------------------------------ FP64 accumulation and true residual
    const uint32_t gtid = blockIdx.x * kThreads + threadIdx.x, gstride = gridDim.x * kThreads;
    auto accumulate = [&]() {  // x64 (+)= e
        const bool fresh = passes == 1 && !S.warm_start;
        for (uint32_t q = gtid; q < P.n; q += gstride) W.x64[q] = (fresh ? 0.0 : W.x64[q]) + static_cast<double>(__ldcg(e + q));
    };
    auto true_residual = [&](double sums[4]) -> bool {  // R[cur] = b - A x64 (FP64)
        double loc[4] = {0, 0, 0, 0};
        float* Rc = W.r[cur];
        march<double, X64Data>(
            G, C, ring_d,
            [&](bool ok, uint32_t q, bool, int, int, int) {
                X64Data d{0.0, 0};
                if (ok) {
                    d.v = __ldcg(W.x64 + q);
                    d.code = __ldg(codes + q);
                }
                return d;
            },
            [&](const X64Data& d) { return d.v; },
            [&](uint32_t q, const X64Data& d, double um1, double u0, double u1, const double* plane, int slot, int, int, int) {
                const double rv = static_cast<double>(__ldg(b + q)) - stencil(d.code, u0, um1, u1, plane, slot);
                Rc[q] = static_cast<float>(rv);
                loc[0] += rv * rv;
            });
        const bool ok = barrier_allreduce<double>(S, ctl, phase, loc, sums);
        if (!ok) aborted = true;
        return ok;
    };

    // ------------------------------------------------------------ setup
    T sums[4] = {0, 0, 0, 0};
    if (S.warm_start && ir) {
        // x64 holds the previous solution: e = 0, r0 = b - A x64
        for (uint32_t q = gtid; q < P.n; q += gstride) e[q] = 0.0f;
        double ds[4];
        if (true_residual(ds)) start_pass(W.r[cur], false, sums);
    } else {
        start_pass(b, true, sums);
    }
    T gamma = sums[0], delta = sums[1], rnorm2 = sums[2];
    const T bb = sums[3];
    T pass_rr0 = rnorm2;

    if (aborted) {
        status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
    } else if (!(bb > T(0))) {
        // b = 0: the solution is 0
        for (uint32_t q = gtid; q < P.n; q += gstride) {
            x[q] = 0.0f;
            if (ir) W.x64[q] = 0.0;
        }
        rnorm2 = 0;
        status = S.fixed ? SMOKE_B200_SOLVE_ITERATION_CAP : SMOKE_B200_SOLVE_CONVERGED;
        if (S.fixed) it = S.max_iterations;
        if (!isfinite(bb)) status = SMOKE_B200_SOLVE_NOT_FINITE;
        if (ir) true_rel = 0.0;
    } else {
        const T tol2 = static_cast<T>(S.tolerance) * static_cast<T>(S.tolerance) * bb;
        for (;;) {  // refinement passes
            // inner target: the total target, or (with refinement) a reduction the FP32 iterate can reach
            T target2 = tol2;
            if (ir) {
                const T floor2 = T(9e-8) * pass_rr0;  // 3e-4 relative to the pass's starting residual
                const T want2 = T(0.09) * tol2;       // 0.3 x the total target
                target2 = want2 > floor2 ? want2 : floor2;
            }
            T alpha = (gamma == T(0) && delta == T(0)) ? T(0) : (S.fixed ? (fabs(delta) > guard ? gamma / delta : T(0)) : gamma / delta);
            T beta = 0;
            bool stop = false;
            if (!finite_all(gamma, delta, rnorm2)) {
                status = SMOKE_B200_SOLVE_NOT_FINITE;
                stop = true;
            } else if (S.fixed ? it >= S.max_iterations : rnorm2 <= target2) {
                status = S.fixed ? SMOKE_B200_SOLVE_ITERATION_CAP : SMOKE_B200_SOLVE_CONVERGED;
                stop = true;
            } else if (!S.fixed && !(delta > T(0))) {
                status = SMOKE_B200_SOLVE_BREAKDOWN;
                stop = true;
            }
            while (!stop) {
                if (!iterate(static_cast<float>(alpha), static_cast<float>(beta), sums)) {
                    status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
                    break;
                }
                ++it;
                const T gn = sums[0], dn = sums[1];
                rnorm2 = sums[2];
                if (!finite_all(gn, dn, rnorm2)) {
                    status = SMOKE_B200_SOLVE_NOT_FINITE;
                    break;
                }
                if (S.fixed) {
                    if (it >= S.max_iterations) {
                        status = SMOKE_B200_SOLVE_ITERATION_CAP;
                        break;
                    }
                } else {
                    if (rnorm2 <= target2) {
                        status = SMOKE_B200_SOLVE_CONVERGED;
                        break;
                    }
                    if (it >= S.max_iterations) {
                        status = SMOKE_B200_SOLVE_ITERATION_CAP;
                        break;
                    }
                }
                if (S.fixed) {
                    beta = fabs(gamma) > guard ? gn / gamma : T(0);
                    const T den = alpha != T(0) ? dn - beta * gn / alpha : dn;
                    alpha = fabs(den) > guard ? gn / den : T(0);
                } else {
                    beta = gn / gamma;
                    const T den = dn - beta * gn / alpha;
                    if (!(den > T(0)) || !(gamma > T(0))) {
                        status = SMOKE_B200_SOLVE_BREAKDOWN;
                        break;
                    }
                    alpha = gn / den;
                }
                gamma = gn;
            }
            if (aborted || !ir) break;
            // FP64: x64 += e, then r = b - A x64
            accumulate();
            T none[4] = {0, 0, 0, 0}, dummy[4];
            if (!barrier_allreduce<T>(S, ctl, phase, none, dummy, false)) {
                aborted = true;
                break;
            }
            double ds[4];
            if (!true_residual(ds)) break;
            true_rel = sqrt(ds[0] / static_cast<double>(bb));
            if (true_rel <= static_cast<double>(S.tolerance)) {
                status = SMOKE_B200_SOLVE_CONVERGED;
                break;
            }
            if (passes > S.refinement || it >= S.max_iterations || status != SMOKE_B200_SOLVE_CONVERGED) {
                if (status == SMOKE_B200_SOLVE_CONVERGED) status = SMOKE_B200_SOLVE_ITERATION_CAP;
                break;
            }
            ++passes;
            if (!start_pass(W.r[cur], true, sums)) break;
            gamma = sums[0];
            delta = sums[1];
            rnorm2 = sums[2];
            pass_rr0 = rnorm2;
        }
        if (aborted) status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
        if (ir && !aborted) {
            // the FP32 pressure is the rounded FP64 solution (x64 is complete: the last barrier followed its writes)
            for (uint32_t q = gtid; q < P.n; q += gstride) x[q] = static_cast<float>(W.x64[q]);
        }
    }

    if (blockIdx.x == 0 && threadIdx.x == 0) {
        PcgStatusDevice st{};
        st.iterations = it;
        st.passes = passes;
        st.status = aborted ? static_cast<uint32_t>(SMOKE_B200_SOLVE_BARRIER_TIMEOUT) : status;
        st.rhs_norm = sqrt(static_cast<double>(bb));
        st.relative_residual = bb > T(0) ? sqrt(static_cast<double>(rnorm2) / static_cast<double>(bb)) : 0.0;
        st.true_relative_residual = true_rel;
        st.flags = 0;
        ctl->status = st;
    }
}

template <bool J, typename T, int MINB>
cudaError_t launch_one(const StepParams& P, const PcgSettings& S, int grid, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s) {
    // co-resident blocks of this kernel instance, per device (devices may differ in SM count)
    static std::mutex cache_mutex;
    static std::map<int, int> cache;
    int dev = 0;
    cudaError_t ed = cudaGetDevice(&dev);
    if (ed != cudaSuccess) return ed;
    int max_blocks = 0;
    {
        std::lock_guard<std::mutex> lock(cache_mutex);
        auto it = cache.find(dev);
        if (it != cache.end()) max_blocks = it->second;
    }
    if (max_blocks == 0) {
        int sms = 0, per_sm = 0;
        cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<J, T, MINB>, kThreads, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorLaunchOutOfResources;
        max_blocks = sms * per_sm;
        if (max_blocks > kPcgMaxBlocks) max_blocks = kPcgMaxBlocks;
        std::lock_guard<std::mutex> lock(cache_mutex);
        cache[dev] = max_blocks;
    }
    Columns C{};
    C.ncx = (P.nx + CX - 1) / CX;
    C.ncy = (P.ny + CY - 1) / CY;
    C.total = static_cast<uint32_t>(C.ncx) * C.ncy * P.nz;
    // at least ~8 planes per block, so the two-plane prologue of a segment stays a small share of its work
    uint32_t want = C.total / 8u;
    if (want < 1u) want = 1u;
    const int shift = grid < 0 ? 0 : (grid >= kPcgGridCount ? kPcgGridCount - 1 : grid);
    const uint32_t cap = static_cast<uint32_t>(max_blocks >> shift) > 0u ? static_cast<uint32_t>(max_blocks >> shift) : 1u;
    const int blocks = static_cast<int>(want < cap ? want : cap);
    cudaError_t e = cudaMemsetAsync(ctl, 0, kPcgControlResetBytes, s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pcg_kernel<J, T, MINB>, P, S, C, codes, b, x, work, ctl);
}

}  // namespace

cudaError_t pcg_launch_shape(PcgLaunchShape* out) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    out->blocks = sms;
    out->threads = kThreads;
    out->grid = 0;
    out->regs = 0;
    return cudaSuccess;
}

template <int MINB>
cudaError_t launch_variant(const StepParams& P, const PcgSettings& S, int g, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s) {
    if (S.jacobi) return S.fp64 ? launch_one<true, double, MINB>(P, S, g, codes, b, x, work, ctl, s) : launch_one<true, float, MINB>(P, S, g, codes, b, x, work, ctl, s);
    return S.fp64 ? launch_one<false, double, MINB>(P, S, g, codes, b, x, work, ctl, s) : launch_one<false, float, MINB>(P, S, g, codes, b, x, work, ctl, s);
}

cudaError_t launch_pcg(const StepParams& P, const PcgSettings& S, const PcgLaunchShape& shape, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s) {
    return shape.regs ? launch_variant<4>(P, S, shape.grid, codes, b, x, work, ctl, s) : launch_variant<1>(P, S, shape.grid, codes, b, x, work, ctl, s);
}

}  // namespace smoke_b200
