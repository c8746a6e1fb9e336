// Persistent matrix-free conjugate-gradient pressure solver for the B200 smoke library.
//
// Replaces the reference's CSR matrix + cuSPARSE SpMV + 11 cuBLAS/scalar graph nodes per iteration
// (backend-cuda.cu:1343-1412, 1788-1824) by ONE cooperative launch that runs all iterations:
//  - the operator is the masked 7-point stencil encoded per cell in a 16-bit code (neighbour bits + diagonal),
//    identical to the reference's matrix values (see stencil_code_kernel);
//  - the iteration is the Chronopoulos-Gear form of (P)CG: both dot products of an iteration are reduced
//    together, so there is ONE grid barrier per iteration. r, s and w are double-buffered so that a block can
//    recompute its neighbours' new residuals from the old buffers while other blocks write the new ones;
//  - reductions are per-block partials, double-buffered by iteration parity and summed by every block in the
//    same fixed order, so all blocks take identical, deterministic scalar decisions;
//  - FIXED mode reproduces the reference: M = I, x0 = 0, exactly N iterations, alpha and beta set to 0 when the
//    denominator magnitude is <= 1e-20. Tolerance mode stops at ||r|| <= tol ||b|| and can check the true
//    residual b - A x in FP64 and restart from it (iterative refinement);
//  - every grid barrier waits at most kBarrierTimeoutNs, then raises an abort flag that makes all blocks leave;
//    the host reads the outcome from the status block.
#include "launch.h"
#include "smoke_b200_ext.h"

namespace smoke_b200 {

namespace {

constexpr int kPcgThreads = 256;
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s
constexpr unsigned kBarrierMaxSpins = 1u << 26;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier for a cooperative launch. Returns false when the solve was aborted (timeout anywhere).
__device__ bool grid_barrier(PcgControl* ctl) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &ctl->gen;
        volatile int* vabort = &ctl->abort;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->count, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(&ctl->count, 0u);
            __threadfence();
            atomicAdd(&ctl->gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            unsigned spins = 0;
            while (*vgen == gen) {
                if (*vabort) {
                    ok = 0;
                    break;
                }
                ++spins;
                if (spins >= kBarrierMaxSpins || ((spins & 63u) == 0 && global_ns() - t0 > kBarrierTimeoutNs)) {
                    atomicExch(&ctl->abort, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(40);
            }
        }
        __threadfence();
        if (*vabort) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of four values; thread 0 writes them to partial[parity][block].
template <typename T>
__device__ void publish_partials(PcgControl* ctl, int parity, T a, T b, T c, T d) {
    __shared__ T red[4][kPcgThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    d = warp_sum(d);
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
        red[2][warp] = c;
        red[3][warp] = d;
    }
    __syncthreads();
    if (warp == 0) {
        constexpr int nw = kPcgThreads / 32;
        a = lane < nw ? red[0][lane] : T(0);
        b = lane < nw ? red[1][lane] : T(0);
        c = lane < nw ? red[2][lane] : T(0);
        d = lane < nw ? red[3][lane] : T(0);
        a = warp_sum(a);
        b = warp_sum(b);
        c = warp_sum(c);
        d = warp_sum(d);
        if (lane == 0) {
            double* slot = ctl->partial[parity][blockIdx.x];
            slot[0] = static_cast<double>(a);
            slot[1] = static_cast<double>(b);
            slot[2] = static_cast<double>(c);
            slot[3] = static_cast<double>(d);
        }
    }
    __syncthreads();
}

// Sum of all blocks' partials in a fixed order (identical in every block); result broadcast through smem.
template <typename T>
__device__ void gather_partials(const PcgControl* ctl, int parity, T out[4]) {
    __shared__ T tot[4];
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        T a = 0, b = 0, c = 0, d = 0;
        for (unsigned blk = lane; blk < gridDim.x; blk += 32) {
            const double* slot = ctl->partial[parity][blk];
            a += static_cast<T>(__ldcg(slot + 0));
            b += static_cast<T>(__ldcg(slot + 1));
            c += static_cast<T>(__ldcg(slot + 2));
            d += static_cast<T>(__ldcg(slot + 3));
        }
        a = warp_sum(a);
        b = warp_sum(b);
        c = warp_sum(c);
        d = warp_sum(d);
        if (lane == 0) {
            tot[0] = a;
            tot[1] = b;
            tot[2] = c;
            tot[3] = d;
        }
    }
    __syncthreads();
    out[0] = tot[0];
    out[1] = tot[1];
    out[2] = tot[2];
    out[3] = tot[3];
    __syncthreads();
}

// Index of neighbour e (0:-x 1:+x 2:-y 3:+y 4:-z 5:+z) of cell q at (x,y,z), wrapping at the domain edge (only
// called for neighbours marked active, which are in range or across a periodic edge).
__device__ __forceinline__ uint32_t neighbour(const StepParams& P, uint32_t q, int x, int y, int z, int e) {
    const uint32_t nx = P.nx, slab = static_cast<uint32_t>(P.nx) * P.ny;
    switch (e) {
    case 0: return x > 0 ? q - 1 : q + (nx - 1);
    case 1: return x < P.nx - 1 ? q + 1 : q - (nx - 1);
    case 2: return y > 0 ? q - nx : q + (P.ny - 1) * nx;
    case 3: return y < P.ny - 1 ? q + nx : q - (P.ny - 1) * nx;
    case 4: return z > 0 ? q - slab : q + (P.nz - 1) * slab;
    default: return z < P.nz - 1 ? q + slab : q - (P.nz - 1) * slab;
    }
}

template <bool JACOBI>
__device__ __forceinline__ float inv_diag(uint16_t code) {
    if constexpr (JACOBI) return __frcp_rn(static_cast<float>((code >> 8) & 7u));
    else return 1.0f;
}

__device__ __forceinline__ float diag_of(uint16_t code) { return static_cast<float>((code >> 8) & 7u); }

template <typename T>
__device__ __forceinline__ bool finite_all(T a, T b, T c) { return isfinite(a) && isfinite(b) && isfinite(c); }

template <bool JACOBI, typename T>
__global__ void __launch_bounds__(kPcgThreads) pcg_kernel(const __grid_constant__ StepParams P, const PcgSettings S, const uint16_t* __restrict__ codes, const float* __restrict__ b, float* x, PcgWork W, PcgControl* ctl) {
    const uint32_t n = P.n;
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    int parity = 0;
    int cur = 0;
    const T tol2 = static_cast<T>(S.tolerance) * static_cast<T>(S.tolerance);
    const T guard = static_cast<T>(1.0e-20);
    uint32_t status = SMOKE_B200_SOLVE_ITERATION_CAP;
    double true_rel = -1.0;
    int it = 0, passes = 1;
    bool aborted = false;

    // ---------------------------------------------------------------- setup: r0, w0 = A M r0, dots
    T g = 0, d = 0, rr = 0, bbp = 0;
    if (!S.warm_start) {
        for (uint32_t q = first; q < n; q += stride) {
            const uint16_t code = __ldg(codes + q);
            const float inv = inv_diag<JACOBI>(code);
            const float r = __ldg(b + q);
            const float u = r * inv;
            float acc = diag_of(code) * u;
            const uint32_t mask = code & 63u;
            if (mask) {
                int cx, cy, cz;
                cell_xyz(P, q, cx, cy, cz);
#pragma unroll
                for (int e = 0; e < 6; ++e)
                    if (mask & (1u << e)) {
                        const uint32_t nb = neighbour(P, q, cx, cy, cz, e);
                        acc -= __ldg(b + nb) * inv_diag<JACOBI>(__ldg(codes + nb));
                    }
            }
            W.r[0][q] = r;
            W.w[0][q] = acc;
            W.s[0][q] = 0.0f;
            W.p[q] = 0.0f;
            x[q] = 0.0f;
            g += static_cast<T>(r) * static_cast<T>(u);
            d += static_cast<T>(acc) * static_cast<T>(u);
            rr += static_cast<T>(r) * static_cast<T>(r);
        }
        bbp = rr;
    } else {
        // r0 = b - A x0 (x0 complete on entry)
        for (uint32_t q = first; q < n; q += stride) {
            const uint16_t code = __ldg(codes + q);
            float acc = diag_of(code) * __ldcg(x + q);
            const uint32_t mask = code & 63u;
            if (mask) {
                int cx, cy, cz;
                cell_xyz(P, q, cx, cy, cz);
#pragma unroll
                for (int e = 0; e < 6; ++e)
                    if (mask & (1u << e)) acc -= __ldcg(x + neighbour(P, q, cx, cy, cz, e));
            }
            const float bv = __ldg(b + q);
            W.r[0][q] = bv - acc;
            W.s[0][q] = 0.0f;
            W.p[q] = 0.0f;
            bbp += static_cast<T>(bv) * static_cast<T>(bv);
        }
        if (!grid_barrier(ctl)) aborted = true;
        if (!aborted) {
            for (uint32_t q = first; q < n; q += stride) {
                const uint16_t code = __ldg(codes + q);
                const float inv = inv_diag<JACOBI>(code);
                const float r = __ldcg(W.r[0] + q);
                const float u = r * inv;
                float acc = diag_of(code) * u;
                const uint32_t mask = code & 63u;
                if (mask) {
                    int cx, cy, cz;
                    cell_xyz(P, q, cx, cy, cz);
#pragma unroll
                    for (int e = 0; e < 6; ++e)
                        if (mask & (1u << e)) {
                            const uint32_t nb = neighbour(P, q, cx, cy, cz, e);
                            acc -= __ldcg(W.r[0] + nb) * inv_diag<JACOBI>(__ldg(codes + nb));
                        }
                }
                W.w[0][q] = acc;
                g += static_cast<T>(r) * static_cast<T>(u);
                d += static_cast<T>(acc) * static_cast<T>(u);
                rr += static_cast<T>(r) * static_cast<T>(r);
            }
        }
    }
    T tot[4] = {0, 0, 0, 0};
    if (!aborted) {
        publish_partials<T>(ctl, parity, g, d, rr, bbp);
        if (!grid_barrier(ctl)) aborted = true;
        else gather_partials<T>(ctl, parity, tot);
        parity ^= 1;
    }
    T gamma = tot[0], delta = tot[1], rnorm2 = tot[2];
    const T bb = tot[3];

    if (aborted) {
        status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
    } else if (!(bb > T(0))) {
        // b = 0: the solution is 0 (for a warm start, overwrite the initial guess)
        if (S.warm_start)
            for (uint32_t q = first; q < n; q += stride) x[q] = 0.0f;
        rnorm2 = 0;
        status = S.fixed ? SMOKE_B200_SOLVE_ITERATION_CAP : SMOKE_B200_SOLVE_CONVERGED;
        if (S.fixed) it = S.max_iterations;
        if (!isfinite(bb)) status = SMOKE_B200_SOLVE_NOT_FINITE;
    } else {
        for (;;) {  // refinement passes
            T alpha = (gamma == T(0) && delta == T(0)) ? T(0) : (S.fixed ? (fabs(delta) > guard ? gamma / delta : T(0)) : gamma / delta);
            T beta = 0;
            bool stop = false;
            if (!finite_all(gamma, delta, rnorm2)) {
                status = SMOKE_B200_SOLVE_NOT_FINITE;
                stop = true;
            } else if (S.fixed ? it >= S.max_iterations : rnorm2 <= tol2 * bb) {
                status = S.fixed ? SMOKE_B200_SOLVE_ITERATION_CAP : SMOKE_B200_SOLVE_CONVERGED;
                stop = true;
            } else if (!S.fixed && !(delta > T(0))) {
                status = SMOKE_B200_SOLVE_BREAKDOWN;
                stop = true;
            }
            while (!stop) {
                const float fa = static_cast<float>(alpha), fb = static_cast<float>(beta);
                const float* Rc = W.r[cur];
                const float* Sc = W.s[cur];
                const float* Wc = W.w[cur];
                float* Rn = W.r[cur ^ 1];
                float* Sn = W.s[cur ^ 1];
                float* Wn = W.w[cur ^ 1];
                T g1 = 0, d1 = 0, r1 = 0;
                for (uint32_t q = first; q < n; q += stride) {
                    const uint16_t code = __ldg(codes + q);
                    const float inv = inv_diag<JACOBI>(code);
                    const float r = __ldcg(Rc + q), s = __ldcg(Sc + q), w = __ldcg(Wc + q);
                    float pv = __ldcg(W.p + q);
                    pv = r * inv + fb * pv;          // p_i = u_i + beta_i p_{i-1}
                    const float sn = w + fb * s;     // s_i = w_i + beta_i s_{i-1}
                    const float xv = __ldcg(x + q) + fa * pv;
                    const float rn = r - fa * sn;    // r_{i+1}
                    const float un = rn * inv;       // u_{i+1} = M r_{i+1}
                    float acc = diag_of(code) * un;  // w_{i+1} = A u_{i+1}
                    const uint32_t mask = code & 63u;
                    if (mask) {
                        int cx, cy, cz;
                        cell_xyz(P, q, cx, cy, cz);
#pragma unroll
                        for (int e = 0; e < 6; ++e)
                            if (mask & (1u << e)) {
                                const uint32_t nb = neighbour(P, q, cx, cy, cz, e);
                                const float snb = __ldcg(Wc + nb) + fb * __ldcg(Sc + nb);
                                const float rnb = __ldcg(Rc + nb) - fa * snb;
                                acc -= rnb * inv_diag<JACOBI>(__ldg(codes + nb));
                            }
                    }
                    W.p[q] = pv;
                    x[q] = xv;
                    Rn[q] = rn;
                    Sn[q] = sn;
                    Wn[q] = acc;
                    g1 += static_cast<T>(rn) * static_cast<T>(un);
                    d1 += static_cast<T>(acc) * static_cast<T>(un);
                    r1 += static_cast<T>(rn) * static_cast<T>(rn);
                }
                publish_partials<T>(ctl, parity, g1, d1, r1, T(0));
                if (!grid_barrier(ctl)) {
                    aborted = true;
                    status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
                    break;
                }
                gather_partials<T>(ctl, parity, tot);
                parity ^= 1;
                cur ^= 1;
                ++it;
                const T gn = tot[0], dn = tot[1];
                rnorm2 = tot[2];
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
                    if (rnorm2 <= tol2 * bb) {
                        status = SMOKE_B200_SOLVE_CONVERGED;
                        break;
                    }
                    if (it >= S.max_iterations * passes) {
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
            if (aborted || S.fixed || S.refinement <= 0 || status != SMOKE_B200_SOLVE_CONVERGED) break;

            // FP64 true residual r = b - A x (x complete: the last barrier followed its writes)
            double tr = 0.0;
            float* Rc = W.r[cur];
            for (uint32_t q = first; q < n; q += stride) {
                const uint16_t code = __ldg(codes + q);
                double acc = static_cast<double>(diag_of(code)) * static_cast<double>(__ldcg(x + q));
                const uint32_t mask = code & 63u;
                if (mask) {
                    int cx, cy, cz;
                    cell_xyz(P, q, cx, cy, cz);
#pragma unroll
                    for (int e = 0; e < 6; ++e)
                        if (mask & (1u << e)) acc -= static_cast<double>(__ldcg(x + neighbour(P, q, cx, cy, cz, e)));
                }
                const double rv = static_cast<double>(__ldg(b + q)) - acc;
                Rc[q] = static_cast<float>(rv);
                tr += rv * rv;
            }
            publish_partials<double>(ctl, parity, tr, 0.0, 0.0, 0.0);
            if (!grid_barrier(ctl)) {
                aborted = true;
                status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
                break;
            }
            double tt[4];
            gather_partials<double>(ctl, parity, tt);
            parity ^= 1;
            true_rel = sqrt(tt[0] / static_cast<double>(bb));
            if (true_rel <= static_cast<double>(S.tolerance) || passes > S.refinement) {
                if (true_rel > static_cast<double>(S.tolerance)) status = SMOKE_B200_SOLVE_ITERATION_CAP;
                break;
            }
            // restart from the true residual: s = p = 0, w = A M r
            ++passes;
            g = d = rr = 0;
            for (uint32_t q = first; q < n; q += stride) {
                const uint16_t code = __ldg(codes + q);
                const float inv = inv_diag<JACOBI>(code);
                const float r = __ldcg(Rc + q);
                const float u = r * inv;
                float acc = diag_of(code) * u;
                const uint32_t mask = code & 63u;
                if (mask) {
                    int cx, cy, cz;
                    cell_xyz(P, q, cx, cy, cz);
#pragma unroll
                    for (int e = 0; e < 6; ++e)
                        if (mask & (1u << e)) {
                            const uint32_t nb = neighbour(P, q, cx, cy, cz, e);
                            acc -= __ldcg(Rc + nb) * inv_diag<JACOBI>(__ldg(codes + nb));
                        }
                }
                W.w[cur][q] = acc;
                W.s[cur][q] = 0.0f;
                W.p[q] = 0.0f;
                g += static_cast<T>(r) * static_cast<T>(u);
                d += static_cast<T>(acc) * static_cast<T>(u);
                rr += static_cast<T>(r) * static_cast<T>(r);
            }
            publish_partials<T>(ctl, parity, g, d, rr, T(0));
            if (!grid_barrier(ctl)) {
                aborted = true;
                status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
                break;
            }
            gather_partials<T>(ctl, parity, tot);
            parity ^= 1;
            gamma = tot[0];
            delta = tot[1];
            rnorm2 = tot[2];
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
        ctl->status = st;
    }
}

template <bool J, typename T>
cudaError_t launch_one(const StepParams& P, const PcgSettings& S, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s) {
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<J, T>, kPcgThreads, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorLaunchOutOfResources;
        max_blocks = sms * per_sm;
        if (max_blocks > kPcgMaxBlocks) max_blocks = kPcgMaxBlocks;
    }
    const uint64_t want = (static_cast<uint64_t>(P.n) + kPcgThreads - 1) / kPcgThreads;
    const int blocks = static_cast<int>(want < static_cast<uint64_t>(max_blocks) ? (want > 0 ? want : 1) : max_blocks);
    cudaError_t e = cudaMemsetAsync(ctl, 0, 4 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kPcgThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pcg_kernel<J, T>, P, S, codes, b, x, work, ctl);
}

}  // namespace

cudaError_t pcg_launch_shape(PcgLaunchShape* out) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<true, double>, kPcgThreads, 0);
    if (e != cudaSuccess) return e;
    out->blocks = sms * per_sm;
    out->threads = kPcgThreads;
    return cudaSuccess;
}

cudaError_t launch_pcg(const StepParams& P, const PcgSettings& S, const PcgLaunchShape&, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s) {
    if (S.jacobi) return S.fp64 ? launch_one<true, double>(P, S, codes, b, x, work, ctl, s) : launch_one<true, float>(P, S, codes, b, x, work, ctl, s);
    return S.fp64 ? launch_one<false, double>(P, S, codes, b, x, work, ctl, s) : launch_one<false, float>(P, S, codes, b, x, work, ctl, s);
}

}  // namespace smoke_b200
