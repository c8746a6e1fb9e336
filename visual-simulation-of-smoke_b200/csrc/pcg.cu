// Persistent matrix-free conjugate-gradient pressure solver for the B200 smoke library.
//
// Replaces the reference's CSR matrix + cuSPARSE SpMV + 11 cuBLAS/scalar graph nodes per iteration
// (backend-cuda.cu:1343-1412, 1788-1824) by ONE cooperative launch that runs every iteration:
//  - the operator is the masked 7-point stencil encoded per cell in a 16-bit code (neighbour bits + diagonal),
//    with the reference's matrix values (stencil_code_kernel in step_kernels.cu);
//  - each block owns fixed 32x8x8 bricks of cells; per iteration it stages r, s, w and the codes of a brick plus a
//    one-cell halo in shared memory (halo cells across a periodic edge are fetched from the opposite side), so
//    every value is read from L2/HBM once per brick instead of once per neighbour;
//  - the iteration is the Chronopoulos-Gear form of (P)CG: both dot products of an iteration are reduced together,
//    so there is ONE grid barrier per iteration. r, s and w are double-buffered: a block recomputes its halo's new
//    residuals from the old buffers while other blocks write the new ones;
//  - reductions: every block publishes its partial sums; the last block to arrive at the barrier adds all of them
//    in block order (the same order whichever block is last) and publishes the totals, so every block takes the
//    same deterministic scalar decisions;
//  - FIXED mode reproduces the reference: M = I, x0 = 0, exactly N iterations, alpha/beta = 0 when the denominator
//    magnitude is <= 1e-20. Tolerance mode stops at ||r|| <= tol ||b||. With refinement, the solution is accumulated
//    in FP64 (x64 += e after each FP32 inner solve of A e = r) and r = b - A x64 is recomputed in FP64, so the
//    residual can go below the FP32 floor of the pressure itself;
//  - every grid barrier waits at most kBarrierTimeoutNs, then raises an abort flag that makes all blocks leave; the
//    host reads the outcome from the status block.
#include "launch.h"
#include "smoke_b200_ext.h"

namespace smoke_b200 {

namespace {

constexpr int kThreads = 512;
constexpr int BX = 32, BY = 8, BZ = 8;
constexpr int TX = BX + 2, TY = BY + 2, TZ = BZ + 2;
constexpr int kTile = TX * TY * TZ;
constexpr int kBrick = BX * BY * BZ;
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s
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
template <typename T>
__device__ void block_sum4(T v[4], T (*scratch)[kThreads / 32]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) scratch[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = warp_sum(lane < kThreads / 32 ? scratch[k][lane] : T(0));
    }
    __syncthreads();
}

// Grid barrier fused with a deterministic all-reduce of 4 sums. Returns false if the solve was aborted.
template <typename T>
__device__ bool barrier_allreduce(PcgControl* ctl, int parity, T local[4], T out[4]) {
    __shared__ T scratch[4][kThreads / 32];
    __shared__ int s_last, s_ok;
    block_sum4(local, scratch);
    unsigned gen = 0;
    if (threadIdx.x == 0) {
        double* slot = ctl->partial[0][blockIdx.x];
#pragma unroll
        for (int k = 0; k < 4; ++k) slot[k] = static_cast<double>(local[k]);
        // read the generation before arriving: it cannot advance until this block has arrived
        gen = *static_cast<volatile unsigned*>(&ctl->gen);
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->count, 1u);
        s_last = arrived == gridDim.x - 1;
    }
    __syncthreads();
    int ok = 1;
    if (s_last) {
        // the last block adds every block's partials in block order
        T v[4] = {0, 0, 0, 0};
        for (unsigned b = threadIdx.x; b < gridDim.x; b += kThreads) {
            const double* slot = ctl->partial[0][b];
#pragma unroll
            for (int k = 0; k < 4; ++k) v[k] += static_cast<T>(__ldcg(slot + k));
        }
        block_sum4(v, scratch);
        if (threadIdx.x == 0) {
            double* tot = ctl->partial[1][parity];
#pragma unroll
            for (int k = 0; k < 4; ++k) tot[k] = static_cast<double>(v[k]);
            atomicExch(&ctl->count, 0u);
            __threadfence();
            atomicAdd(&ctl->gen, 1u);
        }
    } else if (threadIdx.x == 0) {
        volatile unsigned* vgen = &ctl->gen;
        volatile int* vabort = &ctl->abort;
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
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (*static_cast<volatile int*>(&ctl->abort)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    const double* tot = ctl->partial[1][parity];
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = static_cast<T>(__ldcg(tot + k));
    __syncthreads();
    return s_ok != 0;
}

struct Bricks {
    int nbx, nby, count;
};

__device__ __forceinline__ void brick_origin(const Bricks& B, int b, int& x0, int& y0, int& z0) {
    const int bx = b % B.nbx;
    const int t = b / B.nbx;
    const int by = t % B.nby;
    const int bz = t / B.nby;
    x0 = bx * BX;
    y0 = by * BY;
    z0 = bz * BZ;
}

// Global cell of tile slot t (halo included), wrapped across periodic edges; false outside the domain.
__device__ __forceinline__ bool tile_cell(const StepParams& P, int x0, int y0, int z0, int t, uint32_t& q) {
    int gx = x0 + t % TX - 1;
    int gy = y0 + (t / TX) % TY - 1;
    int gz = z0 + t / (TX * TY) - 1;
    if (gx < 0 || gx >= P.nx) {
        if (!P.fper[0]) return false;
        gx = wrapi(gx, P.nx);
    }
    if (gy < 0 || gy >= P.ny) {
        if (!P.fper[1]) return false;
        gy = wrapi(gy, P.ny);
    }
    if (gz < 0 || gz >= P.nz) {
        if (!P.fper[2]) return false;
        gz = wrapi(gz, P.nz);
    }
    q = cidx(P, gx, gy, gz);
    return true;
}

// Own cell c (0..kBrick) of a brick: tile slot and global index; false outside the domain.
__device__ __forceinline__ bool own_cell(const StepParams& P, int x0, int y0, int z0, int c, int& slot, uint32_t& q) {
    const int bx = c % BX, by = (c / BX) % BY, bz = c / (BX * BY);
    const int gx = x0 + bx, gy = y0 + by, gz = z0 + bz;
    slot = ((bz + 1) * TY + (by + 1)) * TX + (bx + 1);
    if (gx >= P.nx || gy >= P.ny || gz >= P.nz) return false;
    q = cidx(P, gx, gy, gz);
    return true;
}

template <bool JACOBI>
__device__ __forceinline__ float inv_diag(uint16_t code) {
    if constexpr (JACOBI) return __frcp_rn(static_cast<float>((code >> 8) & 7u));
    else return 1.0f;
}
__device__ __forceinline__ float diag_of(uint16_t code) { return static_cast<float>((code >> 8) & 7u); }

// Masked 7-point stencil on a tile array: diag * v[slot] - sum of active neighbours.
template <typename V>
__device__ __forceinline__ V stencil(const V* tile, int slot, uint16_t code) {
    V acc = static_cast<V>(diag_of(code)) * tile[slot];
    if (code & 1u) acc -= tile[slot - 1];
    if (code & 2u) acc -= tile[slot + 1];
    if (code & 4u) acc -= tile[slot - TX];
    if (code & 8u) acc -= tile[slot + TX];
    if (code & 16u) acc -= tile[slot - TX * TY];
    if (code & 32u) acc -= tile[slot + TX * TY];
    return acc;
}

struct Smem {
    float r[kTile];
    float s[kTile];
    float w[kTile];
    float u[kTile];
    uint16_t code[kTile];
};

template <typename T>
__device__ __forceinline__ bool finite_all(T a, T b, T c) { return isfinite(a) && isfinite(b) && isfinite(c); }

template <bool JACOBI, typename T>
__global__ void __launch_bounds__(kThreads, 1) pcg_kernel(const __grid_constant__ StepParams P, const PcgSettings S, const Bricks B, const uint16_t* __restrict__ codes, const float* __restrict__ b, float* x, PcgWork W, PcgControl* ctl) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
    const bool ir = !S.fixed && S.refinement > 0;  // FP64 accumulation + true-residual passes
    float* e = ir ? W.e : x;                         // the FP32 iterate
    const T guard = static_cast<T>(1.0e-20);
    int parity = 0;
    int cur = 0;
    uint32_t status = SMOKE_B200_SOLVE_ITERATION_CAP;
    double true_rel = -1.0;
    int it = 0, passes = 1;
    bool aborted = false;

    auto sync_sums = [&](T local[4], T out[4]) -> bool {
        const bool ok = barrier_allreduce<T>(ctl, parity, local, out);
        parity ^= 1;
        if (!ok) aborted = true;
        return ok;
    };

    // ------------------------------------------------------------ pass start: R[cur] = r0 given; W[cur] = A M r0
    // src: the residual to start from; from_b: r0 = b (cold start, nothing else written yet)
    auto start_pass = [&](const float* src, bool zero_x, T sums[4]) -> bool {
        T loc[4] = {0, 0, 0, 0};
        for (int br = blockIdx.x; br < B.count; br += gridDim.x) {
            int x0, y0, z0;
            brick_origin(B, br, x0, y0, z0);
            for (int t = threadIdx.x; t < kTile; t += kThreads) {
                uint32_t q;
                float rv = 0.0f;
                uint16_t cd = 0;
                if (tile_cell(P, x0, y0, z0, t, q)) {
                    rv = __ldcg(src + q);
                    cd = __ldg(codes + q);
                }
                sm.u[t] = rv * inv_diag<JACOBI>(cd);
                sm.code[t] = cd;
            }
            __syncthreads();
            for (int c = threadIdx.x; c < kBrick; c += kThreads) {
                int slot;
                uint32_t q;
                if (!own_cell(P, x0, y0, z0, c, slot, q)) continue;
                const uint16_t cd = sm.code[slot];
                const float r = __ldcg(src + q);
                const float u = sm.u[slot];
                const float w = stencil(sm.u, slot, cd);
                W.r[cur][q] = r;
                W.w[cur][q] = w;
                W.s[cur][q] = 0.0f;
                W.p[q] = 0.0f;
                if (zero_x) e[q] = 0.0f;
                loc[0] += static_cast<T>(r) * static_cast<T>(u);
                loc[1] += static_cast<T>(w) * static_cast<T>(u);
                loc[2] += static_cast<T>(r) * static_cast<T>(r);
                loc[3] += static_cast<T>(__ldg(b + q)) * static_cast<T>(__ldg(b + q));
            }
            __syncthreads();
        }
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
        for (int br = blockIdx.x; br < B.count; br += gridDim.x) {
            int x0, y0, z0;
            brick_origin(B, br, x0, y0, z0);
            for (int t = threadIdx.x; t < kTile; t += kThreads) {
                uint32_t q;
                float r = 0.0f, s = 0.0f, w = 0.0f;
                uint16_t cd = 0;
                if (tile_cell(P, x0, y0, z0, t, q)) {
                    r = __ldcg(Rc + q);
                    s = __ldcg(Sc + q);
                    w = __ldcg(Wc + q);
                    cd = __ldg(codes + q);
                }
                sm.r[t] = r;
                sm.s[t] = s;
                sm.w[t] = w;
                sm.code[t] = cd;
                const float sn = w + fb * s;    // s_i
                const float rn = r - fa * sn;   // r_{i+1}
                sm.u[t] = rn * inv_diag<JACOBI>(cd);  // u_{i+1} = M r_{i+1}
            }
            __syncthreads();
            for (int c = threadIdx.x; c < kBrick; c += kThreads) {
                int slot;
                uint32_t q;
                if (!own_cell(P, x0, y0, z0, c, slot, q)) continue;
                const uint16_t cd = sm.code[slot];
                const float inv = inv_diag<JACOBI>(cd);
                const float r = sm.r[slot], s = sm.s[slot], w = sm.w[slot];
                const float pv = r * inv + fb * __ldcg(W.p + q);  // p_i = u_i + beta p_{i-1}
                const float sn = w + fb * s;
                const float rn = r - fa * sn;
                const float un = sm.u[slot];
                const float wn = stencil(sm.u, slot, cd);  // w_{i+1} = A u_{i+1}
                W.p[q] = pv;
                e[q] = __ldcg(e + q) + fa * pv;
                Rn[q] = rn;
                Sn[q] = sn;
                Wn[q] = wn;
                loc[0] += static_cast<T>(rn) * static_cast<T>(un);
                loc[1] += static_cast<T>(wn) * static_cast<T>(un);
                loc[2] += static_cast<T>(rn) * static_cast<T>(rn);
            }
            __syncthreads();
        }
        const bool ok = sync_sums(loc, sums);
        cur ^= 1;
        return ok;
    };

    // ------------------------------------------------------------ FP64 accumulation and true residual
    auto accumulate = [&]() {  // x64 (+)= e, e = 0
        for (int br = blockIdx.x; br < B.count; br += gridDim.x) {
            int x0, y0, z0;
            brick_origin(B, br, x0, y0, z0);
            for (int c = threadIdx.x; c < kBrick; c += kThreads) {
                int slot;
                uint32_t q;
                if (!own_cell(P, x0, y0, z0, c, slot, q)) continue;
                W.x64[q] = (passes == 1 && !S.warm_start ? 0.0 : W.x64[q]) + static_cast<double>(__ldcg(e + q));
            }
        }
    };
    auto true_residual = [&](double sums[4]) -> bool {  // R[cur] = b - A x64 (FP64), returns ||r||^2
        double* tile = reinterpret_cast<double*>(smem_raw);  // kTile doubles fit in the r/s/w arrays
        double loc[4] = {0, 0, 0, 0};
        for (int br = blockIdx.x; br < B.count; br += gridDim.x) {
            int x0, y0, z0;
            brick_origin(B, br, x0, y0, z0);
            for (int t = threadIdx.x; t < kTile; t += kThreads) {
                uint32_t q;
                double v = 0.0;
                uint16_t cd = 0;
                if (tile_cell(P, x0, y0, z0, t, q)) {
                    v = __ldcg(W.x64 + q);
                    cd = __ldg(codes + q);
                }
                tile[t] = v;
                sm.code[t] = cd;
            }
            __syncthreads();
            for (int c = threadIdx.x; c < kBrick; c += kThreads) {
                int slot;
                uint32_t q;
                if (!own_cell(P, x0, y0, z0, c, slot, q)) continue;
                const double rv = static_cast<double>(__ldg(b + q)) - stencil(tile, slot, sm.code[slot]);
                W.r[cur][q] = static_cast<float>(rv);
                loc[0] += rv * rv;
            }
            __syncthreads();
        }
        const bool ok = barrier_allreduce<double>(ctl, parity, loc, sums);
        parity ^= 1;
        if (!ok) aborted = true;
        return ok;
    };

    // ------------------------------------------------------------ setup
    T sums[4] = {0, 0, 0, 0};
    if (S.warm_start && ir) {
        // x64 was seeded by the host (from the previous pressure); e = 0, r0 = b - A x64
        for (uint32_t q = blockIdx.x * kThreads + threadIdx.x; q < P.n; q += gridDim.x * kThreads) e[q] = 0.0f;
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
        for (uint32_t q = blockIdx.x * kThreads + threadIdx.x; q < P.n; q += gridDim.x * kThreads) {
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
            if (!sync_sums(none, dummy)) break;
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
            // the FP32 pressure is the rounded FP64 solution
            for (uint32_t q = blockIdx.x * kThreads + threadIdx.x; q < P.n; q += gridDim.x * kThreads) x[q] = static_cast<float>(W.x64[q]);
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
        st.reserved = 0;
        ctl->status = st;
    }
}

template <bool J, typename T>
cudaError_t launch_one(const StepParams& P, const PcgSettings& S, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s) {
    static int max_blocks = 0;
    const size_t smem = sizeof(Smem);
    if (max_blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaFuncSetAttribute(pcg_kernel<J, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e == cudaSuccess) e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<J, T>, kThreads, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorLaunchOutOfResources;
        max_blocks = sms * per_sm;
        if (max_blocks > kPcgMaxBlocks) max_blocks = kPcgMaxBlocks;
    }
    Bricks B{};
    B.nbx = (P.nx + BX - 1) / BX;
    B.nby = (P.ny + BY - 1) / BY;
    const int nbz = (P.nz + BZ - 1) / BZ;
    B.count = B.nbx * B.nby * nbz;
    const int blocks = B.count < max_blocks ? B.count : max_blocks;
    cudaError_t e = cudaMemsetAsync(ctl, 0, 4 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pcg_kernel<J, T>, P, S, B, codes, b, x, work, ctl);
}

}  // namespace

cudaError_t pcg_launch_shape(PcgLaunchShape* out) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    out->blocks = sms;
    out->threads = kThreads;
    return cudaSuccess;
}

cudaError_t launch_pcg(const StepParams& P, const PcgSettings& S, const PcgLaunchShape&, const uint16_t* codes, const float* b, float* x, PcgWork work, PcgControl* ctl, cudaStream_t s) {
    if (S.jacobi) return S.fp64 ? launch_one<true, double>(P, S, codes, b, x, work, ctl, s) : launch_one<true, float>(P, S, codes, b, x, work, ctl, s);
    return S.fp64 ? launch_one<false, double>(P, S, codes, b, x, work, ctl, s) : launch_one<false, float>(P, S, codes, b, x, work, ctl, s);
}

}  // namespace smoke_b200
