// Multigrid-preconditioned flexible conjugate gradients for the pressure system (one cooperative launch per solve).
//
// No reference counterpart: the reference solves with unpreconditioned CG (backend-cuda.cu:1788-1824), which at
// 128^3 needs ~900 iterations and stalls near relative residual 2.5e-5 in FP32. Here the preconditioner is one
// geometric multigrid V(1,1) cycle:
//  - levels: level l+1 halves every extent of level l (rounding up) down to <= 4 cells per axis; a coarse cell is
//    fluid when any child is; each level's operator is the masked 7-point stencil of its fluid cells, built with
//    the fine rules (periodic wrap, OUTFLOW faces on the diagonal) but without the anchor;
//  - smoothing: damped Jacobi, weight kOmega; the first pre-smoothing sweep starts from zero;
//  - restriction: r_{l+1}(C) = 1/2 * sum of the residuals of C's (up to 8) children after pre-smoothing; with the
//    trilinear prolongation below this is the Petrov-Galerkin scaling of the 7-point operator (R A P ~ 2 A_coarse);
//  - prolongation: cell-centred trilinear (weights 3/4 and 1/4 per axis); a corner outside the domain or in a
//    non-fluid coarse cell takes the parent's value;
//  - levels with more than kMgBlockLevelCells cells run grid-wide (grid barriers between passes); coarser levels run
//    inside block 0 with block barriers only, while the other blocks wait at the next grid barrier.
// The outer iteration is flexible CG (Notay 2000: beta_k = -(z_k, q_{k-1}) / (p_{k-1}, q_{k-1})), which stays
// valid when the preconditioner is not exactly symmetric. Refinement passes accumulate the solution in FP64 and
// restart from the FP64 residual b - A x64, as in pcg.cu.
#include "grid_sync.cuh"
#include "launch.h"
#include "smoke_b200_ext.h"

namespace smoke_b200 {

namespace {

constexpr int kThreads = 256;
constexpr float kOmega = 0.8f;
constexpr int kCoarsestSweeps = 16;

using gsync::global_ns;

template <typename T>
__device__ __forceinline__ bool barrier_allreduce(PcgControl* ctl, unsigned& phase, T local[4], T out[4], bool reduce = true) {
    return gsync::barrier_allreduce<kThreads, T>(ctl, phase, local, out, reduce);
}

__device__ __forceinline__ void lxyz(const MgLevel& L, uint32_t q, int& x, int& y, int& z) {
    const uint32_t zz = L.div_slab.div(q);
    const uint32_t rem = q - zz * static_cast<uint32_t>(L.nx) * L.ny;
    const uint32_t yy = L.div_nx.div(rem);
    x = static_cast<int>(rem - yy * L.nx);
    y = static_cast<int>(yy);
    z = static_cast<int>(zz);
}
__device__ __forceinline__ uint32_t lidx(const MgLevel& L, int x, int y, int z) { return (static_cast<uint32_t>(z) * L.ny + y) * L.nx + x; }

// Neighbour e of an active stencil bit (in range, or across a periodic edge).
__device__ __forceinline__ uint32_t lnbr(const MgLevel& L, uint32_t q, int x, int y, int z, int e) {
    const uint32_t nx = L.nx, slab = static_cast<uint32_t>(L.nx) * L.ny;
    switch (e) {
    case 0: return x > 0 ? q - 1 : q + (nx - 1);
    case 1: return x < L.nx - 1 ? q + 1 : q - (nx - 1);
    case 2: return y > 0 ? q - nx : q + (L.ny - 1) * nx;
    case 3: return y < L.ny - 1 ? q + nx : q - (L.ny - 1) * nx;
    case 4: return z > 0 ? q - slab : q + (L.nz - 1) * slab;
    default: return z < L.nz - 1 ? q + slab : q - (L.nz - 1) * slab;
    }
}

__device__ __forceinline__ float diagf(uint16_t code) { return static_cast<float>((code >> 8) & 7u); }

// diag * v(q) - sum of v over the active neighbours; v(index) supplies the values.
template <class V>
__device__ __forceinline__ float apply_stencil(const MgLevel& L, uint32_t q, uint16_t code, float vq, V&& v) {
    float acc = diagf(code) * vq;
    const uint32_t mask = code & 63u;
    if (mask) {
        int x, y, z;
        lxyz(L, q, x, y, z);
#pragma unroll
        for (int e = 0; e < 6; ++e)
            if (mask & (1u << e)) acc -= v(lnbr(L, q, x, y, z, e));
    }
    return acc;
}

__device__ __forceinline__ bool wrap_c(int& v, int n, int per) {
    if (v >= 0 && v < n) return true;
    if (!per) return false;
    v %= n;
    if (v < 0) v += n;
    return true;
}

// Cell-centred trilinear prolongation of coarse level C's correction zp at fine cell (x, y, z).
__device__ __forceinline__ float prolong(const MgLevel& C, const int* fper, int x, int y, int z) {
    const int X = x >> 1, Y = y >> 1, Z = z >> 1;
    const int sx = (x & 1) ? 1 : -1, sy = (y & 1) ? 1 : -1, sz = (z & 1) ? 1 : -1;
    const float parent = C.zp[lidx(C, X, Y, Z)];
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const float w = (i ? 0.25f : 0.75f) * (j ? 0.25f : 0.75f) * (k ? 0.25f : 0.75f);
                float v = parent;
                if (i | j | k) {
                    int cx = X + i * sx, cy = Y + j * sy, cz = Z + k * sz;
                    if (wrap_c(cx, C.nx, fper[0]) && wrap_c(cy, C.ny, fper[1]) && wrap_c(cz, C.nz, fper[2])) {
                        const uint32_t cq = lidx(C, cx, cy, cz);
                        if (C.fluid[cq]) v = C.zp[cq];
                    }
                }
                acc += w * v;
            }
    return acc;
}

// ---------------------------------------------------------------------------------------------- V-cycle passes
// Pre-smooth level l from zero (zp = w D^-1 r) and restrict the residual to level l+1 (coarse-cell parallel).
__device__ void restrict_pass(const MgHierarchy& H, int l, uint32_t first, uint32_t stride) {
    const MgLevel& F = H.L[l];
    const MgLevel& C = H.L[l + 1];
    for (uint32_t cq = first; cq < C.n; cq += stride) {
        int X, Y, Z;
        lxyz(C, cq, X, Y, Z);
        float sum = 0.0f;
#pragma unroll
        for (int dz = 0; dz < 2; ++dz)
#pragma unroll
            for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                for (int dx = 0; dx < 2; ++dx) {
                    const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                    if (x >= F.nx || y >= F.ny || z >= F.nz) continue;
                    const uint32_t q = lidx(F, x, y, z);
                    const uint16_t code = F.code[q];
                    const float rq = F.r[q];
                    const float zq = kOmega * rq / diagf(code);
                    F.zp[q] = zq;
                    const float az = apply_stencil(F, q, code, zq, [&](uint32_t nb) { return kOmega * F.r[nb] / diagf(F.code[nb]); });
                    sum += rq - az;
                }
        C.r[cq] = C.fluid[cq] ? 0.5f * sum : 0.0f;
    }
}

// Up, part 1: t = zp + P(z_coarse) on level l (zero on non-fluid cells; on level 0 also on the anchor).
__device__ void prolong_pass(const MgHierarchy& H, int l, int32_t anchor, uint32_t first, uint32_t stride) {
    const MgLevel& F = H.L[l];
    const MgLevel& C = H.L[l + 1];
    for (uint32_t q = first; q < F.n; q += stride) {
        float v = 0.0f;
        if (F.fluid[q] && !(l == 0 && static_cast<int32_t>(q) == anchor)) {
            int x, y, z;
            lxyz(F, q, x, y, z);
            v = F.zp[q] + prolong(C, H.fper, x, y, z);
        }
        F.t[q] = v;
    }
}

// Up, part 2: post-smooth zp = t + w D^-1 (r - A t) on level l. On level 0 the result is the preconditioned residual,
// and the partial sums (z, r) and (z, q) are accumulated.
template <typename T>
__device__ void smooth_pass(const MgHierarchy& H, int l, int32_t anchor, const float* q_prev, uint32_t first, uint32_t stride, T& zr, T& zq) {
    const MgLevel& F = H.L[l];
    for (uint32_t q = first; q < F.n; q += stride) {
        float v = 0.0f;
        if (F.fluid[q] && !(l == 0 && static_cast<int32_t>(q) == anchor)) {
            const uint16_t code = F.code[q];
            const float tq = F.t[q];
            const float at = apply_stencil(F, q, code, tq, [&](uint32_t nb) { return F.t[nb]; });
            v = tq + kOmega * (F.r[q] - at) / diagf(code);
        }
        F.zp[q] = v;
        if (l == 0) {
            zr += static_cast<T>(v) * static_cast<T>(F.r[q]);
            zq += static_cast<T>(v) * static_cast<T>(q_prev[q]);
        }
    }
}

// Coarsest level: Jacobi sweeps from zero, ping-pong between zp and t, result in zp.
__device__ void coarsest_solve(const MgLevel& L, uint32_t first, uint32_t stride, bool block_only) {
    for (uint32_t q = first; q < L.n; q += stride) L.zp[q] = L.fluid[q] ? kOmega * L.r[q] / diagf(L.code[q]) : 0.0f;
    for (int sweep = 0; sweep < kCoarsestSweeps; ++sweep) {
        if (block_only) __syncthreads();
        float* src = (sweep & 1) ? L.t : L.zp;
        float* dst = (sweep & 1) ? L.zp : L.t;
        for (uint32_t q = first; q < L.n; q += stride) {
            float v = 0.0f;
            if (L.fluid[q]) {
                const uint16_t code = L.code[q];
                const float s = src[q];
                v = s + kOmega * (L.r[q] - apply_stencil(L, q, code, s, [&](uint32_t nb) { return src[nb]; })) / diagf(code);
            }
            dst[q] = v;
        }
    }
    if (block_only) __syncthreads();
}

template <typename T>
__device__ __forceinline__ bool finite3(T a, T b, T c) { return isfinite(a) && isfinite(b) && isfinite(c); }

template <typename T>
__global__ void __launch_bounds__(kThreads, 2) mgfcg_kernel(const __grid_constant__ StepParams P, const PcgSettings S, const __grid_constant__ MgHierarchy H, const float* __restrict__ b, float* x, MgWork W, const int32_t* anchor_ptr, PcgControl* ctl) {
    const MgLevel& L0 = H.L[0];
    const uint32_t n = L0.n;
    const uint32_t gfirst = blockIdx.x * kThreads + threadIdx.x, gstride = gridDim.x * kThreads;
    const int32_t anchor = *anchor_ptr;
    const bool ir = !S.fixed && S.refinement > 0;
    float* e = ir ? W.e : x;
    float* r = L0.r;
    float* z = L0.zp;
    unsigned phase = 0;
    int cur = 0;
    uint32_t status = SMOKE_B200_SOLVE_ITERATION_CAP;
    double true_rel = -1.0;
    int it = 0, passes = 1;
    bool aborted = false;
    T none[4] = {0, 0, 0, 0}, dummy[4];

    auto grid_barrier = [&]() -> bool {
        if (!barrier_allreduce<T>(ctl, phase, none, dummy, false)) aborted = true;
        return !aborted;
    };

    // One V-cycle on r -> z; returns the reduced (z, r) and (z, q_prev).
    auto vcycle = [&](const float* q_prev, T& zr_out, T& zq_out) -> bool {
        const int g = H.grid_levels;  // levels [0, g) are grid-wide; level g is the first with <= kMgBlockLevelCells
        for (int l = 0; l < g; ++l) {
            restrict_pass(H, l, gfirst, gstride);
            if (!grid_barrier()) return false;
        }
        // levels g .. coarsest: block 0 only
        if (blockIdx.x == 0) {
            const int lc = H.levels - 1;
            for (int l = g; l < lc; ++l) {
                restrict_pass(H, l, threadIdx.x, kThreads);
                __syncthreads();
            }
            coarsest_solve(H.L[lc], threadIdx.x, kThreads, true);
            for (int l = lc - 1; l >= g; --l) {
                prolong_pass(H, l, anchor, threadIdx.x, kThreads);
                __syncthreads();
                T a = 0, c = 0;
                smooth_pass<T>(H, l, anchor, q_prev, threadIdx.x, kThreads, a, c);
                __syncthreads();
            }
        }
        if (!grid_barrier()) return false;
        T zr = 0, zq = 0;
        for (int l = g - 1; l >= 0; --l) {
            prolong_pass(H, l, anchor, gfirst, gstride);
            if (!grid_barrier()) return false;
            smooth_pass<T>(H, l, anchor, q_prev, gfirst, gstride, zr, zq);
            if (l > 0 && !grid_barrier()) return false;
        }
        T loc[4] = {zr, zq, 0, 0}, tot[4];
        if (!barrier_allreduce<T>(ctl, phase, loc, tot)) {
            aborted = true;
            return false;
        }
        zr_out = tot[0];
        zq_out = tot[1];
        return true;
    };

    // ------------------------------------------------------------ setup: r = b (or b - A x64), e = 0, q = p = 0
    T bb = 0, rr0 = 0;
    {
        T loc[4] = {0, 0, 0, 0}, tot[4];
        for (uint32_t q = gfirst; q < n; q += gstride) {
            const float bv = __ldg(b + q);
            loc[0] += static_cast<T>(bv) * static_cast<T>(bv);
            e[q] = 0.0f;
            W.q[q] = 0.0f;
            W.p[0][q] = 0.0f;
            W.p[1][q] = 0.0f;
            if (!(S.warm_start && ir)) r[q] = bv;
        }
        if (barrier_allreduce<T>(ctl, phase, loc, tot)) bb = tot[0];
        else aborted = true;
        if (!aborted && S.warm_start && ir) {
            T l2[4] = {0, 0, 0, 0};
            for (uint32_t q = gfirst; q < n; q += gstride) {
                const uint16_t code = L0.code[q];
                const double ax = static_cast<double>(diagf(code)) * W.x64[q] - [&]() {
                    double s = 0.0;
                    const uint32_t mask = code & 63u;
                    if (mask) {
                        int cx, cy, cz;
                        lxyz(L0, q, cx, cy, cz);
                        for (int k = 0; k < 6; ++k)
                            if (mask & (1u << k)) s += W.x64[lnbr(L0, q, cx, cy, cz, k)];
                    }
                    return s;
                }();
                const double rv = static_cast<double>(__ldg(b + q)) - ax;
                r[q] = static_cast<float>(rv);
                l2[0] += static_cast<T>(rv * rv);
            }
            if (barrier_allreduce<T>(ctl, phase, l2, tot)) rr0 = tot[0];
            else aborted = true;
        } else {
            rr0 = bb;
        }
    }
    T rnorm2 = rr0;

    if (aborted) {
        status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
    } else if (!(bb > T(0))) {
        for (uint32_t q = gfirst; q < n; q += gstride) {
            x[q] = 0.0f;
            if (ir) W.x64[q] = 0.0;
        }
        rnorm2 = 0;
        status = SMOKE_B200_SOLVE_CONVERGED;
        if (!isfinite(bb)) status = SMOKE_B200_SOLVE_NOT_FINITE;
        if (ir) true_rel = 0.0;
    } else {
        const T tol2 = static_cast<T>(S.tolerance) * static_cast<T>(S.tolerance) * bb;
        T pass_rr0 = rr0;
        for (;;) {  // refinement passes
            T target2 = tol2;
            if (ir) {
                const T floor2 = T(9e-8) * pass_rr0;
                const T want2 = T(0.09) * tol2;
                target2 = want2 > floor2 ? want2 : floor2;
            }
            bool first = true;
            T alpha = 0, pq_prev = 1;
            if (rnorm2 <= target2) status = SMOKE_B200_SOLVE_CONVERGED;
            while (!(rnorm2 <= target2)) {
                T zr, zq;
                if (!vcycle(W.q, zr, zq)) break;
                const T beta = first ? T(0) : -zq / pq_prev;
                if (!isfinite(beta) || !isfinite(zr)) {
                    status = SMOKE_B200_SOLVE_NOT_FINITE;
                    break;
                }
                // pass A: p = z + beta p_old, q = A p, partials (p, q), (p, r)
                const float fb = static_cast<float>(beta);
                const float* po = W.p[cur];
                float* pn = W.p[cur ^ 1];
                T loc[4] = {0, 0, 0, 0}, tot[4];
                for (uint32_t q = gfirst; q < n; q += gstride) {
                    const uint16_t code = L0.code[q];
                    const float pv = z[q] + fb * po[q];
                    const float qv = apply_stencil(L0, q, code, pv, [&](uint32_t nb) { return z[nb] + fb * po[nb]; });
                    pn[q] = pv;
                    W.q[q] = qv;
                    loc[0] += static_cast<T>(pv) * static_cast<T>(qv);
                    loc[1] += static_cast<T>(pv) * static_cast<T>(r[q]);
                }
                if (!barrier_allreduce<T>(ctl, phase, loc, tot)) {
                    aborted = true;
                    break;
                }
                const T pq = tot[0], pr = tot[1];
                if (!(pq > T(0)) || !isfinite(pr)) {
                    status = isfinite(pq) ? SMOKE_B200_SOLVE_BREAKDOWN : SMOKE_B200_SOLVE_NOT_FINITE;
                    break;
                }
                alpha = pr / pq;
                const float fa = static_cast<float>(alpha);
                // pass B: e += alpha p, r -= alpha q
                T l2[4] = {0, 0, 0, 0};
                for (uint32_t q = gfirst; q < n; q += gstride) {
                    e[q] += fa * pn[q];
                    const float rv = r[q] - fa * W.q[q];
                    r[q] = rv;
                    l2[0] += static_cast<T>(rv) * static_cast<T>(rv);
                }
                if (!barrier_allreduce<T>(ctl, phase, l2, tot)) {
                    aborted = true;
                    break;
                }
                rnorm2 = tot[0];
                ++it;
                cur ^= 1;
                pq_prev = pq;
                first = false;
                if (!isfinite(rnorm2)) {
                    status = SMOKE_B200_SOLVE_NOT_FINITE;
                    break;
                }
                if (rnorm2 <= target2) {
                    status = SMOKE_B200_SOLVE_CONVERGED;
                    break;
                }
                if (it >= S.max_iterations) {
                    status = SMOKE_B200_SOLVE_ITERATION_CAP;
                    break;
                }
            }
            if (aborted || !ir) break;
            // FP64: x64 += e, r = b - A x64
            const bool fresh = passes == 1 && !S.warm_start;
            for (uint32_t q = gfirst; q < n; q += gstride) W.x64[q] = (fresh ? 0.0 : W.x64[q]) + static_cast<double>(e[q]);
            if (!grid_barrier()) break;
            double dl[4] = {0, 0, 0, 0}, dt[4];
            for (uint32_t q = gfirst; q < n; q += gstride) {
                const uint16_t code = L0.code[q];
                double ax = static_cast<double>(diagf(code)) * W.x64[q];
                const uint32_t mask = code & 63u;
                if (mask) {
                    int cx, cy, cz;
                    lxyz(L0, q, cx, cy, cz);
                    for (int k = 0; k < 6; ++k)
                        if (mask & (1u << k)) ax -= W.x64[lnbr(L0, q, cx, cy, cz, k)];
                }
                const double rv = static_cast<double>(__ldg(b + q)) - ax;
                r[q] = static_cast<float>(rv);
                e[q] = 0.0f;
                dl[0] += rv * rv;
            }
            if (!gsync::barrier_allreduce<kThreads, double>(ctl, phase, dl, dt)) {
                aborted = true;
                break;
            }
            true_rel = sqrt(dt[0] / static_cast<double>(bb));
            if (true_rel <= static_cast<double>(S.tolerance)) {
                status = SMOKE_B200_SOLVE_CONVERGED;
                break;
            }
            if (passes > S.refinement || it >= S.max_iterations || status != SMOKE_B200_SOLVE_CONVERGED) {
                if (status == SMOKE_B200_SOLVE_CONVERGED) status = SMOKE_B200_SOLVE_ITERATION_CAP;
                break;
            }
            ++passes;
            rnorm2 = static_cast<T>(dt[0]);
            pass_rr0 = rnorm2;
        }
        if (aborted) status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
        if (ir && !aborted)
            for (uint32_t q = gfirst; q < n; q += gstride) x[q] = static_cast<float>(W.x64[q]);
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

// ---------------------------------------------------------------------------------------------- hierarchy setup
__global__ void mg_fluid0_kernel(uint32_t n, const uint8_t* __restrict__ occ, uint8_t* __restrict__ fluid) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) fluid[q] = occ[q] == 0 ? 1 : 0;
}

__global__ void mg_coarsen_kernel(const MgLevel F, const MgLevel C) {
    const uint32_t cq = blockIdx.x * blockDim.x + threadIdx.x;
    if (cq >= C.n) return;
    int X, Y, Z;
    lxyz(C, cq, X, Y, Z);
    uint8_t any = 0;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                if (x < F.nx && y < F.ny && z < F.nz) any |= F.fluid[lidx(F, x, y, z)];
            }
    C.fluid[cq] = any;
}

// Operator codes of a coarse level: the fine rules (stencil_code_kernel) without the anchor.
__global__ void mg_code_kernel(const MgLevel L, const __grid_constant__ StepParams P) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= L.n) return;
    if (!L.fluid[q]) {
        L.code[q] = static_cast<uint16_t>(1u << 8);
        return;
    }
    int c[3];
    lxyz(L, q, c[0], c[1], c[2]);
    const int nn[3] = {L.nx, L.ny, L.nz};
    uint32_t diag = 0, mask = 0;
    for (int e = 0; e < 6; ++e) {
        const int a = e >> 1;
        int d[3] = {c[0], c[1], c[2]};
        d[a] += (e & 1) ? 1 : -1;
        if (d[a] < 0 || d[a] >= nn[a]) {
            if (!P.fper[a]) {
                if (P.flow[e].type == kFlowOutflow) ++diag;
                continue;
            }
            d[a] = wrapi(d[a], nn[a]);
        }
        const uint32_t nb = lidx(L, d[0], d[1], d[2]);
        if (!L.fluid[nb]) continue;
        ++diag;
        if (nb == q) continue;
        if ((e & 1) && nn[a] == 2 && P.fper[a]) continue;
        mask |= 1u << e;
    }
    if (diag == 0) diag = 1;
    L.code[q] = static_cast<uint16_t>(mask | (diag << 8));
}

template <typename T>
cudaError_t launch_mg_one(const StepParams& P, const PcgSettings& S, const MgHierarchy& H, const float* b, float* x, MgWork work, const int32_t* anchor, PcgControl* ctl, cudaStream_t s) {
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mgfcg_kernel<T>, kThreads, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorLaunchOutOfResources;
        max_blocks = sms * per_sm;
        if (max_blocks > kPcgMaxBlocks) max_blocks = kPcgMaxBlocks;
    }
    uint32_t want = (H.L[0].n + kThreads * 4 - 1) / (kThreads * 4);
    if (want < 1u) want = 1u;
    const int blocks = static_cast<int>(want < static_cast<uint32_t>(max_blocks) ? want : static_cast<uint32_t>(max_blocks));
    cudaError_t e = cudaMemsetAsync(ctl, 0, kPcgControlResetBytes, s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, mgfcg_kernel<T>, P, S, H, b, x, work, anchor, ctl);
}

}  // namespace

int mg_level_count(int nx, int ny, int nz) {
    int levels = 1;
    while ((nx > 4 || ny > 4 || nz > 4) && levels < kMgMaxLevels) {
        nx = (nx + 1) / 2;
        ny = (ny + 1) / 2;
        nz = (nz + 1) / 2;
        ++levels;
    }
    return levels < 2 ? 2 : levels;
}

cudaError_t launch_mg_setup(const StepParams& P, const MgHierarchy& H, const uint8_t* occ, cudaStream_t s) {
    mg_fluid0_kernel<<<(H.L[0].n + 255) / 256, 256, 0, s>>>(H.L[0].n, occ, H.L[0].fluid);
    for (int l = 1; l < H.levels; ++l) {
        mg_coarsen_kernel<<<(H.L[l].n + 255) / 256, 256, 0, s>>>(H.L[l - 1], H.L[l]);
        mg_code_kernel<<<(H.L[l].n + 255) / 256, 256, 0, s>>>(H.L[l], P);
    }
    return cudaGetLastError();
}

cudaError_t launch_mgfcg(const StepParams& P, const PcgSettings& S, const MgHierarchy& H, const float* b, float* x, MgWork work, const int32_t* anchor, PcgControl* ctl, cudaStream_t s) {
    return S.fp64 ? launch_mg_one<double>(P, S, H, b, x, work, anchor, ctl, s) : launch_mg_one<float>(P, S, H, b, x, work, anchor, ctl, s);
}

}  // namespace smoke_b200
