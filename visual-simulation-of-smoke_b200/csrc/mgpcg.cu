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
#include "march.cuh"
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

// Masked stencil on the march's ring plane: in-plane neighbours from the plane, -z/+z from registers.
__device__ __forceinline__ float zstencil(uint16_t code, float u0, float um1, float u1, const float* plane, int slot) {
    float acc = diagf(code) * u0;
    if (code & 1u) acc -= plane[slot - 1];
    if (code & 2u) acc -= plane[slot + 1];
    if (code & 4u) acc -= plane[slot - zmarch::PX];
    if (code & 8u) acc -= plane[slot + zmarch::PX];
    if (code & 16u) acc -= um1;
    if (code & 32u) acc -= u1;
    return acc;
}

__device__ __forceinline__ bool wrap_c(int& v, int n, int per) {
    if (v >= 0 && v < n) return true;
    if (!per) return false;
    v %= n;
    if (v < 0) v += n;
    return true;
}

// Cell-centred trilinear prolongation of coarse level C's final correction (C.t) at fine cell (x, y, z).
__device__ __forceinline__ float prolong(const MgLevel& C, const int* fper, int x, int y, int z) {
    const int X = x >> 1, Y = y >> 1, Z = z >> 1;
    const int sx = (x & 1) ? 1 : -1, sy = (y & 1) ? 1 : -1, sz = (z & 1) ? 1 : -1;
    const float parent = C.t[lidx(C, X, Y, Z)];
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
                        if (C.fluid[cq]) v = C.t[cq];
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

// Block-level up pass on level l (block 0 only): zp += P(t_{l+1}), then t = zp + w D^-1 (r - A zp).
__device__ void block_up(const MgHierarchy& H, int l) {
    const MgLevel& F = H.L[l];
    const MgLevel& C = H.L[l + 1];
    for (uint32_t q = threadIdx.x; q < F.n; q += zmarch::kThreads) {
        float v = 0.0f;
        if (F.fluid[q]) {
            int x, y, z;
            lxyz(F, q, x, y, z);
            v = F.zp[q] + prolong(C, H.fper, x, y, z);
        }
        F.zp[q] = v;
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < F.n; q += zmarch::kThreads) {
        float v = 0.0f;
        if (F.fluid[q]) {
            const uint16_t code = F.code[q];
            const float s0 = F.zp[q];
            v = s0 + kOmega * (F.r[q] - apply_stencil(F, q, code, s0, [&](uint32_t nb) { return F.zp[nb]; })) / diagf(code);
        }
        F.t[q] = v;
    }
    __syncthreads();
}

// Coarsest level (block 0 only): Jacobi sweeps from zero, ping-pong between zp and t, result in t.
__device__ void coarsest_solve(const MgLevel& L) {
    for (uint32_t q = threadIdx.x; q < L.n; q += zmarch::kThreads) L.t[q] = L.fluid[q] ? kOmega * L.r[q] / diagf(L.code[q]) : 0.0f;
    for (int sweep = 0; sweep < kCoarsestSweeps; ++sweep) {
        __syncthreads();
        float* src = (sweep & 1) ? L.zp : L.t;
        float* dst = (sweep & 1) ? L.t : L.zp;
        for (uint32_t q = threadIdx.x; q < L.n; q += zmarch::kThreads) {
            float v = 0.0f;
            if (L.fluid[q]) {
                const uint16_t code = L.code[q];
                const float s0 = src[q];
                v = s0 + kOmega * (L.r[q] - apply_stencil(L, q, code, s0, [&](uint32_t nb) { return src[nb]; })) / diagf(code);
            }
            dst[q] = v;
        }
    }
    __syncthreads();  // kCoarsestSweeps is even: the result is in t
}
static_assert(kCoarsestSweeps % 2 == 0, "the coarsest sweeps must end in t");

__device__ __forceinline__ float diag_safe(uint16_t code) {
    const float d = diagf(code);
    return d > 0.0f ? d : 1.0f;
}

struct UpdData {  // level-0 update + restriction pass
    float r, q, p, e;
    uint16_t code;
};
struct ProData {  // prolongation + smoothing pass
    float t, r, qp;
    uint16_t code;
};
struct PqData {  // p / q pass
    float z, p, r;
    uint16_t code;
};

template <typename T>
__device__ __forceinline__ bool finite3(T a, T b, T c) { return isfinite(a) && isfinite(b) && isfinite(c); }

template <typename T>
__global__ void __launch_bounds__(zmarch::kThreads, 2) mgfcg_kernel(const __grid_constant__ StepParams P, const PcgSettings S, const __grid_constant__ MgHierarchy H, const float* __restrict__ b, float* x, MgWork W, const int32_t* anchor_ptr, PcgControl* ctl) {
    __shared__ __align__(16) float ring[3][zmarch::kPlane];
    const MgLevel& L0 = H.L[0];
    const MgLevel& L1 = H.L[1];
    const uint32_t n = L0.n;
    const uint32_t gfirst = blockIdx.x * zmarch::kThreads + threadIdx.x, gstride = gridDim.x * zmarch::kThreads;
    const int32_t anchor = *anchor_ptr;
    const bool ir = !S.fixed && S.refinement > 0;
    float* e = ir ? W.e : x;
    float* rb[2] = {L0.r, W.r_alt};  // residual, double-buffered across the update pass
    int rc = 0;
    float* Z = L0.t;  // the preconditioned residual
    unsigned phase = 0;
    int cur = 0;
    uint32_t status = SMOKE_B200_SOLVE_ITERATION_CAP;
    double true_rel = -1.0;
    int it = 0, passes = 1;
    bool aborted = false;
    T none[4] = {0, 0, 0, 0}, dummy[4];
    const int g = H.grid_levels;
    // phase timing (block 0's timeline; blocks move in lock step between grid barriers)
    const bool prof = S.profile && blockIdx.x == 0 && threadIdx.x == 0;
    unsigned long long prof_acc[kSolverPhases] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned long long prof_last = prof ? global_ns() : 0;
    auto mark = [&](int k) {
        if (prof) {
            const unsigned long long t = global_ns();
            prof_acc[k] += t - prof_last;
            prof_last = t;
        }
    };

    auto level_geom = [&](int l) { return zmarch::geom_of(H.L[l].nx, H.L[l].ny, H.L[l].nz, H.fper); };
    auto level_cols = [&](int l) {
        zmarch::Columns C{};
        C.ncx = (H.L[l].nx + zmarch::CX - 1) / zmarch::CX;
        C.ncy = (H.L[l].ny + zmarch::CY - 1) / zmarch::CY;
        C.total = static_cast<uint32_t>(C.ncx) * C.ncy * H.L[l].nz;
        return C;
    };
    auto grid_barrier = [&]() -> bool {
        if (!gsync::barrier_allreduce<zmarch::kThreads, T>(ctl, phase, none, dummy, false)) aborted = true;
        return !aborted;
    };
    auto reduce = [&](T loc[4], T out[4]) -> bool {
        if (!gsync::barrier_allreduce<zmarch::kThreads, T>(ctl, phase, loc, out, true)) aborted = true;
        return !aborted;
    };
    auto zero_l1r = [&]() {
        for (uint32_t q = gfirst; q < L1.n; q += gstride) L1.r[q] = 0.0f;
    };

    // Level 0, pass 1: r -= alpha q, e += alpha p, pre-smooth (zp = w D^-1 r) and restrict the residual into L1.r
    // (atomic adds of 1/2 res); partial ||r||^2.
    auto update_restrict = [&](float fa, T& rr) {
        const zmarch::MarchGeom G = level_geom(0);
        const zmarch::Columns C = level_cols(0);
        const float* pc = W.p[cur];
        const float* r = rb[rc];
        float* rn_out = rb[rc ^ 1];
        zmarch::march<float, UpdData>(
            G, C, ring,
            [&](bool ok, uint32_t q, bool own, int, int, int) {
                UpdData d{0.0f, 0.0f, 0.0f, 0.0f, 0};
                if (ok) {
                    d.r = r[q];
                    d.q = W.q[q];
                    d.code = L0.code[q];
                    if (own) {
                        d.p = pc[q];
                        d.e = e[q];
                    }
                }
                return d;
            },
            [&](const UpdData& d) { return kOmega * (d.r - fa * d.q) / diag_safe(d.code); },
            [&](uint32_t q, const UpdData& d, float um1, float u0, float u1, const float* plane, int slot, int cx, int cy, int cz) {
                const float rn = d.r - fa * d.q;
                const float res = rn - zstencil(d.code, u0, um1, u1, plane, slot);
                rn_out[q] = rn;
                L0.zp[q] = u0;
                e[q] = d.e + fa * d.p;
                atomicAdd(L1.r + lidx(L1, cx >> 1, cy >> 1, cz >> 1), 0.5f * res);
                rr += static_cast<T>(rn) * static_cast<T>(rn);
            });
        rc ^= 1;
    };

    // Level l: t = zp + P(t_{l+1}) (0 on non-fluid cells and the anchor), then out = t + w D^-1 (r - A t).
    // Level 0 writes Z and accumulates (Z, r), (Z, q_prev); coarser levels write their t... through `dst`.
    auto prolong_smooth = [&](int l, float* dst, T& zr, T& zq) {
        const MgLevel& F = H.L[l];
        const MgLevel& Cn = H.L[l + 1];
        const float* rsrc = l == 0 ? rb[rc] : F.r;
        const zmarch::MarchGeom G = level_geom(l);
        const zmarch::Columns C = level_cols(l);
        zmarch::march<float, ProData>(
            G, C, ring,
            [&](bool ok, uint32_t q, bool own, int cx, int cy, int cz) {
                ProData d{0.0f, 0.0f, 0.0f, 0};
                if (ok && F.fluid[q] && !(l == 0 && static_cast<int32_t>(q) == anchor)) {
                    d.t = F.zp[q] + prolong(Cn, H.fper, cx, cy, cz);
                    d.code = F.code[q];
                    if (own) {
                        d.r = rsrc[q];
                        if (l == 0) d.qp = W.q[q];
                    }
                }
                return d;
            },
            [&](const ProData& d) { return d.t; },
            [&](uint32_t q, const ProData& d, float um1, float u0, float u1, const float* plane, int slot, int, int, int) {
                const float v = d.code ? u0 + kOmega * (d.r - zstencil(d.code, u0, um1, u1, plane, slot)) / diagf(d.code) : 0.0f;
                dst[q] = v;
                if (l == 0) {
                    zr += static_cast<T>(v) * static_cast<T>(d.r);
                    zq += static_cast<T>(v) * static_cast<T>(d.qp);
                }
            });
    };

    // Level 0, pass 3: p = Z + beta p_old, q = A p; partials (p, q), (p, r). Clears L1.r for the next restriction.
    auto pq_pass = [&](float fb, T& pq, T& pr) {
        const zmarch::MarchGeom G = level_geom(0);
        const zmarch::Columns C = level_cols(0);
        const float* po = W.p[cur];
        float* pn = W.p[cur ^ 1];
        zmarch::march<float, PqData>(
            G, C, ring,
            [&](bool ok, uint32_t q, bool own, int, int, int) {
                PqData d{0.0f, 0.0f, 0.0f, 0};
                if (ok) {
                    d.z = Z[q];
                    d.p = po[q];
                    d.code = L0.code[q];
                    if (own) d.r = rb[rc][q];
                }
                return d;
            },
            [&](const PqData& d) { return d.z + fb * d.p; },
            [&](uint32_t q, const PqData& d, float um1, float u0, float u1, const float* plane, int slot, int, int, int) {
                const float qv = zstencil(d.code, u0, um1, u1, plane, slot);
                pn[q] = u0;
                W.q[q] = qv;
                pq += static_cast<T>(u0) * static_cast<T>(qv);
                pr += static_cast<T>(u0) * static_cast<T>(d.r);
            });
        zero_l1r();
    };

    // The coarse part of a V-cycle: levels 1 .. coarsest, given L1.r; leaves L1.t.
    auto coarse_cycle = [&]() -> bool {
        for (int l = 1; l < g; ++l) {
            restrict_pass(H, l, gfirst, gstride);
            if (!grid_barrier()) return false;
        }
        mark(1);
        if (blockIdx.x == 0) {
            const int lc = H.levels - 1;
            for (int l = (g > 1 ? g : 1); l < lc; ++l) {
                restrict_pass(H, l, threadIdx.x, zmarch::kThreads);
                __syncthreads();
            }
            coarsest_solve(H.L[lc]);
            for (int l = lc - 1; l >= (g > 1 ? g : 1); --l) block_up(H, l);
        }
        if (!grid_barrier()) return false;
        mark(2);
        for (int l = g - 1; l >= 1; --l) {
            T a = 0, c = 0;
            prolong_smooth(l, H.L[l].t, a, c);
            if (!grid_barrier()) return false;
        }
        mark(3);
        return true;
    };

    // ------------------------------------------------------------ setup: r = b, e = q = p = 0, L1.r = 0
    T bb = 0;
    {
        T loc[4] = {0, 0, 0, 0}, tot[4];
        for (uint32_t q = gfirst; q < n; q += gstride) {
            const float bv = __ldg(b + q);
            loc[0] += static_cast<T>(bv) * static_cast<T>(bv);
            e[q] = 0.0f;
            W.q[q] = 0.0f;
            W.p[0][q] = 0.0f;
            W.p[1][q] = 0.0f;
            rb[0][q] = bv;
        }
        zero_l1r();
        if (reduce(loc, tot)) bb = tot[0];
    }
    T rnorm2 = bb;

    if (aborted) {
        status = SMOKE_B200_SOLVE_BARRIER_TIMEOUT;
    } else if (!(bb > T(0))) {
        for (uint32_t q = gfirst; q < n; q += gstride) {
            x[q] = 0.0f;
            if (ir) W.x64[q] = 0.0;
        }
        rnorm2 = 0;
        status = isfinite(bb) ? SMOKE_B200_SOLVE_CONVERGED : SMOKE_B200_SOLVE_NOT_FINITE;
        if (ir) true_rel = 0.0;
    } else {
        const T tol2 = static_cast<T>(S.tolerance) * static_cast<T>(S.tolerance) * bb;
        T pass_rr0 = bb;
        for (;;) {  // refinement passes
            T target2 = tol2;
            if (ir) {
                const T floor2 = T(9e-8) * pass_rr0;
                const T want2 = T(0.09) * tol2;
                target2 = want2 > floor2 ? want2 : floor2;
            }
            bool first = true;
            T alpha = 0, pq_prev = 1;
            for (;;) {
                // pass 1 (alpha = 0 on the first round: only the pre-smoothing and restriction of r)
                mark(6);
                T rr = 0;
                update_restrict(static_cast<float>(alpha), rr);
                T loc[4] = {rr, 0, 0, 0}, tot[4];
                if (!reduce(loc, tot)) break;
                mark(0);
                rnorm2 = tot[0];
                if (!first) ++it;
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
                // V-cycle: coarse levels, then level 0's prolongation and post-smoothing into Z
                if (!coarse_cycle()) break;
                T zr = 0, zq = 0;
                prolong_smooth(0, Z, zr, zq);
                T l2[4] = {zr, zq, 0, 0};
                if (!reduce(l2, tot)) break;
                mark(4);
                zr = tot[0];
                zq = tot[1];
                const T beta = first ? T(0) : -zq / pq_prev;
                if (!isfinite(beta) || !isfinite(zr)) {
                    status = SMOKE_B200_SOLVE_NOT_FINITE;
                    break;
                }
                // pass 3: p, q
                T pq = 0, pr = 0;
                pq_pass(static_cast<float>(beta), pq, pr);
                T l3[4] = {pq, pr, 0, 0};
                if (!reduce(l3, tot)) break;
                mark(5);
                pq = tot[0];
                pr = tot[1];
                cur ^= 1;
                if (!(pq > T(0)) || !isfinite(pr)) {
                    status = isfinite(pq) ? SMOKE_B200_SOLVE_BREAKDOWN : SMOKE_B200_SOLVE_NOT_FINITE;
                    break;
                }
                alpha = pr / pq;
                pq_prev = pq;
                first = false;
            }
            if (aborted || !ir) break;
            // FP64: x64 += e, r = b - A x64, e = q = 0, L1.r = 0
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
                rb[rc][q] = static_cast<float>(rv);
                e[q] = 0.0f;
                W.q[q] = 0.0f;
                dl[0] += rv * rv;
            }
            zero_l1r();
            if (!gsync::barrier_allreduce<zmarch::kThreads, double>(ctl, phase, dl, dt)) {
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

    mark(7);
    if (prof)
        for (int k = 0; k < kSolverPhases; ++k) ctl->phase_ns[k] = prof_acc[k];
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
    // at least ~8 column-planes of level 0 per block (see march.cuh)
    const uint32_t planes = zmarch::column_planes(zmarch::geom_of(H.L[0].nx, H.L[0].ny, H.L[0].nz, H.fper));
    uint32_t want = planes / 8u;
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
