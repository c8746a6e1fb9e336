// Multigrid-preconditioned flexible conjugate gradients for the pressure system (one cooperative launch per solve).
//
// No reference counterpart: the reference solves with unpreconditioned CG (backend-cuda.cu:1788-1824), which at
// 128^3 needs ~900 iterations and stalls near relative residual 2.5e-5 in FP32. Here the preconditioner is one
// geometric multigrid V(1,1) cycle:
//  - levels: level l+1 halves every extent of level l (rounding up) down to <= 4 cells per axis; a coarse cell is
//    active (fluid) when any child is; each level's operator is the masked 7-point stencil of its active cells,
//    built with the fine rules (periodic wrap, OUTFLOW faces on the diagonal) but without the anchor;
//  - smoothing: damped Jacobi, weight kOmega; the pre-smoothing sweep starts from zero;
//  - restriction: r_{l+1}(C) = 1/2 * sum of the residuals of C's (up to 8) children after pre-smoothing; with the
//    trilinear prolongation below this is the Petrov-Galerkin scaling of the 7-point operator (R A P ~ 2 A_coarse);
//  - prolongation: cell-centred trilinear (weights 3/4 and 1/4 per axis); a corner outside the domain or on an
//    inactive coarse cell takes the parent's value (inactive coarse cells carry the bit pattern kTag in t);
//  - the fine levels run grid-wide, one asynchronous z-march (amarch.cuh) per pass with grid barriers between
//    passes; the coarsest levels (at most kMgBlockLevelCells cells, kMgBlockBytes in all) run inside block 0 from
//    shared memory, while the other blocks wait at the next grid barrier.
// Per iteration, level 0 takes three passes: (1) r -= alpha q, e += alpha p, pre-smoothing and restriction of the
// residual (atomic adds into level 1, pre-summed over x and z pairs of children), (2) prolongation of the coarse
// correction plus post-smoothing into z, with (z, r) and (z, q), (3) p = z + beta p, q = A p, with (p, q), (p, r).
// The outer iteration is flexible CG (Notay 2000: beta_k = -(z_k, q_{k-1}) / (p_{k-1}, q_{k-1})), which stays
// valid when the preconditioner is not exactly symmetric. Refinement passes accumulate the solution in FP64 and
// restart from the FP64 residual b - A x64, as in pcg.cu.
#include "amarch.cuh"
#include "grid_sync.cuh"
#include "launch.h"
#include "smoke_b200_ext.h"

namespace smoke_b200 {

namespace {

constexpr int kThreads = amarch::kThreads;
constexpr float kOmega = 0.8f;
constexpr int kCoarsestSweeps = 16;
constexpr uint32_t kTag = 0x7fc0feedu;  // t of an inactive coarse cell (a NaN payload arithmetic never produces)
constexpr int kPlanesInFlight = 7;       // amarch look-ahead

// Stage layout of the level passes (32-bit words): up to 4 own fields and the own code word, up to 2 halo fields
// and the halo code word, and the prolongation's coarse tile (2 planes x 6 rows x 18 columns, shared).
constexpr int kOwnCode = 4 * kThreads;
constexpr int kHaloBase = 5 * kThreads;
constexpr int kHaloCode = kHaloBase + 2 * amarch::kHalo;
constexpr int kExtraBase = kHaloBase + 3 * amarch::kHalo;
constexpr int kTileX = 18, kTileY = 6, kTilePlane = kTileX * kTileY, kTileWords = 2 * kTilePlane;
constexpr int kStageWords = kExtraBase + kTileWords;
constexpr uint32_t kStageBytes = (kPlanesInFlight + 1) * kStageWords * 4u;
constexpr uint32_t kDynSmemBytes = kStageBytes > kMgBlockBytes ? kStageBytes : kMgBlockBytes;
static_assert(kStageWords % 4 == 0, "stages stay 16-byte aligned");
static_assert(kTileWords <= kThreads, "one tile word per thread");

using gsync::global_ns;

__device__ __forceinline__ bool active(uint16_t code) { return (code & kCodeActive) != 0; }
__device__ __forceinline__ float diagf(uint16_t code) { return static_cast<float>((code >> 8) & 7u); }
__device__ __forceinline__ bool is_tag(float v) { return __float_as_uint(v) == kTag; }
// Damped Jacobi step size w / diag (the preconditioner needs no correctly rounded quotient).
__device__ __forceinline__ float wdiag(uint16_t code) { return __fdividef(kOmega, diagf(code)); }

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

// diag * v(q) - sum of v over the active neighbours; v(index) supplies the values.
template <typename R, class V>
__device__ __forceinline__ R apply_stencil(const MgLevel& L, uint32_t q, uint16_t code, R vq, V&& v) {
    R acc = static_cast<R>(diagf(code)) * vq;
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

// Masked stencil on a ring plane: in-plane neighbours from the plane, -z/+z from registers.
__device__ __forceinline__ float zstencil(uint16_t code, float u0, float um1, float u1, const float* plane, int slot) {
    float acc = diagf(code) * u0;
    if (code & 1u) acc -= plane[slot - 1];
    if (code & 2u) acc -= plane[slot + 1];
    if (code & 4u) acc -= plane[slot - amarch::PX];
    if (code & 8u) acc -= plane[slot + amarch::PX];
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

// ---------------------------------------------------------------------------------------------- block levels
// Block-level level l in block 0's shared memory: the global level's extents with r, zp, t, code in `area`.
__device__ MgLevel smem_level(const MgHierarchy& H, float* area, int l) {
    uint32_t off = 0;
    for (int k = H.grid_levels; k < l; ++k) off += mg_block_words(H.L[k].n);
    MgLevel S = H.L[l];
    S.r = area + off;
    S.zp = S.r + S.n;
    S.t = S.zp + S.n;
    S.code = reinterpret_cast<uint16_t*>(S.t + S.n);
    S.fluid = nullptr;
    return S;
}

// Trilinear prolongation of C.t at fine cell (x, y, z), C's codes marking the active coarse cells.
__device__ __forceinline__ float prolong_smem(const MgLevel& C, const int* fper, int x, int y, int z) {
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
                        if (active(C.code[cq])) v = C.t[cq];
                    }
                }
                acc += w * v;
            }
    return acc;
}

// The coarse part of the V-cycle below the grid levels, in block 0: reads r of level g (global), runs restriction,
// the coarsest Jacobi sweeps and the up passes in shared memory, and writes t of level g (kTag on inactive cells).
// Block copy of `count` 32-bit words global -> shared with kCopyUnroll loads in flight per thread.
constexpr int kCopyUnroll = 16;
__device__ __forceinline__ void block_copy_words(uint32_t* dst, const uint32_t* src, uint32_t count) {
    for (uint32_t base = threadIdx.x; base < count; base += kThreads * kCopyUnroll) {
        uint32_t v[kCopyUnroll];
#pragma unroll
        for (int u = 0; u < kCopyUnroll; ++u) {
            const uint32_t i = base + u * kThreads;
            v[u] = i < count ? src[i] : 0u;
        }
#pragma unroll
        for (int u = 0; u < kCopyUnroll; ++u) {
            const uint32_t i = base + u * kThreads;
            if (i < count) dst[i] = v[u];
        }
    }
}

__device__ void block_cycle(const MgHierarchy& H, float* area) {
    const int g = H.grid_levels, lc = H.levels - 1;
    for (int l = g; l <= lc; ++l) {  // codes as aligned pairs (the arrays carry two spare entries)
        const MgLevel S = smem_level(H, area, l);
        block_copy_words(reinterpret_cast<uint32_t*>(S.code), reinterpret_cast<const uint32_t*>(H.L[l].code), (S.n + 1) / 2);
    }
    {
        const MgLevel S = smem_level(H, area, g);
        block_copy_words(reinterpret_cast<uint32_t*>(S.r), reinterpret_cast<const uint32_t*>(H.L[g].r), S.n);
    }
    __syncthreads();
    for (int l = g; l < lc; ++l) {
        const MgLevel F = smem_level(H, area, l);
        const MgLevel C = smem_level(H, area, l + 1);
        for (uint32_t q = threadIdx.x; q < C.n; q += kThreads) C.r[q] = 0.0f;
        for (uint32_t q = threadIdx.x; q < F.n; q += kThreads) {
            const uint16_t code = F.code[q];
            F.zp[q] = active(code) ? wdiag(code) * F.r[q] : 0.0f;
        }
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < F.n; q += kThreads) {
            const uint16_t code = F.code[q];
            if (!active(code)) continue;
            const float res = F.r[q] - apply_stencil<float>(F, q, code, F.zp[q], [&](uint32_t nb) { return F.zp[nb]; });
            int x, y, z;
            lxyz(F, q, x, y, z);
            atomicAdd(C.r + lidx(C, x >> 1, y >> 1, z >> 1), 0.5f * res);
        }
        __syncthreads();
    }
    {  // coarsest level: Jacobi sweeps from zero, ping-pong between t and zp, result in t
        const MgLevel L = smem_level(H, area, lc);
        for (uint32_t q = threadIdx.x; q < L.n; q += kThreads) {
            const uint16_t code = L.code[q];
            L.t[q] = active(code) ? wdiag(code) * L.r[q] : 0.0f;
        }
        for (int sweep = 0; sweep < kCoarsestSweeps; ++sweep) {
            __syncthreads();
            float* src = (sweep & 1) ? L.zp : L.t;
            float* dst = (sweep & 1) ? L.t : L.zp;
            for (uint32_t q = threadIdx.x; q < L.n; q += kThreads) {
                const uint16_t code = L.code[q];
                float v = 0.0f;
                if (active(code)) {
                    const float s0 = src[q];
                    v = s0 + wdiag(code) * (L.r[q] - apply_stencil<float>(L, q, code, s0, [&](uint32_t nb) { return src[nb]; }));
                }
                dst[q] = v;
            }
        }
        __syncthreads();
    }
    static_assert(kCoarsestSweeps % 2 == 0, "the coarsest sweeps end in t");
    for (int l = lc - 1; l >= g; --l) {
        const MgLevel F = smem_level(H, area, l);
        const MgLevel C = smem_level(H, area, l + 1);
        for (uint32_t q = threadIdx.x; q < F.n; q += kThreads) {
            if (!active(F.code[q])) continue;
            int x, y, z;
            lxyz(F, q, x, y, z);
            F.zp[q] += prolong_smem(C, H.fper, x, y, z);
        }
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < F.n; q += kThreads) {
            const uint16_t code = F.code[q];
            float v = 0.0f;
            if (active(code)) {
                const float s0 = F.zp[q];
                v = s0 + wdiag(code) * (F.r[q] - apply_stencil<float>(F, q, code, s0, [&](uint32_t nb) { return F.zp[nb]; }));
            }
            F.t[q] = v;
        }
        __syncthreads();
    }
    {
        const MgLevel S = smem_level(H, area, g);
        float* dst = H.L[g].t;
        for (uint32_t q = threadIdx.x; q < S.n; q += kThreads) dst[q] = active(S.code[q]) ? S.t[q] : __uint_as_float(kTag);
    }
}

// ---------------------------------------------------------------------------------------------- level passes
// Stage accessors: own field f, own code word, halo field f, halo code word.
__device__ __forceinline__ float* own_f(float* st, int f) { return st + f * kThreads + threadIdx.x; }
__device__ __forceinline__ uint32_t* own_code(float* st) { return reinterpret_cast<uint32_t*>(st + kOwnCode) + threadIdx.x; }
__device__ __forceinline__ float* halo_f(float* st, int f) { return st + kHaloBase + f * amarch::kHalo + threadIdx.x; }
__device__ __forceinline__ uint32_t* halo_code(float* st) { return reinterpret_cast<uint32_t*>(st + kHaloCode) + threadIdx.x; }

// One slot's copy source: whether the slot maps to a cell of an existing plane, and that cell.
struct SlotCopy {
    bool ok;
    uint32_t q;
};
__device__ __forceinline__ SlotCopy own_copy(const amarch::Slots& s, bool zok, uint32_t base) { return {zok && s.oload, base + s.ooff}; }
__device__ __forceinline__ SlotCopy halo_copy(const amarch::Slots& s, bool zok, uint32_t base) { return {zok && s.hload, base + s.hoff}; }
__device__ __forceinline__ void copy_field(float* dst, const float* src, const SlotCopy& c) { amarch::cp4(dst, c.ok ? src + c.q : src, c.ok); }
__device__ __forceinline__ void copy_code(uint32_t* dst, const uint16_t* code, const SlotCopy& c) {
    amarch::cp4(dst, c.ok ? amarch::code_word(code, c.q) : static_cast<const void*>(code), c.ok);
}

// Code of this thread's own (halo = false) or halo slot in a stage; q: the slot's cell (its parity picks the half).
__device__ __forceinline__ uint16_t slot_code(float* st, bool halo, uint32_t q) { return amarch::code_of(halo ? *halo_code(st) : *own_code(st), q); }

// Restriction of one residual contribution per own cell into the next level: the x pair is summed by a shuffle,
// the z pair in `acc` (held over from the even plane), then one atomic add per pair of pairs. Every thread calls it.
__device__ __forceinline__ void restrict_emit(float c, float& acc, const MgLevel& C, const amarch::Slots& s, int z, bool last) {
    c += __shfl_xor_sync(0xffffffffu, c, 1);
    if ((z & 1) == 0 && !last) {
        acc = c;
        return;
    }
    const float v = acc + c;
    acc = 0.0f;
    if ((threadIdx.x & 1u) == 0 && s.oout && v != 0.0f) atomicAdd(C.r + lidx(C, s.ox >> 1, s.oy >> 1, z >> 1), v);
}

// Coarse tile of fine plane z (unwrapped): coarse planes floor((z-1)/2) + k (k = 0, 1), columns x0/2 - 1 + i
// (i < 18), rows y0/2 - 1 + j (j < 6). Corners outside the domain hold kTag.
__device__ __forceinline__ void issue_tile(const MgLevel& C, const int* fper, const amarch::Slots& s, float* st, int z) {
    const int t = threadIdx.x;
    if (t >= kTileWords) return;
    const int k = t / kTilePlane, rem = t - k * kTilePlane;
    const int j = rem / kTileX, i = rem - j * kTileX;
    int X = (s.x0 >> 1) - 1 + i, Y = (s.y0 >> 1) - 1 + j, Zc = ((z - 1) >> 1) + k;
    float* dst = st + kExtraBase + t;
    if (wrap_c(X, C.nx, fper[0]) && wrap_c(Y, C.ny, fper[1]) && wrap_c(Zc, C.nz, fper[2]))
        amarch::cp4(dst, C.t + lidx(C, X, Y, Zc), true);
    else
        *dst = __uint_as_float(kTag);
}

// Prolongation at fine cell (x, y, z) (unwrapped, in the stage's column) from the stage's coarse tile.
__device__ __forceinline__ float prolong_tile(const float* st, const amarch::Slots& s, int x, int y, int z) {
    const float* tile = st + kExtraBase;
    const int ip = (x >> 1) - (s.x0 >> 1) + 1, jp = (y >> 1) - (s.y0 >> 1) + 1;
    const int kp = (z & 1) ? 0 : 1;
    const int di = (x & 1) ? 1 : -1, dj = (y & 1) ? kTileX : -kTileX, dk = (z & 1) ? kTilePlane : -kTilePlane;
    const int p0 = kp * kTilePlane + jp * kTileX + ip;
    float parent = tile[p0];
    if (is_tag(parent)) parent = 0.0f;
    const float c[8] = {parent, tile[p0 + di], tile[p0 + dj], tile[p0 + di + dj], tile[p0 + dk], tile[p0 + di + dk], tile[p0 + dj + dk], tile[p0 + di + dj + dk]};
    float acc = 0.0f;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const float w = ((m & 1) ? 0.25f : 0.75f) * ((m & 2) ? 0.25f : 0.75f) * ((m & 4) ? 0.25f : 0.75f);
        acc += w * (is_tag(c[m]) ? parent : c[m]);
    }
    return acc;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 2) mgfcg_kernel(const __grid_constant__ StepParams P, const PcgSettings S, const __grid_constant__ MgHierarchy H, const float* __restrict__ b, float* x, MgWork W, PcgControl* ctl) {
    extern __shared__ __align__(16) float dyn[];
    __shared__ __align__(16) float ring[amarch::kRing][amarch::kPlane];
    const MgLevel& L0 = H.L[0];
    const uint32_t n = L0.n;
    const uint32_t gfirst = blockIdx.x * kThreads + threadIdx.x, gstride = gridDim.x * kThreads;
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

    auto geom = [&](int l) {
        amarch::Geom G{H.L[l].nx, H.L[l].ny, H.L[l].nz, {H.fper[0], H.fper[1], H.fper[2]}};
        return G;
    };
    auto cols = [&](int l) { return amarch::columns_of(H.L[l].nx, H.L[l].ny, H.L[l].nz); };
    auto stage = [&](int k) { return dyn + k * kStageWords; };
    auto grid_barrier = [&]() -> bool {
        if (!gsync::barrier_allreduce<kThreads, T>(ctl, phase, none, dummy, false)) aborted = true;
        return !aborted;
    };
    auto reduce = [&](T loc[4], T out[4]) -> bool {
        if (!gsync::barrier_allreduce<kThreads, T>(ctl, phase, loc, out, true)) aborted = true;
        return !aborted;
    };
    auto zero_coarse_r = [&]() {  // levels 1 .. g receive atomic restrictions (level g is read by block 0)
        for (int l = 1; l <= g; ++l) {
            float* r = H.L[l].r;
            for (uint32_t q = gfirst; q < H.L[l].n; q += gstride) r[q] = 0.0f;
        }
    };

    // Level 0, pass 1: r -= alpha q, e += alpha p, pre-smooth (zp = w D^-1 r) and restrict the residual into L1.r;
    // partial ||r||^2. Stage fields: own r q p e, halo r q.
    auto update_restrict = [&](float fa, T& rr) {
        const float* pc = W.p[cur];
        const float* r = rb[rc];
        float* rn_out = rb[rc ^ 1];
        const MgLevel& C = H.L[1];
        float acc = 0.0f;
        amarch::march<kPlanesInFlight>(
            geom(0), cols(0), ring,
            [&](const amarch::Slots& s, int k, int, bool zok, uint32_t base) {
                float* st = stage(k);
                const SlotCopy o = own_copy(s, zok, base);
                copy_field(own_f(st, 0), r, o);
                copy_field(own_f(st, 1), W.q, o);
                copy_field(own_f(st, 2), pc, o);
                copy_field(own_f(st, 3), e, o);
                copy_code(own_code(st), L0.code, o);
                if (s.halo) {
                    const SlotCopy h = halo_copy(s, zok, base);
                    copy_field(halo_f(st, 0), r, h);
                    copy_field(halo_f(st, 1), W.q, h);
                    copy_code(halo_code(st), L0.code, h);
                }
            },
            [&](const amarch::Slots& s, int k, int, uint32_t base, bool halo) {
                float* st = stage(k);
                const uint16_t code = slot_code(st, halo, base + (halo ? s.hoff : s.ooff));
                if (!active(code)) return 0.0f;
                const float rv = halo ? *halo_f(st, 0) : *own_f(st, 0);
                const float qv = halo ? *halo_f(st, 1) : *own_f(st, 1);
                return wdiag(code) * (rv - fa * qv);
            },
            [&](const amarch::Slots& s, int k, int z, uint32_t q, float um1, float u0, float u1, const float* plane, bool last) {
                float c = 0.0f;
                if (s.oout) {
                    float* st = stage(k);
                    const uint16_t code = amarch::code_of(*own_code(st), q);
                    const float rn = *own_f(st, 0) - fa * *own_f(st, 1);
                    if (active(code)) c = 0.5f * (rn - zstencil(code, u0, um1, u1, plane, s.oslot));
                    rn_out[q] = rn;
                    L0.zp[q] = u0;
                    e[q] = *own_f(st, 3) + fa * *own_f(st, 2);
                    rr += static_cast<T>(rn) * static_cast<T>(rn);
                }
                restrict_emit(c, acc, C, s, z, last);
            });
        rc ^= 1;
    };

    // Level l >= 1: pre-smooth from zero (zp = w D^-1 r) and restrict the residual into level l + 1.
    auto restrict_level = [&](int l) {
        const MgLevel& F = H.L[l];
        const MgLevel& C = H.L[l + 1];
        float acc = 0.0f;
        amarch::march<kPlanesInFlight>(
            geom(l), cols(l), ring,
            [&](const amarch::Slots& s, int k, int, bool zok, uint32_t base) {
                float* st = stage(k);
                const SlotCopy o = own_copy(s, zok, base);
                copy_field(own_f(st, 0), F.r, o);
                copy_code(own_code(st), F.code, o);
                if (s.halo) {
                    const SlotCopy h = halo_copy(s, zok, base);
                    copy_field(halo_f(st, 0), F.r, h);
                    copy_code(halo_code(st), F.code, h);
                }
            },
            [&](const amarch::Slots& s, int k, int, uint32_t base, bool halo) {
                float* st = stage(k);
                const uint16_t code = slot_code(st, halo, base + (halo ? s.hoff : s.ooff));
                if (!active(code)) return 0.0f;
                return wdiag(code) * (halo ? *halo_f(st, 0) : *own_f(st, 0));
            },
            [&](const amarch::Slots& s, int k, int z, uint32_t q, float um1, float u0, float u1, const float* plane, bool last) {
                float c = 0.0f;
                if (s.oout) {
                    float* st = stage(k);
                    const uint16_t code = amarch::code_of(*own_code(st), q);
                    if (active(code)) c = 0.5f * (*own_f(st, 0) - zstencil(code, u0, um1, u1, plane, s.oslot));
                    F.zp[q] = u0;
                }
                restrict_emit(c, acc, C, s, z, last);
            });
    };

    // Level l: t = zp + P(t_{l+1}) on active cells (0 elsewhere), then dst = t + w D^-1 (r - A t) (kTag on
    // inactive coarse cells, 0 on inactive level-0 cells). Level 0 writes Z and accumulates (Z, r), (Z, q).
    // Stage fields: own zp r q, halo zp, the coarse tile.
    auto prolong_smooth = [&](int l, float* dst, T& zr, T& zq) {
        const MgLevel& F = H.L[l];
        const MgLevel& C = H.L[l + 1];
        const float* rsrc = l == 0 ? rb[rc] : F.r;
        const float inactive_value = l == 0 ? 0.0f : __uint_as_float(kTag);
        amarch::march<kPlanesInFlight>(
            geom(l), cols(l), ring,
            [&](const amarch::Slots& s, int k, int z, bool zok, uint32_t base) {
                float* st = stage(k);
                const SlotCopy o = own_copy(s, zok, base);
                copy_field(own_f(st, 0), F.zp, o);
                copy_field(own_f(st, 1), rsrc, o);
                if (l == 0) copy_field(own_f(st, 2), W.q, o);
                copy_code(own_code(st), F.code, o);
                if (s.halo) {
                    const SlotCopy h = halo_copy(s, zok, base);
                    copy_field(halo_f(st, 0), F.zp, h);
                    copy_code(halo_code(st), F.code, h);
                }
                if (zok) issue_tile(C, H.fper, s, st, z);
            },
            [&](const amarch::Slots& s, int k, int z, uint32_t base, bool halo) {
                float* st = stage(k);
                const uint16_t code = slot_code(st, halo, base + (halo ? s.hoff : s.ooff));
                if (!active(code)) return 0.0f;
                return halo ? *halo_f(st, 0) + prolong_tile(st, s, s.hx, s.hy, z) : *own_f(st, 0) + prolong_tile(st, s, s.ox, s.oy, z);
            },
            [&](const amarch::Slots& s, int k, int, uint32_t q, float um1, float u0, float u1, const float* plane, bool) {
                if (!s.oout) return;
                float* st = stage(k);
                const uint16_t code = amarch::code_of(*own_code(st), q);
                float v = inactive_value;
                if (active(code)) {
                    const float rv = *own_f(st, 1);
                    v = u0 + wdiag(code) * (rv - zstencil(code, u0, um1, u1, plane, s.oslot));
                    if (l == 0) {
                        zr += static_cast<T>(v) * static_cast<T>(rv);
                        zq += static_cast<T>(v) * static_cast<T>(*own_f(st, 2));
                    }
                }
                dst[q] = v;
            });
    };

    // Level 0, pass 3: p = Z + beta p_old, q = A p; partials (p, q), (p, r). Clears the coarse right-hand sides
    // for the next restriction. Stage fields: own Z p r, halo Z p.
    auto pq_pass = [&](float fb, T& pq, T& pr) {
        const float* po = W.p[cur];
        float* pn = W.p[cur ^ 1];
        const float* r = rb[rc];
        amarch::march<kPlanesInFlight>(
            geom(0), cols(0), ring,
            [&](const amarch::Slots& s, int k, int, bool zok, uint32_t base) {
                float* st = stage(k);
                const SlotCopy o = own_copy(s, zok, base);
                copy_field(own_f(st, 0), Z, o);
                copy_field(own_f(st, 1), po, o);
                copy_field(own_f(st, 2), r, o);
                copy_code(own_code(st), L0.code, o);
                if (s.halo) {
                    const SlotCopy h = halo_copy(s, zok, base);
                    copy_field(halo_f(st, 0), Z, h);
                    copy_field(halo_f(st, 1), po, h);
                }
            },
            [&](const amarch::Slots&, int k, int, uint32_t, bool halo) {
                float* st = stage(k);
                return halo ? *halo_f(st, 0) + fb * *halo_f(st, 1) : *own_f(st, 0) + fb * *own_f(st, 1);
            },
            [&](const amarch::Slots& s, int k, int, uint32_t q, float um1, float u0, float u1, const float* plane, bool) {
                if (!s.oout) return;
                float* st = stage(k);
                const uint16_t code = amarch::code_of(*own_code(st), q);
                const float qv = zstencil(code, u0, um1, u1, plane, s.oslot);
                pn[q] = u0;
                W.q[q] = qv;
                pq += static_cast<T>(u0) * static_cast<T>(qv);
                pr += static_cast<T>(u0) * static_cast<T>(*own_f(st, 2));
            });
        zero_coarse_r();
    };

    // The coarse part of a V-cycle: levels 1 .. coarsest, given L1.r; leaves L1.t.
    auto coarse_cycle = [&]() -> bool {
        for (int l = 1; l < g; ++l) {
            restrict_level(l);
            if (!grid_barrier()) return false;
        }
        mark(1);
        if (blockIdx.x == 0) block_cycle(H, dyn);
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

    // FP64 residual of the accumulated solution into the current residual buffer: r = b - A x64; e = q = 0.
    auto x64_residual = [&](double& rr) {
        rr = 0.0;
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
            const double rv = active(code) ? static_cast<double>(__ldg(b + q)) - ax : 0.0;
            rb[rc][q] = static_cast<float>(rv);
            e[q] = 0.0f;
            W.q[q] = 0.0f;
            rr += rv * rv;
        }
    };

    // ------------------------------------------------------------ setup: r = b (or b - A x64), e = q = p = 0
    T bb = 0, rnorm2 = 0;
    {
        const bool warm = ir && S.warm_start;
        double loc[4] = {0, 0, 0, 0}, tot[4];
        for (uint32_t q = gfirst; q < n; q += gstride) {
            const float bv = __ldg(b + q);
            loc[0] += static_cast<double>(bv) * static_cast<double>(bv);
            W.p[0][q] = 0.0f;
            W.p[1][q] = 0.0f;
            if (!warm) {
                e[q] = 0.0f;
                W.q[q] = 0.0f;
                rb[0][q] = bv;
            }
        }
        if (warm) x64_residual(loc[1]);
        else loc[1] = loc[0];
        zero_coarse_r();
        if (gsync::barrier_allreduce<kThreads, double>(ctl, phase, loc, tot)) {
            bb = static_cast<T>(tot[0]);
            rnorm2 = static_cast<T>(tot[1]);
        } else {
            aborted = true;
        }
    }

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
        T pass_rr0 = rnorm2;
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
            // FP64: x64 += e, r = b - A x64, e = q = 0, coarse r = 0
            const bool fresh = passes == 1 && !S.warm_start;
            for (uint32_t q = gfirst; q < n; q += gstride) W.x64[q] = (fresh ? 0.0 : W.x64[q]) + static_cast<double>(e[q]);
            if (!grid_barrier()) break;
            double dl[4] = {0, 0, 0, 0}, dt[4];
            x64_residual(dl[0]);
            zero_coarse_r();
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

// Operator codes of a coarse level: the fine rules (stencil_code_kernel) without the anchor. The two spare
// entries past the end are zero (inactive).
__global__ void mg_code_kernel(const MgLevel L, const __grid_constant__ StepParams P) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= L.n + 2) return;
    if (q >= L.n) {
        L.code[q] = 0;
        return;
    }
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
    L.code[q] = static_cast<uint16_t>(mask | (diag << 8) | kCodeActive);
}

// Zeroes the two spare entries past the level-0 codes (read as the upper half of the last aligned pair).
__global__ void mg_code_tail_kernel(uint16_t* code, uint32_t n) {
    if (threadIdx.x < 2) code[n + threadIdx.x] = 0;
}

template <typename T>
cudaError_t launch_mg_one(const StepParams& P, const PcgSettings& S, const MgHierarchy& H, const float* b, float* x, MgWork work, PcgControl* ctl, cudaStream_t s) {
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(mgfcg_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kDynSmemBytes));
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mgfcg_kernel<T>, kThreads, kDynSmemBytes);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorLaunchOutOfResources;
        max_blocks = sms * per_sm;
        if (max_blocks > kPcgMaxBlocks) max_blocks = kPcgMaxBlocks;
    }
    // at least ~8 column-planes of level 0 per block
    const uint32_t planes = amarch::columns_of(H.L[0].nx, H.L[0].ny, H.L[0].nz).total;
    uint32_t want = planes / 8u;
    if (want < 1u) want = 1u;
    const int blocks = static_cast<int>(want < static_cast<uint32_t>(max_blocks) ? want : static_cast<uint32_t>(max_blocks));
    cudaError_t e = cudaMemsetAsync(ctl, 0, kPcgControlResetBytes, s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kDynSmemBytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, mgfcg_kernel<T>, P, S, H, b, x, work, ctl);
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
    mg_code_tail_kernel<<<1, 32, 0, s>>>(H.L[0].code, H.L[0].n);
    for (int l = 1; l < H.levels; ++l) {
        mg_coarsen_kernel<<<(H.L[l].n + 255) / 256, 256, 0, s>>>(H.L[l - 1], H.L[l]);
        mg_code_kernel<<<(H.L[l].n + 2 + 255) / 256, 256, 0, s>>>(H.L[l], P);
    }
    return cudaGetLastError();
}

cudaError_t launch_mgfcg(const StepParams& P, const PcgSettings& S, const MgHierarchy& H, const float* b, float* x, MgWork work, PcgControl* ctl, cudaStream_t s) {
    return S.fp64 ? launch_mg_one<double>(P, S, H, b, x, work, ctl, s) : launch_mg_one<float>(P, S, H, b, x, work, ctl, s);
}

}  // namespace smoke_b200
