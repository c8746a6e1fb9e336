// Multigrid-preconditioned flexible conjugate gradients for the pressure system, driven by a CUDA graph.
//
// No reference counterpart: the reference solves with unpreconditioned CG (backend-cuda.cu:1788-1824), which at
// 128^3 needs ~900 iterations and stalls near relative residual 2.5e-5 in FP32. Here the preconditioner is one
// geometric multigrid V(1,1) cycle:
//  - levels: level l+1 halves every extent of level l (rounding up) down to a single cell; a coarse cell is
//    active (fluid) when any child is; each level's operator is the masked 7-point stencil of its active cells,
//    built with the fine rules (periodic wrap, OUTFLOW faces on the diagonal) but without the anchor;
//  - smoothing: damped Jacobi, weight kOmega = 6/7; the pre-smoothing sweep starts from zero;
//  - restriction: r_{l+1}(C) = 1/2 * sum of the residuals of C's (up to 8) children after pre-smoothing; with the
//    trilinear prolongation below this is the Petrov-Galerkin scaling of the 7-point operator (R A P ~ 2 A_coarse);
//  - prolongation: cell-centred trilinear (weights 3/4 and 1/4 per axis); a corner outside the domain or on an
//    inactive coarse cell takes the parent's value (inactive coarse cells carry the bit pattern kTag in t);
//  - the coarsest levels (at most kMgBlockLevelCells cells, kMgBlockBytes in all) run in one block from shared
//    memory, the coarsest one with kCoarsestSweeps Jacobi sweeps in a single warp; every other level pass is one
//    kernel with one thread per cell at full occupancy. Going down to one cell (instead of stopping at 4^3) brings
//    the coarse-grid correction of the smoothest modes close to exact: 14 -> 12 iterations at 128^3 and 16 -> 12 at
//    256^3 on the plume.
// The outer iteration is flexible CG (Notay 2000: beta_k = -(z_k, q_{k-1}) / (p_{k-1}, q_{k-1})), which stays
// valid when the preconditioner is not exactly symmetric. Refinement passes accumulate the solution in FP64 and
// restart from the FP64 residual b - A x64, as in pcg.cu.
//
// Execution: the solve is a graph (enqueue_mg_solve is called while the stream is being captured). Per iteration
// the body of a graph `while` node runs: coarse restrictions, the block-level cycle, coarse prolongation +
// smoothing, level-0 prolongation, level-0 smoothing with (z, r) (z, q), p/q with (p, q) (p, r), and the level-0
// update r -= alpha q, e += alpha p with pre-smoothing, restriction and ||r||^2. The last block of the update
// kernel tests convergence and sets the loop condition (cudaGraphSetConditional), so the host never waits. A learned
// solve's pass has two `while` nodes: the first body runs the network, and its update ends that loop when the next
// iteration goes without it (past the schedule's iterations, or after a fallback); the second body is the V-cycle
// alone, entered when the first loop ended without stopping. So iterations without the network launch none of the
// network's kernels. The network runs on level 1: its input is the restriction of what the V-cycle leaves, and its
// output comes back through the V-cycle's prolongation.
// Dot products: block sums in a fixed order, stored per block in FP64 and added in block order by the last block to
// finish, so the solve is deterministic.
// Each restriction block covers whole 2x2x2 parents and writes the coarse right-hand side directly.
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "launch.h"
#include "pdl.cuh"
#include "unet.h"
#include "smoke_b200_ext.h"

namespace smoke_b200 {

namespace {

constexpr int TX = 32, TY = 4, TZ = 2;  // cells of one block; even extents, so blocks hold whole parents
constexpr int kThreads = TX * TY * TZ;
constexpr int kBlockLevelThreads = 512;
constexpr float kOmega = 6.0f / 7.0f;  // damped Jacobi weight: the optimal smoothing factor of the 7-point Laplacian in 3D
constexpr int kCoarsestSweeps = 16;
constexpr uint32_t kWarpCoarsestCells = 128;  // coarsest levels this small sweep in one warp
// Coarse levels of at most this many cells take the up-pass as one kernel (mg_up_kernel). Its halo recomputes about
// 3x the cells: on 64^3 and smaller levels the saved launch wins (128^3 solve -2.5%); on a 128^3 level it does not.
constexpr uint32_t kFusedUpCells = 64u * 64u * 64u;
constexpr uint32_t kTag = 0x7fc0feedu;  // t of an inactive coarse cell (a NaN payload arithmetic never produces)
constexpr int kMaxPasses = 8;           // refinement passes in the graph (refinement is clamped to kMaxPasses - 1)
// Refined solves: one FP32 pass may reduce ||r|| by at most 1e5 (||r||^2 by 1e10) of its starting residual before
// the FP64 true residual is recomputed. The multigrid FCG takes ~12 iterations, so its FP32 recurrence residual stays
// close to the true one over that range and one pass usually meets 1e-5; a limit of 3.3e3 per pass forced a second
// pass, with its restart, on every solve at 128^3. The FP64 check still adds passes when needed.
constexpr double kPassReduction2 = 1e-10;
// An FP32 pass stops when its recurrence residual reaches a fraction of the tolerance, because the recurrence drifts
// below the true residual as the pass goes on: a pass from ||r0|| = ||b|| (a cold start) ends about 3x below its true
// residual at 1e-5, so it aims at 0.3 tol (squared: 0.09). A pass that starts within 0.5 ||b|| (a warm start from the
// previous step's pressure, about 0.37 ||b|| on the 128^3 plume, or a later refinement pass) drifts at most about
// 1.4x, so 0.7 tol (0.49) still ends below tol: one iteration fewer per warm solve at 128^3. The FP64 check decides
// either way.
__device__ __forceinline__ double pass_target2(double tol2, double rtot, double btot) {
    const double margin2 = rtot <= 0.25 * btot ? 0.49 : 0.09;
    return fmax(margin2 * tol2, kPassReduction2 * rtot);
}

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

// Neighbour e (0..5 = -x +x -y +y -z +z) of an active stencil bit: in range, or across a periodic edge.
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
// diag * v0 - sum of v over the active neighbours of (q; x, y, z); v(index) supplies the values.
template <typename R, class V>
__device__ __forceinline__ R stencil_xyz(const MgLevel& L, uint32_t q, int x, int y, int z, uint16_t code, R v0, V&& v) {
    R acc = static_cast<R>(diagf(code)) * v0;
#pragma unroll
    for (int e = 0; e < 6; ++e)
        if (code & (1u << e)) acc -= v(lnbr(L, q, x, y, z, e));
    return acc;
}

// Masked 7-point stencil from preloaded values: diag * v0 - sum of vn[e] over the code's active neighbour bits.
__device__ __forceinline__ float masked_stencil(uint16_t code, float v0, const float vn[6]) {
    float acc = diagf(code) * v0;
#pragma unroll
    for (int e = 0; e < 6; ++e)
        if (code & (1u << e)) acc -= vn[e];
    return acc;
}

// v in [-1, n]: wraps one step across a periodic edge; false when v is outside a non-periodic axis.
__device__ __forceinline__ bool wrap_c(int& v, int n, int per) {
    if (v < 0) {
        v += n;
        return per != 0;
    }
    if (v >= n) {
        v -= n;
        return per != 0;
    }
    return true;
}


// Trilinear weights of the 8 corners of a fine cell; c(m) loads corner m (bit 0: the x neighbour, bit 1: y, bit 2: z
// of the parent, corner 0). A corner clamped at a wall (w*), or on an inactive coarse cell (kTag), takes the
// parent's value; a corner beyond an OUTFLOW face (o*, where the pressure is held at 0) takes minus the parent's value,
// the linear extrapolation through 0 at the face. With parent values there the correction does not vanish at the
// face, and on scenes with outflow faces the FCG needed half again to twice the iterations of a closed box, more the
// finer the grid (a float64 model of this cycle: 15-24 iterations at 64x80x64 against 10 with the extrapolation).
template <class T>
__device__ __forceinline__ float prolong_corners(bool wx, bool wy, bool wz, bool ox, bool oy, bool oz, T&& c) {
    const float c0 = c(0), c1 = c(1), c2 = c(2), c3 = c(3), c4 = c(4), c5 = c(5), c6 = c(6), c7 = c(7);
    const float parent = is_tag(c0) ? 0.0f : c0;
    auto v = [&](float x, bool wall, bool out) { return out ? -parent : ((wall || is_tag(x)) ? parent : x); };
    // weights (3/4 or 1/4 per axis): 27/64 parent, 9/64 edge, 3/64 face-diagonal, 1/64 opposite corner
    const float near = 0.421875f * parent + 0.140625f * (v(c1, wx, ox) + v(c2, wy, oy) + v(c4, wz, oz));
    const float far = 0.046875f * (v(c3, wx || wy, ox || oy) + v(c5, wx || wz, ox || oz) + v(c6, wy || wz, oy || oz)) + 0.015625f * v(c7, wx || wy || wz, ox || oy || oz);
    return near + far;
}


// ---------------------------------------------------------------------------------------------- block helpers
// Level kernels: one thread per cell of a TX x TY x TZ tile; block (bx, by, bz) walks the tiles (bx, by, k) for k in
// its share of the z range, so that a wave of resident blocks covers the level and z-neighbours come from L1.
struct Cell {
    int x, y, z;     // coordinates
    int bx, by, bz;  // tile
    uint32_t q;
    bool in;
};
__device__ __forceinline__ int tiles_z(const MgLevel& L) { return (L.nz + TZ - 1) / TZ; }
template <class F>
__device__ __forceinline__ void for_tiles(const MgLevel& L, F&& f) {
    const int nzt = tiles_z(L);
    const int share = (nzt + gridDim.z - 1) / gridDim.z;
    const int k0 = blockIdx.z * share, k1 = min(nzt, k0 + share);
    Cell c;
    c.bx = blockIdx.x;
    c.by = blockIdx.y;
    c.x = c.bx * TX + threadIdx.x;
    c.y = c.by * TY + threadIdx.y;
    const bool in_xy = c.x < L.nx && c.y < L.ny;
    for (int k = k0; k < k1; ++k) {
        c.bz = k;
        c.z = k * TZ + threadIdx.z;
        c.in = in_xy && c.z < L.nz;
        c.q = c.in ? lidx(L, c.x, c.y, c.z) : 0u;
        f(c);
    }
}
__device__ __forceinline__ uint32_t block_linear() { return (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x; }
__device__ __forceinline__ uint32_t grid_blocks() { return gridDim.x * gridDim.y * gridDim.z; }
__device__ __forceinline__ int tid() { return (threadIdx.z * TY + threadIdx.y) * TX + threadIdx.x; }

// Indices of the 6 neighbours of an in-domain cell, computed from its coordinates alone (wrapped across periodic
// edges, the cell itself where a non-periodic boundary cuts the stencil), so that every load of a stencil can be
// issued before the operator code arrives; the code's bits then pick the terms.
__device__ __forceinline__ void nbr_all(const MgLevel& L, const int* per, const Cell& c, uint32_t nb[6]) {
    const uint32_t nx = L.nx, slab = nx * L.ny, q = c.q;
    nb[0] = c.x > 0 ? q - 1 : (per[0] ? q + (nx - 1) : q);
    nb[1] = c.x < L.nx - 1 ? q + 1 : (per[0] ? q - (nx - 1) : q);
    nb[2] = c.y > 0 ? q - nx : (per[1] ? q + (L.ny - 1) * nx : q);
    nb[3] = c.y < L.ny - 1 ? q + nx : (per[1] ? q - (L.ny - 1) * nx : q);
    nb[4] = c.z > 0 ? q - slab : (per[2] ? q + (L.nz - 1) * slab : q);
    nb[5] = c.z < L.nz - 1 ? q + slab : (per[2] ? q - (L.nz - 1) * slab : q);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Programmatic dependent launch (pdl.cuh): the iteration's kernels are launched with launch_pdl and begin with
// pdl_begin, so a kernel's launch and block dispatch overlap its predecessor's tail; nothing is read before the wait.

// Block sums of a and b (in a fixed order) stored as this block's partials of accumulators ka and kb (kb < 0: only
// a). Thread 0 writes them.
template <typename T>
__device__ __forceinline__ void block_accumulate(const MgWork& W, int ka, T a, int kb, T b) {
    __shared__ T part[2][kThreads / 32];
    const int t = tid(), lane = t & 31, warp = t >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        part[0][warp] = a;
        part[1][warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        a = warp_sum(lane < kThreads / 32 ? part[0][lane] : T(0));
        b = warp_sum(lane < kThreads / 32 ? part[1][lane] : T(0));
        if (lane == 0) {
            const uint32_t blk = block_linear();
            W.part[static_cast<size_t>(ka) * W.part_stride + blk] = static_cast<double>(a);
            if (kb >= 0) W.part[static_cast<size_t>(kb) * W.part_stride + blk] = static_cast<double>(b);
        }
    }
}

// Last-block election with the totals of accumulators ka and kb (kb < 0: only ka): true in every thread of the block
// that finishes last, after every block's partials are visible to it. The partials are added in a fixed order
// (thread i takes blocks i, i + kThreads, ..., then a fixed tree over lanes and warps), so a solve's scalars do not
// depend on the order in which blocks finish, and every thread of the last block holds the same totals.
__device__ bool last_block_totals(unsigned int* counter, const MgWork& W, int ka, int kb, double& ta, double& tb) {
    __shared__ bool s_last;
    __shared__ double red[2][kThreads / 32];
    __syncthreads();
    if (tid() == 0) {
        __threadfence();
        const unsigned int ticket = atomicAdd(counter, 1u);
        s_last = ticket == grid_blocks() - 1;
        if (s_last) {
            *counter = 0;
            __threadfence();
        }
    }
    __syncthreads();
    if (!s_last) return false;
    const uint32_t nb = grid_blocks();
    const double* pa = W.part + static_cast<size_t>(ka) * W.part_stride;
    const double* pb = W.part + static_cast<size_t>(kb < 0 ? ka : kb) * W.part_stride;
    double a = 0.0, b = 0.0;
    for (uint32_t i = tid(); i < nb; i += kThreads) {
        a += __ldcg(pa + i);
        if (kb >= 0) b += __ldcg(pb + i);
    }
    const int lane = tid() & 31, warp = tid() >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    ta = 0.0;
    tb = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        ta += red[0][w];
        tb += red[1][w];
    }
    return true;
}


// The 2x2x2 child sums of a tile's cells written into the coarse level's right-hand side (whole block calls it).
// Returns the sum in the thread that wrote it, 0 in the others.
__device__ __forceinline__ float restrict_tile(float c, const MgLevel& C, const Cell& cell) {
    __shared__ float sm[TZ][TY][TX];
    sm[threadIdx.z][threadIdx.y][threadIdx.x] = c;
    __syncthreads();
    float written = 0.0f;
    const int t = tid();
    if (t < (TX / 2) * (TY / 2)) {
        const int cx = t % (TX / 2), cy = t / (TX / 2);
        const float s = (sm[0][2 * cy][2 * cx] + sm[0][2 * cy][2 * cx + 1]) + (sm[0][2 * cy + 1][2 * cx] + sm[0][2 * cy + 1][2 * cx + 1]) +
                        (sm[1][2 * cy][2 * cx] + sm[1][2 * cy][2 * cx + 1]) + (sm[1][2 * cy + 1][2 * cx] + sm[1][2 * cy + 1][2 * cx + 1]);
        const int X = cell.bx * (TX / 2) + cx, Y = cell.by * (TY / 2) + cy, Z = cell.bz;
        if (X < C.nx && Y < C.ny && Z < C.nz) {
            C.r[lidx(C, X, Y, Z)] = s;
            written = s;
        }
    }
    __syncthreads();
    return written;
}

// ---------------------------------------------------------------------------------------------- level-0 z-march
// The level-0 passes of an iteration (update, smoothing, p/q) march in z. Level 0 is cut into MX x MY = 32 x 8
// columns; each block owns a balanced range of (column, plane pair) units and walks its column segments in z, two
// planes per unit. Thread (tx, ty) owns one cell of the column plane, and a warp holds two y rows of 16 x cells
// (lanes 0-15 row 2k, lanes 16-31 row 2k + 1), so the 2 x 2 x 2 children of a coarse cell are a lane pair (^1), a
// half-warp pair (^16) and two consecutive planes: the restriction is two shuffles and a register. The value whose
// stencil a pass takes is formed once per cell and plane. The 32 x 8 plane and its 84-cell halo go through a
// three-plane ring in shared memory (the in-plane neighbours); the column's own -z / +z values stay in registers.
// The loads of plane z + 2 are issued before plane z is computed; one __syncthreads per plane.
constexpr int MX = 32, MY = 8, MPX = MX + 2, MPY = MY + 2;
constexpr int kMPlane = MPX * MPY;
constexpr int kMHalo = kMPlane - MX * MY;
static_assert(MX * MY == kThreads && kMHalo <= kThreads, "one column cell per thread, at most one halo slot");

struct MarchUnits {
    int ncx, ncy, nzu;  // columns along x and y, plane pairs along z
    uint32_t total;     // ncx * ncy * nzu
};
__host__ __device__ inline MarchUnits march_units(const MgLevel& L) {
    MarchUnits u;
    u.ncx = (L.nx + MX - 1) / MX;
    u.ncy = (L.ny + MY - 1) / MY;
    u.nzu = (L.nz + 1) / 2;
    u.total = static_cast<uint32_t>(u.ncx) * static_cast<uint32_t>(u.ncy) * static_cast<uint32_t>(u.nzu);
    return u;
}

// A ring slot: the in-plane cell it holds (wrapped across periodic edges), if that cell exists.
struct MSlot {
    int slot;
    uint32_t off;  // y * nx + x of the cell
    bool load;
};
__device__ __forceinline__ MSlot march_slot(const MgLevel& L, const int* per, int x0, int y0, int hx, int hy) {
    MSlot s;
    s.slot = (hy + 1) * MPX + hx + 1;
    int x = x0 + hx, y = y0 + hy;
    bool ok = true;
    if (x < 0 || x >= L.nx) {
        if (per[0]) x = wrapi(x, L.nx);
        else ok = false;
    }
    if (y < 0 || y >= L.ny) {
        if (per[1]) y = wrapi(y, L.ny);
        else ok = false;
    }
    s.load = ok;
    s.off = ok ? static_cast<uint32_t>(y) * static_cast<uint32_t>(L.nx) + static_cast<uint32_t>(x) : 0u;
    return s;
}

// March over this block's units of level L. Per plane z of a segment:
//   lo(ok, q) -> Own, lh(ok, q) -> Halo       loads of the own cell / the halo slot (zeros when !ok)
//   uo(Own), uh(Halo) -> float                 the value whose stencil is taken (into the ring)
//   cell(out, q, Own, um1, u0, u1, plane, slot) -> float
//       the own cell's work at plane z (out: the cell is inside the level; um1 / u1 its -z / +z values, plane the
//       ring plane of z); called by every thread. RESTRICT: its result (0 outside the level) is the cell's residual,
//       summed over the 2 x 2 x 2 children into C.r, in restrict_tile's order.
template <bool RESTRICT, class Own, class Halo, class LO, class LH, class UO, class UH, class CellF>
__device__ __forceinline__ void march0(const MgLevel& L, const int* per, const MgLevel& C, float (*ring)[kMPlane], LO&& lo, LH&& lh, UO&& uo, UH&& uh, CellF&& cell) {
    const MarchUnits U = march_units(L);
    const uint32_t a = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x) * U.total) / gridDim.x);
    const uint32_t b = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x + 1) * U.total) / gridDim.x);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tx = (lane & 15) + 16 * (warp & 1), ty = (lane >> 4) + 2 * (warp >> 1);
    const bool halo = threadIdx.x < kMHalo;
    int hx = 0, hy = 0;
    if (halo) {
        const int h = threadIdx.x;
        if (h < MPX) {
            hx = h - 1;
            hy = -1;
        } else if (h < 2 * MPX) {
            hx = h - MPX - 1;
            hy = MY;
        } else if (h < 2 * MPX + MY) {
            hx = -1;
            hy = h - 2 * MPX;
        } else {
            hx = MX;
            hy = h - 2 * MPX - MY;
        }
    }
    const uint32_t slab = static_cast<uint32_t>(L.nx) * static_cast<uint32_t>(L.ny);
    uint32_t u = a;
    while (u < b) {
        const uint32_t col = u / static_cast<uint32_t>(U.nzu);
        const int zu = static_cast<int>(u - col * static_cast<uint32_t>(U.nzu));
        const int zub = zu + static_cast<int>(min(static_cast<uint32_t>(U.nzu - zu), b - u));
        u += static_cast<uint32_t>(zub - zu);
        const int za = 2 * zu, zb = min(L.nz, 2 * zub);
        const int x0 = static_cast<int>(col % static_cast<uint32_t>(U.ncx)) * MX, y0 = static_cast<int>(col / static_cast<uint32_t>(U.ncx)) * MY;
        const MSlot so = march_slot(L, per, x0, y0, tx, ty);
        const MSlot sh = march_slot(L, per, x0, y0, hx, hy);
        const bool out = x0 + tx < L.nx && y0 + ty < L.ny;
        // plane z's offset (wrapped across a periodic z edge); false outside a non-periodic level
        auto zbase = [&](int z, uint32_t& base) {
            if (z < 0 || z >= L.nz) {
                if (!per[2]) return false;
                z = wrapi(z, L.nz);
            }
            base = static_cast<uint32_t>(z) * slab;
            return true;
        };
        auto fetch = [&](int z, Own& od, Halo& hd, bool with_halo) {
            uint32_t base = 0;
            const bool ok = zbase(z, base);
            od = lo(ok && so.load, base + so.off);
            if (with_halo && halo) hd = lh(ok && sh.load, base + sh.off);
        };
        Own om1, o0, o1, o2;
        Halo hunused, h0, h1, h2;
        fetch(za - 1, om1, hunused, false);
        fetch(za, o0, h0, true);
        fetch(za + 1, o1, h1, true);
        float um1 = uo(om1), u0 = uo(o0);
        ring[za % 3][so.slot] = u0;
        if (halo) ring[za % 3][sh.slot] = uh(h0);
        float pair = 0.0f;
        for (int z = za; z < zb; ++z) {
            if (z + 2 <= zb) fetch(z + 2, o2, h2, true);
            const float u1 = uo(o1);
            ring[(z + 1) % 3][so.slot] = u1;
            if (halo) ring[(z + 1) % 3][sh.slot] = uh(h1);
            __syncthreads();
            const float res = cell(out, static_cast<uint32_t>(z) * slab + so.off, o0, um1, u0, u1, ring[z % 3], so.slot);
            if (RESTRICT) {
                // restrict_tile's association: ((a + b) + c) + d over the x pairs a, b (even plane, rows 2Y, 2Y + 1)
                // and c, d (odd plane); the writer is the even-x lane of row 2Y
                const float xs = res + __shfl_xor_sync(0xffffffffu, res, 1);
                const float other = __shfl_xor_sync(0xffffffffu, xs, 16);
                const bool last = (z & 1) != 0 || z == L.nz - 1;
                if ((z & 1) == 0) pair = xs + other;
                else pair = (pair + xs) + other;
                if (last && (tx & 1) == 0 && (ty & 1) == 0) {
                    const int X = (x0 + tx) >> 1, Y = (y0 + ty) >> 1, Z = z >> 1;
                    if (X < C.nx && Y < C.ny) C.r[lidx(C, X, Y, Z)] = pair;
                }
            }
            um1 = u0;
            u0 = u1;
            o0 = o1;
            o1 = o2;
            h1 = h2;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------- kernels
// Solve set-up on level 0: r = b (or b - A x64 for a warm start), e = q = p = 0; ||b||^2 and ||r0||^2. The last
// block initialises the solve's scalars.
template <typename T>
__global__ void __launch_bounds__(kThreads) mg_setup_kernel(const __grid_constant__ MgSolveArgs A) {
    const MgLevel& L0 = A.H.L[0];
    MgState* st = A.st;
    T bb = 0, rr = 0;
    for_tiles(L0, [&](const Cell& c) {
        if (!c.in) return;
        const float bv = A.b[c.q];
        bb += static_cast<T>(bv) * static_cast<T>(bv);
        A.W.p[0][c.q] = 0.0f;
        A.W.p[1][c.q] = 0.0f;
        A.W.q[c.q] = 0.0f;
        A.e[c.q] = 0.0f;
        if (A.warm) {
            const uint16_t code = L0.code[c.q];
            double rv = 0.0;
            if (active(code)) rv = static_cast<double>(bv) - stencil_xyz<double>(L0, c.q, c.x, c.y, c.z, code, A.W.x64[c.q], [&](uint32_t nb) { return A.W.x64[nb]; });
            else A.W.x64[c.q] = 0.0;  // solid or anchor now (occupancy may have changed): its pressure is 0, as from zero
            A.W.r[0][c.q] = static_cast<float>(rv);
            rr += static_cast<T>(rv * rv);
        } else {
            A.W.r[0][c.q] = bv;
            rr += static_cast<T>(bv) * static_cast<T>(bv);
        }
    });
    block_accumulate<T>(A.W, kAccBB, bb, kAccRR, rr);
    double btot, rtot;
    if (!last_block_totals(&st->done[0], A.W, kAccBB, kAccRR, btot, rtot) || tid() != 0) return;
    st->bb = btot;
    st->rnorm2 = rtot;
    st->pass_rr0 = rtot;
    st->parity = 0;
    st->first_iter = 1;
    st->it = 0;
    st->passes = 1;
    st->alpha = 0.0f;
    st->beta = 0.0f;
    st->status = SMOKE_B200_SOLVE_ITERATION_CAP;
    const double tol2 = static_cast<double>(A.tol) * A.tol * btot;
    st->target2 = A.ir ? pass_target2(tol2, rtot, btot) : tol2;
    if (!(btot > 0.0)) {  // b = 0 (solution 0) or not finite
        st->status = isfinite(btot) ? SMOKE_B200_SOLVE_CONVERGED : SMOKE_B200_SOLVE_NOT_FINITE;
        st->halt = 1;
        st->zero_solution = 1;
        st->rnorm2 = 0.0;
    }
}

// Level-0 update: r' = r - alpha q, e += alpha p, zp = w D^-1 r', restriction of r' - A zp into level 1, ||r'||^2.
// initial = 1: the pass's first round (alpha = 0, no iteration counted). The last block tests convergence, flips
// the buffer parity and sets the loop condition `cond`: continue unless stopped, and (net_loop = 1, the loop of a
// learned solve whose body runs the network) unless the next iteration goes without the network.
// z-march: the ring holds w D^-1 (r - alpha q) of every cell (the pre-smoothed zp on active cells; the stencil's
// mask never reaches the others).
template <typename T, bool LEARNED>
__global__ void __launch_bounds__(kThreads) mg_update_kernel(const __grid_constant__ MgSolveArgs A, int initial, cudaGraphConditionalHandle cond, int in_graph, int net_loop) {
    pdl_begin();
    __shared__ float ring[3][kMPlane];
    const MgLevel& L0 = A.H.L[0];
    MgState* st = A.st;
    const bool skip = st->halt || st->fail;  // uniform over the grid
    const int par = st->parity;
    const float a = initial ? 0.0f : st->alpha;
    T rr = 0;
    if (!skip) {
        const float* r = A.W.r[par];
        float* rn_out = A.W.r[par ^ 1];
        const float* pn = A.W.p[par ^ 1];
        struct Own {
            uint32_t code;
            float r, q, p, e;
        };
        struct Halo {
            uint32_t code;
            float r, q;
        };
        march0<true, Own, Halo>(
            L0, A.H.fper, A.H.L[1], ring,
            [&](bool ok, uint32_t q) {
                Own d{0u, 0.0f, 0.0f, 0.0f, 0.0f};
                if (ok) {
                    d.code = L0.code[q];
                    d.r = r[q];
                    d.q = A.W.q[q];
                    if (!initial) {
                        d.p = pn[q];
                        d.e = A.e[q];
                    }
                }
                return d;
            },
            [&](bool ok, uint32_t q) {
                Halo d{0u, 0.0f, 0.0f};
                if (ok) {
                    d.code = L0.code[q];
                    d.r = r[q];
                    d.q = A.W.q[q];
                }
                return d;
            },
            [&](const Own& d) { return wdiag(static_cast<uint16_t>(d.code)) * (d.r - a * d.q); },
            [&](const Halo& d) { return wdiag(static_cast<uint16_t>(d.code)) * (d.r - a * d.q); },
            [&](bool out, uint32_t q, const Own& d, float um1, float u0, float u1, const float* pl, int s) {
                if (!out) return 0.0f;
                const uint16_t code = static_cast<uint16_t>(d.code);
                const float rn = d.r - a * d.q;
                float zp = 0.0f, res = 0.0f;
                if (active(code)) {
                    zp = u0;
                    const float un[6] = {pl[s - 1], pl[s + 1], pl[s - MPX], pl[s + MPX], um1, u1};
                    res = 0.5f * (rn - masked_stencil(code, zp, un));
                }
                L0.zp[q] = zp;
                rn_out[q] = rn;
                if (!initial) A.e[q] = d.e + a * d.p;
                rr += static_cast<T>(rn) * static_cast<T>(rn);
                return res;
            });
        block_accumulate<T>(A.W, kAccRR, rr, -1, T(0));
    }
    double rn2_total, unused;
    if (!last_block_totals(&st->done[1], A.W, kAccRR, -1, rn2_total, unused) || tid() != 0) return;
    if (st->halt) {
        st->loop = 0;
        if (in_graph) cudaGraphSetConditional(cond, 0);
        return;
    }
    int stop = 0;
    if (st->fail) {
        st->status = st->fail;
        stop = 1;
    } else {
        const double rn2 = rn2_total;
        if (!initial) st->it += 1;
        st->rnorm2 = rn2;
        if (!isfinite(rn2)) {
            st->status = SMOKE_B200_SOLVE_NOT_FINITE;
            stop = 1;
        } else if (rn2 <= st->target2) {
            st->status = SMOKE_B200_SOLVE_CONVERGED;
            stop = 1;
        } else if (st->it >= A.max_iterations) {
            st->status = SMOKE_B200_SOLVE_ITERATION_CAP;
            stop = 1;
        }
    }
    if (!initial) st->first_iter = 0;
    if (LEARNED && !stop && !st->fallback) {  // the V-cycle alone, once the learned solve stagnates
        if (initial) {
            st->stall_it = st->it;
            st->stall_ref = st->rnorm2;
        } else if (st->it - st->stall_it >= kLearnedStallWindow) {
            if (st->rnorm2 > st->stall_ref * kLearnedStallReduction2) st->fallback = 1;
            st->stall_it = st->it;
            st->stall_ref = st->rnorm2;
        }
    }
    if (LEARNED) {  // the next loop body runs the network unless dropped or past the schedule's iterations
        if (initial) st->pass_it0 = st->it;
        st->net_off = (st->fallback || (A.net_iterations > 0 && st->it - st->pass_it0 >= A.net_iterations)) ? 1u : 0u;
    }
    st->parity ^= 1;
    st->loop = stop ? 0u : 1u;
    __threadfence();
    if (in_graph) cudaGraphSetConditional(cond, (stop || (LEARNED && net_loop && st->net_off)) ? 0u : 1u);
}

// The condition of a learned solve's second loop (the V-cycle alone, after the network's iterations): the loop flag
// the last update left.
__global__ void mg_loop_gate_kernel(const MgState* __restrict__ st, cudaGraphConditionalHandle cond) {
    pdl_begin();
    cudaGraphSetConditional(cond, st->loop);
}

// Level l >= 1: zp = w D^-1 r (pre-smoothing from zero), restriction of r - A zp into level l + 1.
__global__ void __launch_bounds__(kThreads) mg_restrict_kernel(const __grid_constant__ MgHierarchy H, int l) {
    pdl_begin();
    const MgLevel& F = H.L[l];
    for_tiles(F, [&](const Cell& c) {
        float res = 0.0f;
        if (c.in) {
            uint32_t nb[6];
            nbr_all(F, H.fper, c, nb);
            const uint16_t code = F.code[c.q];
            const float rv = F.r[c.q];
            float un[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) un[k] = wdiag(F.code[nb[k]]) * F.r[nb[k]];
            float zp = 0.0f;
            if (active(code)) {
                zp = wdiag(code) * rv;
                res = 0.5f * (rv - masked_stencil(code, zp, un));
            }
            F.zp[c.q] = zp;
        }
        restrict_tile(res, H.L[l + 1], c);
    });
}

// The trilinear prolongation from level C into level F = C - 1 at coarse cell c (in range): it loads the 3 x 3 x 3
// coarse neighbourhood once (load(index): the level-C value, kTag on an inactive cell) and hands each of its up to 8
// children to store(fine index, blend of the parent and the 7 corners toward the child; see prolong_corners).
template <class Load, class Store>
__device__ __forceinline__ void prolong_children(const MgLevel& F, const MgLevel& C, const int* fper, const int* fout, const Cell& c, Load&& load, Store&& store) {
    // per axis: index of the neighbour on each side (wrapped on a periodic axis, the cell itself at a wall)
    auto side = [](int v, int n, int per, int d) {
        int s = v + d;
        if (s < 0) s = per ? s + n : v;
        else if (s >= n) s = per ? s - n : v;
        return s;
    };
    const int xs[3] = {side(c.x, C.nx, fper[0], -1), c.x, side(c.x, C.nx, fper[0], 1)};
    const int ys[3] = {side(c.y, C.ny, fper[1], -1), c.y, side(c.y, C.ny, fper[1], 1)};
    const int zs[3] = {side(c.z, C.nz, fper[2], -1), c.z, side(c.z, C.nz, fper[2], 1)};
    float t[3][3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const uint32_t row = (static_cast<uint32_t>(zs[k]) * C.ny + ys[j]) * C.nx;
#pragma unroll
            for (int i = 0; i < 3; ++i) t[k][j][i] = load(row + xs[i]);
        }
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int x = 2 * c.x + dx, y = 2 * c.y + dy, z = 2 * c.z + dz;
                if (x >= F.nx || y >= F.ny || z >= F.nz) continue;
                const int ix = dx ? 2 : 0, iy = dy ? 2 : 0, iz = dz ? 2 : 0;  // the corner side of each axis
                const bool wx = xs[ix] == c.x, wy = ys[iy] == c.y, wz = zs[iz] == c.z;
                const float p = prolong_corners(wx, wy, wz, wx && fout[dx], wy && fout[2 + dy], wz && fout[4 + dz], [&](int m) {
                    return t[(m & 4) ? iz : 1][(m & 2) ? iy : 1][(m & 1) ? ix : 1];
                });
                store(lidx(F, x, y, z), p);
            }
}

// Level l: zp += P(t_{l+1}) on active cells (in place). One thread per coarse cell (X, Y, Z) of level l + 1, which
// writes its up to 8 children (prolong_children).
__global__ void __launch_bounds__(kThreads) mg_prolong_kernel(const __grid_constant__ MgHierarchy H, int l) {
    pdl_begin();
    const MgLevel& F = H.L[l];
    const MgLevel& C = H.L[l + 1];
    for_tiles(C, [&](const Cell& c) {
        if (!c.in) return;
        prolong_children(F, C, H.fper, H.fout, c, [&](uint32_t i) { return C.t[i]; }, [&](uint32_t fq, float p) {
            if (active(F.code[fq])) F.zp[fq] += p;
        });
    });
}

// The learned preconditioner's correction on level 0: out = P(y / s) on active cells, 0 elsewhere, for the network's
// output y on level 1 (s = sqrt(n_1 / norm2), the input scale of net_input_kernel; inactive level-1 cells take the
// parent's value, as in the V-cycle's prolongation). Nothing to do once the solve dropped the network (st->net_off).
__global__ void __launch_bounds__(kThreads) mg_net_prolong_kernel(const __grid_constant__ MgHierarchy H, const MgState* __restrict__ st, const float* __restrict__ y, const double* __restrict__ norm2, float* __restrict__ out) {
    pdl_begin();
    if (st != nullptr && st->net_off) return;  // uniform over the grid
    const MgLevel& F = H.L[0];
    const MgLevel& C = H.L[1];
    const double nn = *norm2;
    const float inv_s = nn > 0.0 ? static_cast<float>(sqrt(nn / static_cast<double>(C.n))) : 0.0f;
    for_tiles(C, [&](const Cell& c) {
        if (!c.in) return;
        prolong_children(F, C, H.fper, H.fout, c, [&](uint32_t i) { return active(C.code[i]) ? y[i] * inv_s : __uint_as_float(kTag); },
                         [&](uint32_t fq, float p) { out[fq] = active(F.code[fq]) ? p : 0.0f; });
    });
}

// The network's input for an initial guess: the 2 x 2 x 2 child sums of b on level 1's zp.
__global__ void __launch_bounds__(kThreads) mg_net_restrict_kernel(const __grid_constant__ MgHierarchy H, const float* __restrict__ b) {
    const MgLevel& F = H.L[0];
    MgLevel C = H.L[1];
    C.r = C.zp;
    for_tiles(F, [&](const Cell& c) { restrict_tile(c.in ? b[c.q] : 0.0f, C, c); });
}

// Level l >= 1 post-smoothing: t = zp + w D^-1 (r - A zp) on active cells, kTag on inactive cells.
__global__ void __launch_bounds__(kThreads) mg_smooth_kernel(const __grid_constant__ MgSolveArgs A, int l) {
    pdl_begin();
    const MgLevel& F = A.H.L[l];
    for_tiles(F, [&](const Cell& c) {
        if (!c.in) return;
        uint32_t nb[6];
        nbr_all(F, A.H.fper, c, nb);
        const uint16_t code = F.code[c.q];
        const float s0 = F.zp[c.q], rv = F.r[c.q];
        float sn[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) sn[k] = F.zp[nb[k]];
        F.t[c.q] = active(code) ? s0 + wdiag(code) * (rv - masked_stencil(code, s0, sn)) : __uint_as_float(kTag);
    });
}

// Level-0 post-smoothing (z-march): z = zp + w D^-1 (r - A zp) on active cells, 0 elsewhere, into t; with DOTS,
// (z, r) and (z, q), and the last block computes beta (0 on a pass's first iteration). DOTS = false (a learned
// solve's iteration with the network): z only; the network's correction and the dot products follow.
template <typename T, bool DOTS>
__global__ void __launch_bounds__(kThreads) mg_smooth0_kernel(const __grid_constant__ MgSolveArgs A) {
    pdl_begin();
    __shared__ float ring[3][kMPlane];
    const MgLevel& F = A.H.L[0];
    MgState* st = A.st;
    const float* r = A.W.r[st->parity];
    T zr = 0, zq = 0;
    struct Own {
        uint32_t code;
        float s, r, q;
    };
    march0<false, Own, float>(
        F, A.H.fper, F, ring,
        [&](bool ok, uint32_t q) {
            Own d{0u, 0.0f, 0.0f, 0.0f};
            if (ok) {
                d.code = F.code[q];
                d.s = F.zp[q];
                d.r = r[q];
                if (DOTS) d.q = A.W.q[q];
            }
            return d;
        },
        [&](bool ok, uint32_t q) { return ok ? F.zp[q] : 0.0f; },
        [&](const Own& d) { return d.s; },
        [&](float v) { return v; },
        [&](bool out, uint32_t q, const Own& d, float um1, float u0, float u1, const float* pl, int s) {
            if (!out) return 0.0f;
            const uint16_t code = static_cast<uint16_t>(d.code);
            float z = 0.0f;
            if (active(code)) {
                const float sn[6] = {pl[s - 1], pl[s + 1], pl[s - MPX], pl[s + MPX], um1, u1};
                z = u0 + wdiag(code) * (d.r - masked_stencil(code, u0, sn));
                if (DOTS) {
                    zr += static_cast<T>(z) * static_cast<T>(d.r);
                    zq += static_cast<T>(z) * static_cast<T>(d.q);
                }
            }
            F.t[q] = z;
            return 0.0f;
        });
    if (!DOTS) return;
    block_accumulate<T>(A.W, kAccZR, zr, kAccZQ, zq);
    double tzr, tzq;
    if (!last_block_totals(&st->done[3], A.W, kAccZR, kAccZQ, tzr, tzq) || tid() != 0) return;
    const double beta = st->first_iter ? 0.0 : -tzq / st->pq_prev;
    if (!isfinite(beta) || !isfinite(tzr)) st->fail = SMOKE_B200_SOLVE_NOT_FINITE;
    st->beta = static_cast<float>(beta);
}

// Level l >= 1 up-pass in one kernel: mg_prolong_kernel(l) followed by mg_smooth_kernel(l), with the same
// arithmetic. Per tile, zp + P(t_{l+1}) is formed for the tile and a one-cell halo in shared memory (every fine cell
// from its own 8 coarse corners, as the prolongation kernel forms each child), then the tile is smoothed from there;
// the prolonged zp is not written back (nothing reads it after the smoothing).
__global__ void __launch_bounds__(kThreads) mg_up_kernel(const __grid_constant__ MgHierarchy H, int l) {
    pdl_begin();
    constexpr int RX = TX + 2, RY = TY + 2, RZ = TZ + 2;
    __shared__ float s_zp[RZ][RY][RX];
    const MgLevel& F = H.L[l];
    const MgLevel& C = H.L[l + 1];
    for_tiles(F, [&](const Cell& c) {
        const int x0 = c.bx * TX - 1, y0 = c.by * TY - 1, z0 = c.bz * TZ - 1;
        for (int idx = tid(); idx < RX * RY * RZ; idx += kThreads) {
            const int rx = idx % RX, ry = (idx / RX) % RY, rz = idx / (RX * RY);
            int x = x0 + rx, y = y0 + ry, z = z0 + rz;
            float v = 0.0f;
            // only cells within one step of the level are neighbours of its cells; wrap_c maps [-1, n]
            if (x <= F.nx && y <= F.ny && z <= F.nz && wrap_c(x, F.nx, H.fper[0]) && wrap_c(y, F.ny, H.fper[1]) && wrap_c(z, F.nz, H.fper[2])) {
                const uint32_t fq = lidx(F, x, y, z);
                v = F.zp[fq];
                if (active(F.code[fq])) {
                    auto side = [](int p, int n, int per, int d) {
                        int s = p + d;
                        if (s < 0) s = per ? s + n : p;
                        else if (s >= n) s = per ? s - n : p;
                        return s;
                    };
                    const int X = x >> 1, Y = y >> 1, Z = z >> 1;
                    const int cx = side(X, C.nx, H.fper[0], (x & 1) ? 1 : -1);
                    const int cy = side(Y, C.ny, H.fper[1], (y & 1) ? 1 : -1);
                    const int cz = side(Z, C.nz, H.fper[2], (z & 1) ? 1 : -1);
                    const bool wx = cx == X, wy = cy == Y, wz = cz == Z;
                    v += prolong_corners(wx, wy, wz, wx && H.fout[x & 1], wy && H.fout[2 + (y & 1)], wz && H.fout[4 + (z & 1)], [&](int m) {
                        return C.t[lidx(C, (m & 1) ? cx : X, (m & 2) ? cy : Y, (m & 4) ? cz : Z)];
                    });
                }
            }
            s_zp[rz][ry][rx] = v;
        }
        __syncthreads();
        if (c.in) {
            const int tx = threadIdx.x + 1, ty = threadIdx.y + 1, tz = threadIdx.z + 1;
            const uint16_t code = F.code[c.q];
            const float s0 = s_zp[tz][ty][tx];
            const float sn[6] = {s_zp[tz][ty][tx - 1], s_zp[tz][ty][tx + 1], s_zp[tz][ty - 1][tx], s_zp[tz][ty + 1][tx], s_zp[tz - 1][ty][tx], s_zp[tz + 1][ty][tx]};
            F.t[c.q] = active(code) ? s0 + wdiag(code) * (F.r[c.q] - masked_stencil(code, s0, sn)) : __uint_as_float(kTag);
        }
        __syncthreads();  // the next tile reuses s_zp
    });
}

// Learned preconditioner, part 1: the residual the V-cycle leaves, r_V = r - A z_V on active cells (z_V = t of level
// 0, just smoothed), into level 0's zp (free after the smoothing), and its 2 x 2 x 2 child sums R r_V on level 1's zp
// (free between V-cycles) with ||R r_V||^2 into st->net_rr: the network runs on level 1, and these are its input and
// its scale. Nothing to do once the solve fell back to the V-cycle alone.
template <typename T>
__global__ void __launch_bounds__(kThreads) mg_net_residual_kernel(const __grid_constant__ MgSolveArgs A) {
    pdl_begin();
    const MgLevel& F = A.H.L[0];
    MgLevel C = A.H.L[1];
    C.r = C.zp;
    MgState* st = A.st;
    if (st->net_off) return;  // uniform over the grid
    const float* r = A.W.r[st->parity];
    T rr = 0;
    for_tiles(F, [&](const Cell& c) {
        float rv_net = 0.0f;
        if (c.in) {
            uint32_t nb[6];
            nbr_all(F, A.H.fper, c, nb);
            const uint16_t code = F.code[c.q];
            const float rv = r[c.q], z0 = F.t[c.q];
            float zn[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) zn[k] = F.t[nb[k]];
            rv_net = active(code) ? rv - masked_stencil(code, z0, zn) : 0.0f;
            F.zp[c.q] = rv_net;
        }
        const float sum = restrict_tile(rv_net, C, c);
        rr += static_cast<T>(sum) * static_cast<T>(sum);
    });
    block_accumulate<T>(A.W, kAccNet, rr, -1, T(0));
    double tnet, unused;
    if (!last_block_totals(&st->done[5], A.W, kAccNet, -1, tnet, unused) || tid() != 0) return;
    st->net_rr = tnet;
}

// Learned preconditioner, part 2: the step along the network's correction N = P(y / s) (on level 0, from
// mg_net_prolong_kernel) that minimises the energy norm of what z_V + gamma N leaves of the error e - z_V (whose
// residual is r_V): gamma = (N, r_V) / (N, A N), 0 when that is not defined. So a network that helps little is scaled
// down instead of being added at full weight. (A z-marching form of this pass measured slower: 18.5 against 16.6 us.)
template <typename T>
__global__ void __launch_bounds__(kThreads) mg_net_gamma_kernel(const __grid_constant__ MgSolveArgs A, const float* __restrict__ N) {
    pdl_begin();
    const MgLevel& F = A.H.L[0];
    MgState* st = A.st;
    if (st->net_off) return;  // uniform over the grid
    T nr = 0, nan_ = 0;
    for_tiles(F, [&](const Cell& c) {
        if (!c.in) return;
        const uint16_t code = F.code[c.q];
        if (!active(code)) return;
        uint32_t nb[6];
        nbr_all(F, A.H.fper, c, nb);
        const float n0 = N[c.q];
        float nn[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) nn[k] = N[nb[k]];
        nr += static_cast<T>(n0) * static_cast<T>(F.zp[c.q]);
        nan_ += static_cast<T>(n0) * static_cast<T>(masked_stencil(code, n0, nn));
    });
    block_accumulate<T>(A.W, kAccNet, nr, kAccNetA, nan_);
    double a, b;
    if (!last_block_totals(&st->done[6], A.W, kAccNet, kAccNetA, a, b) || tid() != 0) return;
    st->net_gamma = (b > 0.0 && isfinite(a) && isfinite(b)) ? a / b : 0.0;
}

// Learned preconditioner, part 3: the network's correction N (level 0), scaled by gamma, added to the V-cycle's z_V
// and post-smoothed by one damped Jacobi step on what it leaves of r_V: z = z_V + gamma N + w D^-1 (r_V - gamma A N)
// on active cells (z = z_V in iterations without the network). The network supplies the smooth part of the
// correction; the Jacobi step removes the rough part of its error (BF16 output, fitting noise and the prolongation),
// which the energy norm the FCG minimises would amplify. Then (z, r) and (z, q), and the last block computes beta (0
// on a pass's first iteration), as level 0's smoothing does for the V-cycle alone. z-march: the ring holds gamma N
// (32 -> 25 us against the per-cell form at 128^3).
template <typename T>
__global__ void __launch_bounds__(kThreads) mg_net_add_kernel(const __grid_constant__ MgSolveArgs A, const float* __restrict__ N) {
    pdl_begin();
    __shared__ float ring[3][kMPlane];
    const MgLevel& F = A.H.L[0];
    MgState* st = A.st;
    const bool use_net = st->net_off == 0;
    const float g = use_net ? static_cast<float>(st->net_gamma) : 0.0f;
    const float* r = A.W.r[st->parity];
    T zr = 0, zq = 0;
    struct Own {
        uint32_t code;
        float n, t, rv, r, q;
    };
    march0<false, Own, float>(
        F, A.H.fper, F, ring,
        [&](bool ok, uint32_t q) {
            Own d{0u, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            if (ok) {
                d.code = F.code[q];
                d.t = F.t[q];
                d.r = r[q];
                d.q = A.W.q[q];
                if (use_net) {
                    d.n = N[q];
                    d.rv = F.zp[q];
                }
            }
            return d;
        },
        [&](bool ok, uint32_t q) { return ok && use_net ? N[q] : 0.0f; },
        [&](const Own& d) { return d.n * g; },
        [&](float v) { return v * g; },
        [&](bool out, uint32_t q, const Own& d, float um1, float u0, float u1, const float* pl, int s) {
            const uint16_t code = static_cast<uint16_t>(d.code);
            if (!out || !active(code)) return 0.0f;  // t stays 0 there
            float z = d.t;
            if (use_net) {
                const float nn[6] = {pl[s - 1], pl[s + 1], pl[s - MPX], pl[s + MPX], um1, u1};
                z += u0 + wdiag(code) * (d.rv - masked_stencil(code, u0, nn));
                F.t[q] = z;
            }
            zr += static_cast<T>(z) * static_cast<T>(d.r);
            zq += static_cast<T>(z) * static_cast<T>(d.q);
            return 0.0f;
        });
    block_accumulate<T>(A.W, kAccZR, zr, kAccZQ, zq);
    double tzr, tzq;
    if (!last_block_totals(&st->done[3], A.W, kAccZR, kAccZQ, tzr, tzq) || tid() != 0) return;
    const double beta = st->first_iter ? 0.0 : -tzq / st->pq_prev;
    if (!isfinite(beta) || !isfinite(tzr)) st->fail = SMOKE_B200_SOLVE_NOT_FINITE;
    st->beta = static_cast<float>(beta);
}

// Initial guess of a learned solve: x64 = the network's estimate on active cells, 0 elsewhere.
__global__ void __launch_bounds__(kThreads) mg_net_guess_kernel(const __grid_constant__ MgSolveArgs A, const float* __restrict__ guess) {
    const MgLevel& F = A.H.L[0];
    for_tiles(F, [&](const Cell& c) {
        if (c.in) A.W.x64[c.q] = active(F.code[c.q]) ? static_cast<double>(guess[c.q]) : 0.0;
    });
}

// p' = z + beta p, q = A p'; (p', q) and (p', r). The last block computes alpha = (p', r) / (p', q). z-march: the
// ring holds p' of every cell.
template <typename T>
__global__ void __launch_bounds__(kThreads) mg_pq_kernel(const __grid_constant__ MgSolveArgs A) {
    pdl_begin();
    __shared__ float ring[3][kMPlane];
    const MgLevel& F = A.H.L[0];
    MgState* st = A.st;
    const bool skip = st->fail;  // uniform over the grid
    const int par = st->parity;
    const float fb = st->beta;
    T pq = 0, pr = 0;
    if (!skip) {
        const float* Z = F.t;
        const float* po = A.W.p[par];
        float* pn = A.W.p[par ^ 1];
        const float* r = A.W.r[par];
        struct Own {
            uint32_t code;
            float z, p, r;
        };
        struct Halo {
            float z, p;
        };
        march0<false, Own, Halo>(
            F, A.H.fper, F, ring,
            [&](bool ok, uint32_t q) {
                Own d{0u, 0.0f, 0.0f, 0.0f};
                if (ok) {
                    d.code = F.code[q];
                    d.z = Z[q];
                    d.p = po[q];
                    d.r = r[q];
                }
                return d;
            },
            [&](bool ok, uint32_t q) {
                Halo d{0.0f, 0.0f};
                if (ok) {
                    d.z = Z[q];
                    d.p = po[q];
                }
                return d;
            },
            [&](const Own& d) { return d.z + fb * d.p; },
            [&](const Halo& d) { return d.z + fb * d.p; },
            [&](bool out, uint32_t q, const Own& d, float um1, float u0, float u1, const float* pl, int s) {
                if (!out) return 0.0f;
                const float pnb[6] = {pl[s - 1], pl[s + 1], pl[s - MPX], pl[s + MPX], um1, u1};
                const float qv = masked_stencil(static_cast<uint16_t>(d.code), u0, pnb);
                pn[q] = u0;
                A.W.q[q] = qv;
                pq += static_cast<T>(u0) * static_cast<T>(qv);
                pr += static_cast<T>(u0) * static_cast<T>(d.r);
                return 0.0f;
            });
        block_accumulate<T>(A.W, kAccPQ, pq, kAccPR, pr);
    }
    double pqt, prt;
    if (!last_block_totals(&st->done[4], A.W, kAccPQ, kAccPR, pqt, prt) || tid() != 0 || skip) return;
    if (!(pqt > 0.0) || !isfinite(prt)) {
        st->fail = isfinite(pqt) ? SMOKE_B200_SOLVE_BREAKDOWN : SMOKE_B200_SOLVE_NOT_FINITE;
        return;
    }
    st->alpha = static_cast<float>(prt / pqt);
    st->pq_prev = pqt;
}

// Block-level part of the V-cycle: the levels of at most kMgBlockLevelCells cells, in one block's shared memory.
template <int THREADS>
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

// Cell q of a block level: its coordinates and the indices of its 6 stencil neighbours (nbr_all's rule).
__device__ __forceinline__ Cell block_cell(const MgLevel& L, const int* per, uint32_t q, uint32_t nb[6]) {
    Cell c;
    lxyz(L, q, c.x, c.y, c.z);
    c.bx = c.by = c.bz = 0;
    c.q = q;
    c.in = true;
    nbr_all(L, per, c, nb);
    return c;
}

// Trilinear prolongation of C.t (shared memory) at fine cell (x, y, z), C's codes marking its active cells: a corner
// beyond an OUTFLOW face takes minus the parent, a corner outside the level or on an inactive coarse cell the parent.
// Every corner's value and code are loaded before any is used; the sum runs over the corners in order.
__device__ __forceinline__ float prolong_codes(const MgLevel& C, const int* fper, const int* fout, int x, int y, int z) {
    const int X = x >> 1, Y = y >> 1, Z = z >> 1;
    const int sx = (x & 1) ? 1 : -1, sy = (y & 1) ? 1 : -1, sz = (z & 1) ? 1 : -1;
    const uint32_t pq = lidx(C, X, Y, Z);
    uint32_t idx[8];
    bool outflow[8], inside[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        int cx = X + ((m & 1) ? sx : 0), cy = Y + ((m & 2) ? sy : 0), cz = Z + ((m & 4) ? sz : 0);
        const bool ox = (m & 1) && (cx < 0 || cx >= C.nx) && fout[sx > 0 ? 1 : 0];
        const bool oy = (m & 2) && (cy < 0 || cy >= C.ny) && fout[sy > 0 ? 3 : 2];
        const bool oz = (m & 4) && (cz < 0 || cz >= C.nz) && fout[sz > 0 ? 5 : 4];
        outflow[m] = ox || oy || oz;
        inside[m] = !outflow[m] && wrap_c(cx, C.nx, fper[0]) && wrap_c(cy, C.ny, fper[1]) && wrap_c(cz, C.nz, fper[2]);
        idx[m] = inside[m] ? lidx(C, cx, cy, cz) : pq;
    }
    float tv[8];
    uint16_t code[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        tv[m] = C.t[idx[m]];
        code[m] = C.code[idx[m]];
    }
    const float parent = tv[0];
    float acc = 0.0f;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const float w = ((m & 1) ? 0.25f : 0.75f) * ((m & 2) ? 0.25f : 0.75f) * ((m & 4) ? 0.25f : 0.75f);
        float v = parent;
        if (m) {
            if (outflow[m]) v = -parent;
            else if (inside[m] && active(code[m])) v = tv[m];
        }
        acc += w * v;
    }
    return acc;
}

// The coarse part of the V-cycle below the grid levels, in one block, one cell per thread on every level (a block
// level has at most kMgBlockLevelCells = kBlockLevelThreads cells): reads r of level g (global), pre-smooths and
// restricts level by level, runs the coarsest Jacobi sweeps, then the up passes, and writes t of level g (kTag on
// inactive cells). The level codes do not change during a solve, so they are copied before the wait for the
// previous kernel. The restriction gathers each coarse cell's children in a fixed order (deterministic sums); every
// stencil issues its 6 neighbour loads before using any.
__global__ void __launch_bounds__(kBlockLevelThreads) mg_block_kernel(const __grid_constant__ MgHierarchy H) {
    extern __shared__ __align__(16) float area[];
    constexpr int NT = kBlockLevelThreads;
    static_assert(NT >= kMgBlockLevelCells, "one thread per cell of a block level");
    const int g = H.grid_levels, lc = H.levels - 1;
    const uint32_t t = threadIdx.x;
    for (int l = g; l <= lc; ++l) {  // codes as aligned pairs (the arrays carry two spare entries)
        const MgLevel S = smem_level<NT>(H, area, l);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(H.L[l].code);
        uint32_t* dst = reinterpret_cast<uint32_t*>(S.code);
        for (uint32_t i = t; i < (S.n + 1) / 2; i += NT) dst[i] = src[i];
    }
    pdl_begin();
    {
        const MgLevel S = smem_level<NT>(H, area, g);
        if (t < S.n) S.r[t] = H.L[g].r[t];
    }
    __syncthreads();
    for (int l = g; l < lc; ++l) {  // down: zp = w D^-1 r, then r of l + 1 = 1/2 sum of the children's r - A zp
        const MgLevel F = smem_level<NT>(H, area, l);
        const MgLevel C = smem_level<NT>(H, area, l + 1);
        uint16_t code = 0;
        float rv = 0.0f, zp = 0.0f;
        if (t < F.n) {
            code = F.code[t];
            rv = F.r[t];
            zp = active(code) ? wdiag(code) * rv : 0.0f;
            F.zp[t] = zp;
        }
        __syncthreads();
        if (t < F.n) {
            uint32_t nb[6];
            block_cell(F, H.fper, t, nb);
            float vn[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) vn[k] = F.zp[nb[k]];
            F.t[t] = active(code) ? 0.5f * (rv - masked_stencil(code, zp, vn)) : 0.0f;  // t is free until the up pass
        }
        __syncthreads();
        if (t < C.n) {
            int X, Y, Z;
            lxyz(C, t, X, Y, Z);
            float v[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const int x = 2 * X + (m & 1), y = 2 * Y + ((m >> 1) & 1), z = 2 * Z + (m >> 2);
                v[m] = (x < F.nx && y < F.ny && z < F.nz) ? F.t[lidx(F, x, y, z)] : 0.0f;
            }
            float sum = 0.0f;
#pragma unroll
            for (int m = 0; m < 8; ++m) sum += v[m];
            C.r[t] = sum;
        }
        __syncthreads();
    }
    {  // coarsest level: Jacobi sweeps from zero, result in t
        const MgLevel L = smem_level<NT>(H, area, lc);
        if (L.n == 1) {  // one cell (its stencil neighbours, across periodic edges, are itself): in registers
            if (t == 0) {
                const uint16_t code = L.code[0];
                const float rv = L.r[0];
                float v = active(code) ? wdiag(code) * rv : 0.0f;
                for (int sweep = 0; sweep < kCoarsestSweeps; ++sweep) {
                    const float vn[6] = {v, v, v, v, v, v};
                    v = active(code) ? v + wdiag(code) * (rv - masked_stencil(code, v, vn)) : 0.0f;
                }
                L.t[0] = v;
            }
        } else {  // ping-pong between t and zp; a level of at most kWarpCoarsestCells cells sweeps in warp 0
            const bool by_warp = L.n <= kWarpCoarsestCells;
            const uint32_t lanes = by_warp ? 32u : static_cast<uint32_t>(NT);
            if (t < lanes) {
                for (uint32_t q = t; q < L.n; q += lanes) {
                    const uint16_t code = L.code[q];
                    L.t[q] = active(code) ? wdiag(code) * L.r[q] : 0.0f;
                }
                for (int sweep = 0; sweep < kCoarsestSweeps; ++sweep) {
                    if (by_warp) __syncwarp();
                    else __syncthreads();
                    float* src = (sweep & 1) ? L.zp : L.t;
                    float* dst = (sweep & 1) ? L.t : L.zp;
                    for (uint32_t q = t; q < L.n; q += lanes) {
                        const uint16_t code = L.code[q];
                        uint32_t nb[6];
                        block_cell(L, H.fper, q, nb);
                        const float s0 = src[q], rv = L.r[q];
                        float vn[6];
#pragma unroll
                        for (int k = 0; k < 6; ++k) vn[k] = src[nb[k]];
                        dst[q] = active(code) ? s0 + wdiag(code) * (rv - masked_stencil(code, s0, vn)) : 0.0f;
                    }
                }
            }
        }
        __syncthreads();
    }
    static_assert(kCoarsestSweeps % 2 == 0, "the coarsest sweeps end in t");
    for (int l = lc - 1; l >= g; --l) {  // up: zp += P(t of l + 1), then t = zp + w D^-1 (r - A zp)
        const MgLevel F = smem_level<NT>(H, area, l);
        const MgLevel C = smem_level<NT>(H, area, l + 1);
        uint16_t code = 0;
        float rv = 0.0f, zp = 0.0f;
        uint32_t nb[6];
        if (t < F.n) {
            code = F.code[t];
            rv = F.r[t];
            zp = F.zp[t];
            const Cell c = block_cell(F, H.fper, t, nb);
            if (active(code)) {
                zp += prolong_codes(C, H.fper, H.fout, c.x, c.y, c.z);
                F.zp[t] = zp;
            }
        }
        __syncthreads();
        if (t < F.n) {
            float vn[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) vn[k] = F.zp[nb[k]];
            F.t[t] = active(code) ? zp + wdiag(code) * (rv - masked_stencil(code, zp, vn)) : 0.0f;
        }
        __syncthreads();
    }
    const MgLevel S = smem_level<NT>(H, area, g);
    if (t < S.n) H.L[g].t[t] = active(S.code[t]) ? S.t[t] : __uint_as_float(kTag);
}

// Standalone V-cycle, level 0 down: zp = w D^-1 r, and (r - A zp) / 2 restricted into level 1 (the pre-smoothing the
// solve's update kernel performs, for an r given by the caller).
__global__ void __launch_bounds__(kThreads) mg_presmooth_kernel(const __grid_constant__ MgHierarchy H, const float* __restrict__ r) {
    const MgLevel& L0 = H.L[0];
    for_tiles(L0, [&](const Cell& c) {
        float res = 0.0f;
        if (c.in) {
            uint32_t nb[6];
            nbr_all(L0, H.fper, c, nb);
            const uint16_t code = L0.code[c.q];
            const float rv = r[c.q];
            float un[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) un[k] = wdiag(L0.code[nb[k]]) * r[nb[k]];
            float zp = 0.0f;
            if (active(code)) {
                zp = wdiag(code) * rv;
                res = 0.5f * (rv - masked_stencil(code, zp, un));
            }
            L0.zp[c.q] = zp;
        }
        restrict_tile(res, H.L[1], c);
    });
}

// Standalone V-cycle, level 0 up: z = zp + w D^-1 (r - A zp) on active cells, 0 elsewhere.
__global__ void __launch_bounds__(kThreads) mg_postsmooth_kernel(const __grid_constant__ MgHierarchy H, const float* __restrict__ r, float* __restrict__ z) {
    const MgLevel& F = H.L[0];
    for_tiles(F, [&](const Cell& c) {
        if (!c.in) return;
        uint32_t nb[6];
        nbr_all(F, H.fper, c, nb);
        const uint16_t code = F.code[c.q];
        const float s0 = F.zp[c.q];
        float sn[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) sn[k] = F.zp[nb[k]];
        z[c.q] = active(code) ? s0 + wdiag(code) * (r[c.q] - masked_stencil(code, s0, sn)) : 0.0f;
    });
}

// Refinement: x64 = (first pass of a cold start ? 0 : x64) + e.
__global__ void __launch_bounds__(kThreads) mg_accumulate_kernel(const __grid_constant__ MgSolveArgs A) {
    pdl_begin();
    const MgState* st = A.st;
    if (st->halt) return;
    const bool fresh = st->passes == 1 && !A.warm;
    const MgLevel& L0 = A.H.L[0];
    for_tiles(L0, [&](const Cell& c) {
        if (c.in) A.W.x64[c.q] = (fresh ? 0.0 : A.W.x64[c.q]) + static_cast<double>(A.e[c.q]);
    });
}

// Refinement: r = b - A x64 (FP64) into the current residual buffer, e = q = 0, ||r||^2. The last block decides
// between another pass and the end of the solve.
__global__ void __launch_bounds__(kThreads) mg_residual_kernel(const __grid_constant__ MgSolveArgs A) {
    pdl_begin();
    const MgLevel& L0 = A.H.L[0];
    MgState* st = A.st;
    if (st->halt) return;  // uniform: no block reaches the election
    float* r = A.W.r[st->parity];
    double rr = 0.0;
    for_tiles(L0, [&](const Cell& c) {
        if (!c.in) return;
        const uint16_t code = L0.code[c.q];
        double rv = 0.0;
        if (active(code)) rv = static_cast<double>(A.b[c.q]) - stencil_xyz<double>(L0, c.q, c.x, c.y, c.z, code, A.W.x64[c.q], [&](uint32_t nb) { return A.W.x64[nb]; });
        r[c.q] = static_cast<float>(rv);
        A.e[c.q] = 0.0f;
        A.W.q[c.q] = 0.0f;
        rr += rv * rv;
    });
    block_accumulate<double>(A.W, kAccRR, rr, -1, 0.0);
    double rtot, unused;
    if (!last_block_totals(&st->done[2], A.W, kAccRR, -1, rtot, unused) || tid() != 0) return;
    const double true_rel = sqrt(rtot / st->bb);
    st->true_rel = true_rel;
    if (true_rel <= static_cast<double>(A.tol)) {
        st->status = SMOKE_B200_SOLVE_CONVERGED;
        st->halt = 1;
    } else if (st->passes > A.refinement || st->it >= A.max_iterations || st->status != SMOKE_B200_SOLVE_CONVERGED) {
        if (st->status == SMOKE_B200_SOLVE_CONVERGED) st->status = SMOKE_B200_SOLVE_ITERATION_CAP;
        st->halt = 1;
    } else {
        st->passes += 1;
        st->rnorm2 = rtot;
        st->pass_rr0 = rtot;
        const double tol2 = static_cast<double>(A.tol) * A.tol * st->bb;
        st->target2 = pass_target2(tol2, rtot, st->bb);
        st->first_iter = 1;
        st->status = SMOKE_B200_SOLVE_ITERATION_CAP;
    }
}

// Solution write-back and status record.
__global__ void __launch_bounds__(kThreads) mg_finalize_kernel(const __grid_constant__ MgSolveArgs A, PcgStatusDevice* out) {
    pdl_begin();
    const MgState* st = A.st;
    const MgLevel& L0 = A.H.L[0];
    if (st->zero_solution || A.ir) {
        for_tiles(L0, [&](const Cell& c) {
            if (!c.in) return;
            if (st->zero_solution) {
                A.x[c.q] = 0.0f;
                if (A.ir) A.W.x64[c.q] = 0.0;
            } else {
                A.x[c.q] = static_cast<float>(A.W.x64[c.q]);
            }
        });
    }
    if (block_linear() != 0 || tid() != 0) return;
    PcgStatusDevice s{};
    s.iterations = st->it;
    s.flags = st->fallback ? 1u : 0u;
    s.passes = st->passes;
    s.status = st->status;
    s.rhs_norm = sqrt(st->bb);
    s.relative_residual = st->bb > 0.0 ? sqrt(st->rnorm2 / st->bb) : 0.0;
    s.true_relative_residual = A.ir ? (st->zero_solution ? 0.0 : st->true_rel) : -1.0;
    *out = s;
}

// out = A x with the level-0 operator (identity rows at solid cells and the anchor).
__global__ void __launch_bounds__(kThreads) mg_apply_kernel(const __grid_constant__ MgHierarchy H, const float* __restrict__ x, float* __restrict__ out) {
    const MgLevel& L = H.L[0];
    for_tiles(L, [&](const Cell& c) {
        if (!c.in) return;
        uint32_t nb[6];
        nbr_all(L, H.fper, c, nb);
        float v[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = x[nb[k]];
        out[c.q] = masked_stencil(L.code[c.q], x[c.q], v);
    });
}

// ---------------------------------------------------------------------------------------------- host side
const dim3 kBlock(TX, TY, TZ);

// Grid for `kernel` on level L: the level's tile columns (x, y), and as many z shares as `depth` waves of resident
// blocks (per SM x SMs, cached per kernel and device) allow: depth code 0..3 = 1/2, 1, 2, 4 waves, 4 = one z tile
// per block.
// Blocks of `kernel` (kThreads each) resident on the device at once (SMs x blocks per SM), cached per kernel and
// device.
template <class K>
int resident_blocks(K kernel) {
    static std::mutex lock;
    static std::map<std::pair<const void*, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> guard(lock);
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
    auto it = cache.find(key);
    if (it == cache.end()) {
        int sms = 0, per_sm = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
        it = cache.emplace(key, sms * per_sm).first;
    }
    return it->second;
}

template <class K>
dim3 wave(K kernel, const MgLevel& L, int depth) {
    const int resident = resident_blocks(kernel);
    const int tx = (L.nx + TX - 1) / TX, ty = (L.ny + TY - 1) / TY, tz = (L.nz + TZ - 1) / TZ;
    if (depth >= kMgWaveCount - 1) return dim3(tx, ty, tz);
    const long long blocks = depth <= 0 ? resident / 2 : static_cast<long long>(resident) << (depth - 1);
    int gz = static_cast<int>(std::min<long long>(blocks / (tx * ty), tz));
    if (gz < 1) gz = 1;
    if (gz > tz) gz = tz;
    gz = (tz + ((tz + gz - 1) / gz) - 1) / ((tz + gz - 1) / gz);  // no empty z shares
    return dim3(tx, ty, gz);
}

// Grid of a level-0 z-march kernel: the same depth codes over its (column, plane pair) units (4 = one unit per
// block).
template <class K>
unsigned march_grid(K kernel, const MgLevel& L, int depth) {
    const long long units = march_units(L).total;
    long long blocks = units;
    if (depth < kMgWaveCount - 1) {
        const int resident = resident_blocks(kernel);
        blocks = depth <= 0 ? resident / 2 : static_cast<long long>(resident) << (depth - 1);
    }
    return static_cast<unsigned>(std::max<long long>(1, std::min(blocks, units)));
}

// Adds a `while` node after the capture's current dependencies and captures `body` into it on `body_stream`.
template <class Body>
cudaError_t add_while(cudaStream_t s, cudaStream_t body_stream, cudaGraphConditionalHandle h, Body&& body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, graph, deps, ndeps, &np);
    if (e != cudaSuccess) return e;
    e = cudaStreamBeginCaptureToGraph(body_stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    body(body_stream);
    cudaGraph_t captured = nullptr;
    const cudaError_t eb = cudaGetLastError();
    e = cudaStreamEndCapture(body_stream, &captured);
    if (eb != cudaSuccess) return eb;
    if (e != cudaSuccess) return e;
    return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

// The level-0 update of the solve's preconditioner kind.
template <typename T>
void launch_update(const MgSolveArgs& A, int initial, cudaGraphConditionalHandle h, int in_graph, int net_loop, cudaStream_t s) {
    if (A.learned) launch_pdl(mg_update_kernel<T, true>, march_grid(mg_update_kernel<T, true>, A.H.L[0], A.wave), kThreads, 0, s, A, initial, h, in_graph, net_loop);
    else launch_pdl(mg_update_kernel<T, false>, march_grid(mg_update_kernel<T, false>, A.H.L[0], A.wave), kThreads, 0, s, A, initial, h, in_graph, 0);
}

// The V-cycle below level 0: restrictions of levels 1..g-1, the block-level cycle, the up passes of levels g-1..1,
// then the prolongation into level 0's zp (level 1's right-hand side must be in place).
void launch_coarse_cycle(const MgSolveArgs& A, uint32_t block_bytes, cudaStream_t bs) {
    const MgHierarchy& H = A.H;
    const int g = H.grid_levels;
    for (int l = 1; l < g; ++l) launch_pdl(mg_restrict_kernel, wave(mg_restrict_kernel, H.L[l], A.wave), kBlock, 0, bs, H, l);
    launch_pdl(mg_block_kernel, 1, kBlockLevelThreads, block_bytes, bs, H);
    for (int l = g - 1; l >= 1; --l) {
        if (H.L[l].n <= kFusedUpCells) {
            launch_pdl(mg_up_kernel, wave(mg_up_kernel, H.L[l], A.wave), kBlock, 0, bs, H, l);
        } else {
            launch_pdl(mg_prolong_kernel, wave(mg_prolong_kernel, H.L[l + 1], A.wave), kBlock, 0, bs, H, l);
            launch_pdl(mg_smooth_kernel, wave(mg_smooth_kernel, H.L[l], A.wave), kBlock, 0, bs, A, l);
        }
    }
    launch_pdl(mg_prolong_kernel, wave(mg_prolong_kernel, H.L[1], A.wave), kBlock, 0, bs, H, 0);
}

// One iteration's loop body (everything after the update that tests convergence, up to the next update); net = 1:
// a learned solve's iteration with the network, net = 0: the V-cycle alone (a learned solve's iterations past its
// schedule or after it dropped the network run this body, with the learned solve's update).
template <typename T>
void launch_body(const MgSolveArgs& A, int net, cudaGraphConditionalHandle h, int in_graph, uint32_t block_bytes, cudaStream_t bs) {
    const MgLevel& L0 = A.H.L[0];
    launch_coarse_cycle(A, block_bytes, bs);
    if (net) {  // z = z_V + N(r - A z_V), post-smoothed: the network corrects what the V-cycle leaves
        const LearnedSolve& N = *A.net;
        launch_pdl(mg_smooth0_kernel<T, false>, march_grid(mg_smooth0_kernel<T, false>, L0, A.wave), kThreads, 0, bs, A);
        launch_pdl(mg_net_residual_kernel<T>, wave(mg_net_residual_kernel<T>, L0, A.wave), kBlock, 0, bs, A);
        if (net_forward(N.images, N.acts, A.H.L[1].zp, nullptr, nullptr, &A.st->net_rr, N.occupancy, bs, &A.st->net_off) != cudaSuccess) return;
        launch_pdl(mg_net_prolong_kernel, wave(mg_net_prolong_kernel, A.H.L[1], A.wave), kBlock, 0, bs, A.H, A.st, N.acts.y, &A.st->net_rr, N.fine);
        launch_pdl(mg_net_gamma_kernel<T>, wave(mg_net_gamma_kernel<T>, L0, A.wave), kBlock, 0, bs, A, N.fine);
        launch_pdl(mg_net_add_kernel<T>, march_grid(mg_net_add_kernel<T>, L0, A.wave), kThreads, 0, bs, A, N.fine);
        launch_pdl(mg_pq_kernel<T>, march_grid(mg_pq_kernel<T>, L0, A.wave), kThreads, 0, bs, A);
        launch_pdl(mg_update_kernel<T, true>, march_grid(mg_update_kernel<T, true>, L0, A.wave), kThreads, 0, bs, A, 0, h, in_graph, 1);
        return;
    }
    launch_pdl(mg_smooth0_kernel<T, true>, march_grid(mg_smooth0_kernel<T, true>, L0, A.wave), kThreads, 0, bs, A);
    launch_pdl(mg_pq_kernel<T>, march_grid(mg_pq_kernel<T>, L0, A.wave), kThreads, 0, bs, A);
    launch_update<T>(A, 0, h, in_graph, 0, bs);
}

// Learned solve with the network's warm start: x64 = P(N(R b)) (the network on level 1, its output prolonged to level
// 0), so the set-up's warm path starts from r = b - A x64.
cudaError_t learned_guess(const MgSolveArgs& A, cudaStream_t s) {
    if (!A.learned || !A.net_warm) return cudaSuccess;
    const LearnedSolve& N = *A.net;
    mg_net_restrict_kernel<<<wave(mg_net_restrict_kernel, A.H.L[0], A.wave), kBlock, 0, s>>>(A.H, A.b);
    cudaError_t e = net_forward(N.images, N.acts, A.H.L[1].zp, nullptr, nullptr, nullptr, N.occupancy, s);
    if (e != cudaSuccess) return e;
    mg_net_prolong_kernel<<<wave(mg_net_prolong_kernel, A.H.L[1], A.wave), kBlock, 0, s>>>(A.H, nullptr, N.acts.y, N.acts.norm2, N.fine);
    mg_net_guess_kernel<<<wave(mg_net_guess_kernel, A.H.L[0], A.wave), kBlock, 0, s>>>(A, N.fine);
    return cudaGetLastError();
}

uint32_t block_level_bytes(const MgHierarchy& H) {
    uint32_t bytes = 0;
    for (int l = H.grid_levels; l < H.levels; ++l) bytes += 4u * mg_block_words(H.L[l].n);
    return bytes;
}

template <typename T>
cudaError_t enqueue_typed(const MgSolveArgs& A, PcgStatusDevice* out, cudaStream_t s, cudaStream_t body_stream) {
    const MgLevel& L0 = A.H.L[0];
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureImplicit;
    const uint32_t block_bytes = block_level_bytes(A.H);
    e = cudaMemsetAsync(A.st, 0, sizeof(MgState), s);
    if (e != cudaSuccess) return e;
    if ((e = learned_guess(A, s)) != cudaSuccess) return e;
    mg_setup_kernel<T><<<wave(mg_setup_kernel<T>, L0, A.wave), kBlock, 0, s>>>(A);
    const int passes = A.ir ? A.refinement + 1 : 1;
    for (int pass = 0; pass < passes; ++pass) {
        cudaGraphConditionalHandle h;
        e = cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) return e;
        launch_update<T>(A, 1, h, 1, A.learned, s);
        e = add_while(s, body_stream, h, [&](cudaStream_t bs) { launch_body<T>(A, A.learned, h, 1, block_bytes, bs); });
        if (e != cudaSuccess) return e;
        if (A.learned) {  // then the V-cycle alone, for the iterations past the schedule or after a fallback
            cudaGraphConditionalHandle h2;
            e = cudaGraphConditionalHandleCreate(&h2, graph, 0, cudaGraphCondAssignDefault);
            if (e != cudaSuccess) return e;
            launch_pdl(mg_loop_gate_kernel, 1, 1, 0, s, A.st, h2);
            e = add_while(s, body_stream, h2, [&](cudaStream_t bs) { launch_body<T>(A, 0, h2, 1, block_bytes, bs); });
            if (e != cudaSuccess) return e;
        }
        if (A.ir) {
            launch_pdl(mg_accumulate_kernel, wave(mg_accumulate_kernel, L0, A.wave), kBlock, 0, s, A);
            launch_pdl(mg_residual_kernel, wave(mg_residual_kernel, L0, A.wave), kBlock, 0, s, A);
        }
    }
    launch_pdl(mg_finalize_kernel, wave(mg_finalize_kernel, L0, A.wave), kBlock, 0, s, A, out);
    return cudaGetLastError();
}

template <typename T>
cudaError_t run_typed(const MgSolveArgs& A, PcgStatusDevice* out, cudaStream_t s) {
    const MgLevel& L0 = A.H.L[0];
    const uint32_t block_bytes = block_level_bytes(A.H);
    cudaError_t e = cudaMemsetAsync(A.st, 0, sizeof(MgState), s);
    if (e != cudaSuccess) return e;
    if ((e = learned_guess(A, s)) != cudaSuccess) return e;
    mg_setup_kernel<T><<<wave(mg_setup_kernel<T>, L0, A.wave), kBlock, 0, s>>>(A);
    const int passes = A.ir ? A.refinement + 1 : 1;
    auto loop_flags = [&](uint32_t& flag, uint32_t& net_off) {
        cudaError_t r = cudaMemcpyAsync(&flag, &A.st->loop, sizeof(flag), cudaMemcpyDeviceToHost, s);
        if (r == cudaSuccess) r = cudaMemcpyAsync(&net_off, &A.st->net_off, sizeof(net_off), cudaMemcpyDeviceToHost, s);
        return r == cudaSuccess ? cudaStreamSynchronize(s) : r;
    };
    for (int pass = 0; pass < passes; ++pass) {
        launch_update<T>(A, 1, 0, 0, 0, s);
        for (;;) {  // bounded: every update counts an iteration and stops at max_iterations
            uint32_t flag = 0, net_off = 1;
            if ((e = loop_flags(flag, net_off)) != cudaSuccess) return e;
            if (!flag) break;
            launch_body<T>(A, A.learned && !net_off, 0, 0, block_bytes, s);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (A.ir) {
            launch_pdl(mg_accumulate_kernel, wave(mg_accumulate_kernel, L0, A.wave), kBlock, 0, s, A);
            launch_pdl(mg_residual_kernel, wave(mg_residual_kernel, L0, A.wave), kBlock, 0, s, A);
        }
    }
    launch_pdl(mg_finalize_kernel, wave(mg_finalize_kernel, L0, A.wave), kBlock, 0, s, A, out);
    return cudaGetLastError();
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

// Operator codes of a coarse level: the fine rules (stencil_code_kernel) without the anchor, except on periodic axes
// of one or two cells (below). The two spare entries past the end are zero (inactive).
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
        // A periodic axis that coarsened to one cell couples a cell to itself (no term: p - 2p + p = 0); one of two
        // cells couples the pair once (p - p_other). Counting those on the diagonal, as the fine level's rules do,
        // would add a mass term to the coarse operator and damp its correction of the smoothest modes.
        if (nb == q) continue;
        if ((e & 1) && nn[a] == 2 && P.fper[a]) continue;
        ++diag;
        mask |= 1u << e;
    }
    if (diag == 0) diag = 1;
    L.code[q] = static_cast<uint16_t>(mask | (diag << 8) | kCodeActive);
}

// Zeroes the two spare entries past the level-0 codes.
__global__ void mg_code_tail_kernel(uint16_t* code, uint32_t n) {
    if (threadIdx.x < 2) code[n + threadIdx.x] = 0;
}

}  // namespace

uint32_t mg_partial_blocks(int nx, int ny, int nz) {
    return static_cast<uint32_t>((nx + TX - 1) / TX) * static_cast<uint32_t>((ny + TY - 1) / TY) * static_cast<uint32_t>((nz + TZ - 1) / TZ);
}

int mg_level_count(int nx, int ny, int nz) {
    int levels = 1;
    while ((nx > 1 || ny > 1 || nz > 1) && levels < kMgMaxLevels) {  // down to a single cell
        nx = (nx + 1) / 2;
        ny = (ny + 1) / 2;
        nz = (nz + 1) / 2;
        ++levels;
    }
    return levels < 2 ? 2 : levels;
}

int mg_max_refinement() { return kMaxPasses - 1; }

// solid[q] = 1 where level-1 cell q has no fluid child (the learned preconditioner network's mask on that level).
__global__ void mg_net_mask_kernel(uint32_t n, const uint8_t* __restrict__ fluid, uint8_t* __restrict__ solid) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) solid[q] = fluid[q] ? 0 : 1;
}

cudaError_t launch_mg_net_mask(const MgHierarchy& H, uint8_t* solid, cudaStream_t s) {
    mg_net_mask_kernel<<<(H.L[1].n + 255) / 256, 256, 0, s>>>(H.L[1].n, H.L[1].fluid, solid);
    return cudaGetLastError();
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

cudaError_t launch_mg_apply(const MgHierarchy& H, const float* x, float* out, cudaStream_t s) {
    mg_apply_kernel<<<wave(mg_apply_kernel, H.L[0], kMgWaveDefault), kBlock, 0, s>>>(H, x, out);
    return cudaGetLastError();
}

cudaError_t launch_mg_vcycle(const MgHierarchy& H, int wave_depth, const float* r, float* z, cudaStream_t s) {
    MgSolveArgs A{};
    A.H = H;
    A.wave = wave_depth;
    mg_presmooth_kernel<<<wave(mg_presmooth_kernel, H.L[0], wave_depth), kBlock, 0, s>>>(H, r);
    launch_coarse_cycle(A, block_level_bytes(H), s);
    mg_postsmooth_kernel<<<wave(mg_postsmooth_kernel, H.L[0], wave_depth), kBlock, 0, s>>>(H, r, z);
    return cudaGetLastError();
}

cudaError_t enqueue_mg_solve(const MgSolveArgs& args, bool fp64, PcgStatusDevice* status_out, cudaStream_t s, cudaStream_t body_stream) {
    return fp64 ? enqueue_typed<double>(args, status_out, s, body_stream) : enqueue_typed<float>(args, status_out, s, body_stream);
}

cudaError_t run_mg_solve_eager(const MgSolveArgs& args, bool fp64, PcgStatusDevice* status_out, cudaStream_t s) {
    return fp64 ? run_typed<double>(args, status_out, s) : run_typed<float>(args, status_out, s);
}

}  // namespace smoke_b200
