// Step kernels of the B200 smoke library (everything except the pressure solve, which is in pcg.cu).
//
// Reference behaviour: backend-cuda.cu:840-1609 and the step order of :2000-2057. Design differences:
//  - every face kernel produces the SETTLED face value in one pass: the reference's update kernel, its three
//    enforce_*_boundaries passes and its periodic sync become one read-only-input kernel writing a separate
//    output buffer (no in-place races, no D2D copies). A non-periodic domain face copies the settled value of
//    its interior neighbour for OUTFLOW (backend-cuda.cu:1023-1024), a face touching a solid cell takes the
//    mean solid velocity (:1036-1063), and face n of a periodic axis equals face 0 (:1170-1189);
//  - the three face axes run in one launch (block ranges per axis);
//  - temperature and density share one back-trace per cell;
//  - the density fill of solid cells is a precomputed (cell, nearest fluid cell) list built when occupancy
//    changes, instead of a per-step Chebyshev-shell search (:1243-1290).
#include <cmath>

#include "launch.h"
#include "pdl.cuh"

namespace smoke_b200 {

namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(uint64_t count, int threads = kThreads) { return static_cast<unsigned>((count + threads - 1) / threads); }

// Flow-resolved cell lookup: wraps periodic axes, false when outside a non-periodic domain (:146-151).
__device__ __forceinline__ bool resolve_flow(const StepParams& P, int& x, int& y, int& z) {
    if (P.fper[0]) x = wrapi(x, P.nx);
    if (P.fper[1]) y = wrapi(y, P.ny);
    if (P.fper[2]) z = wrapi(z, P.nz);
    return x >= 0 && x < P.nx && y >= 0 && y < P.ny && z >= 0 && z < P.nz;
}

// Mean solid velocity of the solid cells on either side of face (i,j,k) of axis A, if any (:1036-1063).
template <int A>
__device__ __forceinline__ bool solid_face(const StepParams& P, int i, int j, int k, const uint8_t* __restrict__ occ, const float* __restrict__ solid, float& out) {
    int l[3] = {i, j, k};
    int r[3] = {i, j, k};
    l[A] -= 1;
    const bool hl = resolve_flow(P, l[0], l[1], l[2]);
    const bool hr = resolve_flow(P, r[0], r[1], r[2]);
    const uint32_t li = hl ? cidx(P, l[0], l[1], l[2]) : 0u;
    const uint32_t ri = hr ? cidx(P, r[0], r[1], r[2]) : 0u;
    const bool ol = hl && occ[li] != 0;
    const bool orr = hr && occ[ri] != 0;
    if (!ol && !orr) return false;
    float value = 0.0f, weight = 0.0f;
    if (ol) {
        value += solid[li];
        weight += 1.0f;
    }
    if (orr) {
        value += solid[ri];
        weight += 1.0f;
    }
    out = value / weight;
    return true;
}

// Settled value of face (i,j,k) of axis A: domain-face rule, periodic duplicate, solid rule, else the
// stage's own interior value `inner(i,j,k)`.
// An OUTFLOW domain face copies its interior neighbour. In the reference that copy and the neighbour's solid rule
// run in the same enforce kernel and the copy reads first (observed on B200, :1023-1024 vs :1036-1063), so after
// the force and advection stages the copy does NOT see the neighbour's solid rule. The projection kernel applies
// the solid rule itself before its enforce pass (:1465-1475), so there the copy does see it: OUTFLOW_SEES_SOLID.
template <int A, bool OUTFLOW_SEES_SOLID, class Inner>
__device__ __forceinline__ float settle(const StepParams& P, int i, int j, int k, const uint8_t* __restrict__ occ, const float* __restrict__ solid, Inner&& inner) {
    int c[3] = {i, j, k};
    const int n = axis_n(P, A);
    const SmokeSimulationFlowBoundaryFaceDesc lo = P.flow[2 * A], hi = P.flow[2 * A + 1];
    bool outflow_copy = false;
    if (!P.fper[A]) {
        if (c[A] == 0) {
            if (!(lo.type == kFlowOutflow && n > 0)) return face_comp(lo, A);
            c[A] = 1;
            outflow_copy = true;
        } else if (c[A] == n) {
            if (hi.type != kFlowOutflow) return face_comp(hi, A);
            c[A] = n - 1;
            outflow_copy = true;
        }
    } else if (c[A] == n) {
        c[A] = 0;
    }
    // an index that is itself a domain face (possible only when n == 1) takes no solid rule
    const bool domain_index = !P.fper[A] && (c[A] == 0 || c[A] == n);
    float v;
    if ((OUTFLOW_SEES_SOLID || !outflow_copy) && !domain_index && solid_face<A>(P, c[0], c[1], c[2], occ, solid, v)) return v;
    return inner(c[0], c[1], c[2]);
}

template <int A>
__device__ __forceinline__ const float* pick(const float* a, const float* b, const float* c) {
    return A == 0 ? a : (A == 1 ? b : c);
}
template <int A>
__device__ __forceinline__ float* pick(float* a, float* b, float* c) {
    return A == 0 ? a : (A == 1 ? b : c);
}

// Index of element (i, j, k) of a field of kind KIND (0-2 faces, 3-4 cells) in its padded copy (see PadField).
template <int KIND>
__device__ __forceinline__ uint32_t pad_index(const StepParams& P, int i, int j, int k) {
    const uint32_t px = P.nx + (KIND == 0) + 2 * kPad, py = P.ny + (KIND == 1) + 2 * kPad;
    return (static_cast<uint32_t>(k + kPad) * py + static_cast<uint32_t>(j + kPad)) * px + static_cast<uint32_t>(i + kPad);
}

// ------------------------------------------------------------------------------------------ forces
__global__ void __launch_bounds__(kThreads) vorticity_kernel(const __grid_constant__ StepParams P, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w, const uint8_t* __restrict__ occ, float* __restrict__ wx, float* __restrict__ wy, float* __restrict__ wz, float* __restrict__ wm) {
    pdl_begin();
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n) return;
    int x, y, z;
    cell_xyz(P, q, x, y, z);
    const bool solid = occ[q] != 0;
    const float4 o = vorticity_at(u, v, w, x, y, z, P);  // also for solid cells: no load waits on occupancy
    wx[q] = solid ? 0.0f : o.x;
    wy[q] = solid ? 0.0f : o.y;
    wz[q] = solid ? 0.0f : o.z;
    wm[q] = solid ? 0.0f : o.w;
}

// |w| lookup with clamp (or wrap on periodic axes), no occupancy test (load_flow_cell, :202-226).
__device__ __forceinline__ float flow_cell(const float* __restrict__ f, int x, int y, int z, const StepParams& P) {
    if (x < 0 || x >= P.nx) x = P.fper[0] ? wrapi(x, P.nx) : (x < 0 ? 0 : P.nx - 1);
    if (y < 0 || y >= P.ny) y = P.fper[1] ? wrapi(y, P.ny) : (y < 0 ? 0 : P.ny - 1);
    if (z < 0 || z >= P.nz) z = P.fper[2] ? wrapi(z, P.nz) : (z < 0 ? 0 : P.nz - 1);
    return __ldg(f + cidx(P, x, y, z));
}

// f = user force; fluid cells add buoyancy (:910-918) and confinement eps*h*(N x w) (:920-948).
__global__ void __launch_bounds__(kThreads) cell_force_kernel(const __grid_constant__ StepParams P, const float* __restrict__ wx, const float* __restrict__ wy, const float* __restrict__ wz, const float* __restrict__ wm, const float* __restrict__ density, const float* __restrict__ temperature, const float* __restrict__ ufx,
                                                               const float* __restrict__ ufy, const float* __restrict__ ufz, const uint8_t* __restrict__ occ, float* __restrict__ fx, float* __restrict__ fy, float* __restrict__ fz,
                                                               const __grid_constant__ ScalarSources S) {
    pdl_begin();
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n) return;
    // The scalar stage's sourced fields and their padded copies: t_tmp = T' + dt * src_T, T' being T with solid cells at
    // the solid temperature (the step-start apply_solid_temperature of :2001 folded in); d_tmp = rho + dt * src_rho
    // (add_source, :852-857). T and rho do not change between this stage and the scalar advection.
    if (S.t_tmp) {
        const float tv = occ[q] != 0 ? S.solid_t[q] : temperature[q];
        const float tt = tv + P.dt * S.ts[q], dd = density[q] + P.dt * S.ds[q];
        S.t_tmp[q] = tt;
        S.d_tmp[q] = dd;
        if (S.t_pad) {
            int x, y, z;
            cell_xyz(P, q, x, y, z);
            S.t_pad[pad_index<4>(P, x, y, z)] = tt;
            S.d_pad[pad_index<3>(P, x, y, z)] = dd;
        }
    }
    float ax = ufx[q], ay = ufy[q], az = ufz[q];
    if (occ[q] == 0) {
        int x, y, z;
        cell_xyz(P, q, x, y, z);
        ay += -P.alpha * density[q] + P.beta * (temperature[q] - P.ambient);
        const float h = P.h, hh = 0.5f * P.inv_h;
        float gx, gy, gz;
        if (x > 0 && x < P.nx - 1 && y > 0 && y < P.ny - 1 && z > 0 && z < P.nz - 1) {  // all six neighbours in range
            const uint32_t sy = P.nx, sz = static_cast<uint32_t>(P.nx) * P.ny;
            gx = hh * (__ldg(wm + q + 1) - __ldg(wm + q - 1));
            gy = hh * (__ldg(wm + q + sy) - __ldg(wm + q - sy));
            gz = hh * (__ldg(wm + q + sz) - __ldg(wm + q - sz));
        } else {
            gx = hh * (flow_cell(wm, x + 1, y, z, P) - flow_cell(wm, x - 1, y, z, P));
            gy = hh * (flow_cell(wm, x, y + 1, z, P) - flow_cell(wm, x, y - 1, z, P));
            gz = hh * (flow_cell(wm, x, y, z + 1, P) - flow_cell(wm, x, y, z - 1, P));
        }
        const float gmag = sqrtf(gx * gx + gy * gy + gz * gz);
        if (!(gmag < 1.0e-6f)) {
            const float inv = 1.0f / gmag;
            const float nxv = gx * inv, nyv = gy * inv, nzv = gz * inv;
            const float ox = wx[q], oy = wy[q], oz = wz[q];
            ax += P.epsilon * h * (nyv * oz - nzv * oy);
            ay += P.epsilon * h * (nzv * ox - nxv * oz);
            az += P.epsilon * h * (nxv * oy - nyv * ox);
        }
    }
    fx[q] = ax;
    fy[q] = ay;
    fz[q] = az;
}

template <int A>
__device__ __forceinline__ void face_force_one(const StepParams& P, uint32_t q, const float* __restrict__ in, const float* __restrict__ f, const uint8_t* __restrict__ occ, const float* __restrict__ solid, float* __restrict__ out, float* __restrict__ pad) {
    int i, j, k;
    face_ijk<A>(P, q, i, j, k);
    // the settled value, also into the interior of the padded copy that the velocity advection reads
    auto put = [&](float v) {
        out[q] = v;
        if (pad) pad[pad_index<A>(P, i, j, k)] = v;
    };
    const int n = axis_n(P, A);
    const int s = A == 0 ? i : (A == 1 ? j : k);
    if (s > 0 && s < n) {
        // interior face: all loads first, then the rules (same values as the general path below)
        const uint32_t ri = cidx(P, i, j, k), li = ri - (A == 0 ? 1u : (A == 1 ? static_cast<uint32_t>(P.nx) : static_cast<uint32_t>(P.nx) * P.ny));
        const uint8_t ol = occ[li], orr = occ[ri];
        const float base = in[q], fl = f[li], fr = f[ri];
        if (ol != 0 || orr != 0) {
            float value = 0.0f, weight = 0.0f;
            if (ol != 0) {
                value += solid[li];
                weight += 1.0f;
            }
            if (orr != 0) {
                value += solid[ri];
                weight += 1.0f;
            }
            put(value / weight);
        } else {
            put(base + P.dt * (0.5f * (0.0f + fl + fr)));
        }
        return;
    }
    put(settle<A, false>(P, i, j, k, occ, solid, [&](int a, int b, int c) {
        const int s = A == 0 ? a : (A == 1 ? b : c);
        float sum = 0.0f, weight = 0.0f;
        int lc[3] = {a, b, c};
        if (s > 0) {
            lc[A] = s - 1;
            sum += f[cidx(P, lc[0], lc[1], lc[2])];
            weight += 1.0f;
        }
        if (s < n) {
            lc[A] = s;
            sum += f[cidx(P, lc[0], lc[1], lc[2])];
            weight += 1.0f;
        }
        const float base = in[fidx<A>(P, a, b, c)];
        return weight > 0.0f ? base + P.dt * (weight > 1.0f ? 0.5f * sum : sum) : base;  // exact halving
    }));
}

// Block ranges: [0, bu) -> x faces, [bu, bu+bv) -> y faces, rest -> z faces.
__global__ void __launch_bounds__(kThreads) face_force_kernel(const __grid_constant__ StepParams P, const float* __restrict__ iu, const float* __restrict__ iv, const float* __restrict__ iw, const float* __restrict__ fx, const float* __restrict__ fy, const float* __restrict__ fz, const uint8_t* __restrict__ occ, const float* __restrict__ su,
                                                               const float* __restrict__ sv, const float* __restrict__ sw, float* __restrict__ ou, float* __restrict__ ov, float* __restrict__ ow, float* __restrict__ pu, float* __restrict__ pv, float* __restrict__ pw, unsigned bu, unsigned bv) {
    pdl_begin();
    const unsigned b = blockIdx.x;
    if (b < bu) {
        const uint32_t q = b * kThreads + threadIdx.x;
        if (q < P.nu) face_force_one<0>(P, q, iu, fx, occ, su, ou, pu);
    } else if (b < bu + bv) {
        const uint32_t q = (b - bu) * kThreads + threadIdx.x;
        if (q < P.nv) face_force_one<1>(P, q, iv, fy, occ, sv, ov, pv);
    } else {
        const uint32_t q = (b - bu - bv) * kThreads + threadIdx.x;
        if (q < P.nw) face_force_one<2>(P, q, iw, fz, occ, sw, ow, pw);
    }
}

// ------------------------------------------------------------------------------------------ velocity advection
// Point (i, j, k) of this thread in block b of an nx x ny x nz grid of points covered by boxes of P.tile; false
// outside the grid. Boxes run x fastest, then y, then z.
__device__ __forceinline__ bool tile_point(const StepParams& P, unsigned b, int nx, int ny, int nz, int& i, int& j, int& k) {
    const int lx = P.tile[0], ly = P.tile[1], lz = P.tile[2];
    const unsigned ntx = (nx + (1 << lx) - 1) >> lx, nty = (ny + (1 << ly) - 1) >> ly;
    const unsigned r = b / ntx, bx = b - r * ntx, bz = r / nty, by = r - bz * nty;
    const unsigned t = threadIdx.x;
    i = static_cast<int>((bx << lx) + (t & ((1u << lx) - 1u)));
    j = static_cast<int>((by << ly) + ((t >> lx) & ((1u << ly) - 1u)));
    k = static_cast<int>((bz << lz) + (t >> (lx + ly)));
    return i < nx && j < ny && k < nz;
}
// Blocks of kThreads that cover an nx x ny x nz grid of points in the advection shape of P.
unsigned advect_blocks(const StepParams& P, int nx, int ny, int nz) {
    if (P.tile[0] < 0) return blocks_for(static_cast<uint64_t>(nx) * ny * nz);
    const uint64_t tx = 1u << P.tile[0], ty = 1u << P.tile[1], tz = 1u << P.tile[2];
    return static_cast<unsigned>(((nx + tx - 1) / tx) * ((ny + ty - 1) / ty) * ((nz + tz - 1) / tz));
}

template <int A, bool CUBIC, bool TILED, bool POW2>
__device__ __forceinline__ void advect_face_one(const StepParams& P, unsigned blk, const PadField& u, const PadField& v, const PadField& w, const uint8_t* __restrict__ occ, const float* __restrict__ solid, float* __restrict__ out) {
    int i, j, k;
    uint32_t q;
    if (TILED) {
        if (!tile_point(P, blk, fsx<A>(P), fsy<A>(P), fsz<A>(P), i, j, k)) return;
        q = fidx<A>(P, i, j, k);
    } else {
        q = blk * kThreads + threadIdx.x;
        if (q >= (A == 0 ? P.nu : (A == 1 ? P.nv : P.nw))) return;
        face_ijk<A>(P, q, i, j, k);
    }
    const PadField& src = A == 0 ? u : (A == 1 ? v : w);
    out[q] = settle<A, false>(P, i, j, k, occ, solid, [&](int a, int b, int c) {
        const float h = P.h;
        const float px = A == 0 ? static_cast<float>(a) * h : (static_cast<float>(a) + 0.5f) * h;
        const float py = A == 1 ? static_cast<float>(b) * h : (static_cast<float>(b) + 0.5f) * h;
        const float pz = A == 2 ? static_cast<float>(c) * h : (static_cast<float>(c) + 0.5f) * h;
        const float3 p = trace_rk2<POW2, A>(px, py, pz, a, b, c, u, v, w, occ, P);
        return sample_pad<A, CUBIC, POW2>(src, p.x, p.y, p.z, P);
    });
}

// Samples and traces read the padded copies of the velocity (ghost cells hold the boundary taps). Blocks
// [0, bu) advect u faces, [bu, bu + bv) v faces, the rest w faces, each in the shape P.tile selects. POW2: the cell
// size is a power of two, so grid coordinates are products instead of divisions (over_h, the same floats).
// Six blocks per SM (at most 42 registers): the gathers wait on L1/L2 latency, and the extra resident warps hide more
// of it than the few spilled registers cost (240 -> 224 us at 128^3 against the compiler's 64 registers, 4 blocks).
template <bool CUBIC, bool TILED, bool POW2>
__global__ void __launch_bounds__(kThreads, 6) advect_velocity_kernel(const __grid_constant__ StepParams P, const PadField u, const PadField v, const PadField w, const uint8_t* __restrict__ occ, const float* __restrict__ su, const float* __restrict__ sv, const float* __restrict__ sw, float* __restrict__ ou, float* __restrict__ ov,
                                                                    float* __restrict__ ow, unsigned bu, unsigned bv) {
    pdl_begin();
    const unsigned b = blockIdx.x;
    if (b < bu) advect_face_one<0, CUBIC, TILED, POW2>(P, b, u, v, w, occ, su, ou);
    else if (b < bu + bv) advect_face_one<1, CUBIC, TILED, POW2>(P, b - bu, u, v, w, occ, sv, ov);
    else advect_face_one<2, CUBIC, TILED, POW2>(P, b - bu - bv, u, v, w, occ, sw, ow);
}

// Padded copies (see PadField) of up to 3 fields in one launch: block z-range c * pz_blocks .. for field c; each
// thread fills kPadPlanes cells of one column (loads first, then stores), 32 x 8 columns per block.
constexpr int kPadPlanes = 4;
struct PadJob {
    const float* f[3];
    float* out[3];
    int kind[3];
    int count;
    int pz_blocks;  // blocks per field along z (kPadPlanes planes each)
};

template <int KIND>
__device__ __forceinline__ float pad_value(const StepParams& P, const float* __restrict__ f, int i, int j, int k) {
    const int fx = P.nx + (KIND == 0), fy = P.ny + (KIND == 1), fz = P.nz + (KIND == 2);
    if (i >= 0 && i < fx && j >= 0 && j < fy && k >= 0 && k < fz) return __ldg(f + (static_cast<uint32_t>(k) * fy + j) * fx + i);
    return boundary_tap<KIND>(f, i, j, k, P);
}

__global__ void __launch_bounds__(256) pad_kernel(const __grid_constant__ StepParams P, const __grid_constant__ PadJob J) {
    const int c = blockIdx.z / J.pz_blocks, kp0 = (blockIdx.z - c * J.pz_blocks) * kPadPlanes;
    if (c >= J.count) return;
    const int kind = c == 0 ? J.kind[0] : (c == 1 ? J.kind[1] : J.kind[2]);
    const int px = P.nx + (kind == 0) + 2 * kPad, py = P.ny + (kind == 1) + 2 * kPad, pz = P.nz + (kind == 2) + 2 * kPad;
    const int ip = blockIdx.x * 32 + threadIdx.x, jp = blockIdx.y * 8 + threadIdx.y;
    if (ip >= px || jp >= py || kp0 >= pz) return;
    const int i = ip - kPad, j = jp - kPad;
    const float* f = c == 0 ? J.f[0] : (c == 1 ? J.f[1] : J.f[2]);
    float* out = c == 0 ? J.out[0] : (c == 1 ? J.out[1] : J.out[2]);
    float v[kPadPlanes];
#pragma unroll
    for (int u = 0; u < kPadPlanes; ++u) {
        const int k = kp0 + u - kPad;
        switch (kind) {
        case 0: v[u] = pad_value<0>(P, f, i, j, k); break;
        case 1: v[u] = pad_value<1>(P, f, i, j, k); break;
        case 2: v[u] = pad_value<2>(P, f, i, j, k); break;
        case 3: v[u] = pad_value<3>(P, f, i, j, k); break;
        default: v[u] = pad_value<4>(P, f, i, j, k); break;
        }
    }
#pragma unroll
    for (int u = 0; u < kPadPlanes; ++u)
        if (kp0 + u < pz) out[(static_cast<uint32_t>(kp0 + u) * py + jp) * px + ip] = v[u];
}

// Ghost cells only, for padded copies whose interior the producing kernel wrote: thread g of field c (blockIdx.y)
// takes ghost cell g of the shell, enumerated as the 2 kPad whole z-planes, then in each interior plane the 2 kPad
// y-rows, then in each interior row the 2 kPad x-cells; its value is the boundary tap, as in pad_kernel.
__global__ void __launch_bounds__(256) pad_ghost_kernel(const __grid_constant__ StepParams P, const __grid_constant__ PadJob J) {
    pdl_begin();
    const int c = blockIdx.y;
    if (c >= J.count) return;
    const int kind = c == 0 ? J.kind[0] : (c == 1 ? J.kind[1] : J.kind[2]);
    const uint32_t fx = P.nx + (kind == 0), fy = P.ny + (kind == 1), fz = P.nz + (kind == 2);
    const uint32_t px = fx + 2 * kPad, py = fy + 2 * kPad;
    const uint32_t na = 2u * kPad * px * py, nb = fz * 2u * kPad * px, nc = fz * fy * 2u * kPad;
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= na + nb + nc) return;
    uint32_t ip, jp, kp;
    if (g < na) {  // whole ghost z-planes
        const uint32_t plane = g / (px * py), r = g - plane * px * py;
        kp = plane < static_cast<uint32_t>(kPad) ? plane : fz + plane;
        jp = r / px;
        ip = r - jp * px;
    } else if (g < na + nb) {  // ghost y-rows of the interior planes
        const uint32_t h = g - na, per = 2u * kPad * px, plane = h / per, r = h - plane * per, row = r / px;
        kp = kPad + plane;
        jp = row < static_cast<uint32_t>(kPad) ? row : fy + row;
        ip = r - row * px;
    } else {  // ghost x-cells of the interior rows
        const uint32_t h = g - na - nb, per = fy * 2u * kPad, plane = h / per, r = h - plane * per, row = r / (2u * kPad), xi = r - row * (2u * kPad);
        kp = kPad + plane;
        jp = kPad + row;
        ip = xi < static_cast<uint32_t>(kPad) ? xi : fx + xi;
    }
    const int i = static_cast<int>(ip) - kPad, j = static_cast<int>(jp) - kPad, k = static_cast<int>(kp) - kPad;
    const float* f = c == 0 ? J.f[0] : (c == 1 ? J.f[1] : J.f[2]);
    float* out = c == 0 ? J.out[0] : (c == 1 ? J.out[1] : J.out[2]);
    float v;
    switch (kind) {
    case 0: v = pad_value<0>(P, f, i, j, k); break;
    case 1: v = pad_value<1>(P, f, i, j, k); break;
    case 2: v = pad_value<2>(P, f, i, j, k); break;
    case 3: v = pad_value<3>(P, f, i, j, k); break;
    default: v = pad_value<4>(P, f, i, j, k); break;
    }
    out[(kp * py + jp) * px + ip] = v;
}

// ------------------------------------------------------------------------------------------ pressure rhs
// b = -(h^2/dt) div u* + sum of OUTFLOW face pressures; 0 at solid cells and at the anchor (:1304-1328).
__global__ void __launch_bounds__(kThreads) rhs_kernel(const __grid_constant__ StepParams P, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w, const uint8_t* __restrict__ occ, const int32_t* __restrict__ anchor, float* __restrict__ rhs) {
    pdl_begin();
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n) return;
    // every load is issued before the anchor/solid test (the six faces of a cell always exist)
    const bool zero = static_cast<int32_t>(q) == __ldg(anchor) || occ[q] != 0;
    int x, y, z;
    cell_xyz(P, q, x, y, z);
    const float h = P.h;
    const float div = (u[fidx<0>(P, x + 1, y, z)] - u[fidx<0>(P, x, y, z)] + v[fidx<1>(P, x, y + 1, z)] - v[fidx<1>(P, x, y, z)] + w[fidx<2>(P, x, y, z + 1)] - w[fidx<2>(P, x, y, z)]) * P.inv_h;
    if (zero) {
        rhs[q] = 0.0f;
        return;
    }
    float bsum = 0.0f;
    if (x == 0 && P.flow[0].type == kFlowOutflow) bsum += P.flow[0].pressure;
    if (x == P.nx - 1 && P.flow[1].type == kFlowOutflow) bsum += P.flow[1].pressure;
    if (y == 0 && P.flow[2].type == kFlowOutflow) bsum += P.flow[2].pressure;
    if (y == P.ny - 1 && P.flow[3].type == kFlowOutflow) bsum += P.flow[3].pressure;
    if (z == 0 && P.flow[4].type == kFlowOutflow) bsum += P.flow[4].pressure;
    if (z == P.nz - 1 && P.flow[5].type == kFlowOutflow) bsum += P.flow[5].pressure;
    rhs[q] = -(h * h / P.dt) * div + bsum;
}

// ------------------------------------------------------------------------------------------ projection
template <int A>
__device__ __forceinline__ void project_one(const StepParams& P, uint32_t q, const float* __restrict__ in, const float* __restrict__ p, const double* __restrict__ p64, const uint8_t* __restrict__ occ, const float* __restrict__ solid, float* __restrict__ out, float* __restrict__ pad) {
    int i, j, k;
    face_ijk<A>(P, q, i, j, k);
    // the projected value, also into the interior of the padded copy that the scalar advection reads
    auto put = [&](float v) {
        out[q] = v;
        if (pad) pad[pad_index<A>(P, i, j, k)] = v;
    };
    const int s = A == 0 ? i : (A == 1 ? j : k);
    if (s > 0 && s < axis_n(P, A)) {
        // interior face: both cells exist unwrapped, so every load is issued before any rule is decided; the
        // values are those of the general path below (solid rule, else the gradient step)
        const uint32_t ri = cidx(P, i, j, k), li = ri - (A == 0 ? 1u : (A == 1 ? static_cast<uint32_t>(P.nx) : static_cast<uint32_t>(P.nx) * P.ny));
        const uint8_t ol = occ[li], orr = occ[ri];
        const float base = in[q];
        float g;
        if (p64 != nullptr) g = static_cast<float>(P.dt_over_h64 * (p64[ri] - p64[li]));
        else g = P.dt * (p[ri] - p[li]) / P.h;
        if (ol != 0 || orr != 0) {
            float value = 0.0f, weight = 0.0f;
            if (ol != 0) {
                value += solid[li];
                weight += 1.0f;
            }
            if (orr != 0) {
                value += solid[ri];
                weight += 1.0f;
            }
            put(value / weight);
        } else {
            put(base - g);
        }
        return;
    }
    put(settle<A, true>(P, i, j, k, occ, solid, [&](int a, int b, int c) {
        int l[3] = {a, b, c};
        int r[3] = {a, b, c};
        l[A] -= 1;
        const bool hl = resolve_flow(P, l[0], l[1], l[2]);
        const bool hr = resolve_flow(P, r[0], r[1], r[2]);
        const float base = in[fidx<A>(P, a, b, c)];
        if (!(hl && hr)) return base;
        if (p64 != nullptr) {  // FP64 solution of a refined solve: the gradient keeps its precision
            const double g = P.dt_over_h64 * (p64[cidx(P, r[0], r[1], r[2])] - p64[cidx(P, l[0], l[1], l[2])]);
            return base - static_cast<float>(g);
        }
        const float pr = p[cidx(P, r[0], r[1], r[2])];
        const float pl = p[cidx(P, l[0], l[1], l[2])];
        return base - P.dt * (pr - pl) / P.h;
    }));
}

__global__ void __launch_bounds__(kThreads) project_kernel(const __grid_constant__ StepParams P, const float* __restrict__ iu, const float* __restrict__ iv, const float* __restrict__ iw, const float* __restrict__ p, const double* __restrict__ p64, const uint8_t* __restrict__ occ, const float* __restrict__ su, const float* __restrict__ sv, const float* __restrict__ sw, float* __restrict__ ou,
                                                            float* __restrict__ ov, float* __restrict__ ow, float* __restrict__ pu, float* __restrict__ pv, float* __restrict__ pw, unsigned bu, unsigned bv) {
    pdl_begin();
    const unsigned b = blockIdx.x;
    if (b < bu) {
        const uint32_t q = b * kThreads + threadIdx.x;
        if (q < P.nu) project_one<0>(P, q, iu, p, p64, occ, su, ou, pu);
    } else if (b < bu + bv) {
        const uint32_t q = (b - bu) * kThreads + threadIdx.x;
        if (q < P.nv) project_one<1>(P, q, iv, p, p64, occ, sv, ov, pv);
    } else {
        const uint32_t q = (b - bu - bv) * kThreads + threadIdx.x;
        if (q < P.nw) project_one<2>(P, q, iw, p, p64, occ, sw, ow, pw);
    }
}

// ------------------------------------------------------------------------------------------ scalars
// Fluid cells: one back-trace, then both scalars sampled with their own boundary rules (:1221-1233).
// Solid cells: temperature = solid temperature (:1235-1241), density = 0 until the fill pass.
template <bool CUBIC, bool TILED, bool POW2>
__global__ void __launch_bounds__(kThreads) advect_scalars_kernel(const __grid_constant__ StepParams P, const PadField u, const PadField v, const PadField w, const uint8_t* __restrict__ occ, const PadField t_tmp, const PadField d_tmp, const float* __restrict__ solid_t, float* __restrict__ t, float* __restrict__ d) {
    pdl_begin();
    int x, y, z;
    uint32_t q;
    if (TILED) {
        if (!tile_point(P, blockIdx.x, P.nx, P.ny, P.nz, x, y, z)) return;
        q = cidx(P, x, y, z);
    } else {
        q = blockIdx.x * blockDim.x + threadIdx.x;
        if (q >= P.n) return;
        cell_xyz(P, q, x, y, z);
    }
    if (occ[q] != 0) {
        t[q] = solid_t[q];
        d[q] = 0.0f;
        return;
    }
    const float h = P.h;
    const float3 p = trace_rk2<POW2, 3>((static_cast<float>(x) + 0.5f) * h, (static_cast<float>(y) + 0.5f) * h, (static_cast<float>(z) + 0.5f) * h, x, y, z, u, v, w, occ, P);
    float tv, dv;
    sample_pad_scalars<CUBIC, POW2>(t_tmp, d_tmp, p.x, p.y, p.z, P, tv, dv);
    t[q] = tv;
    d[q] = dv;
}

__global__ void density_fill_kernel(const FillEntry* __restrict__ list, const uint32_t* __restrict__ count, float* __restrict__ d) {
    pdl_begin();
    const uint32_t n = *count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const FillEntry e = list[t];
        d[e.cell] = e.source >= 0 ? d[e.source] : 0.0f;
    }
}

// ------------------------------------------------------------------------------------------ views
__global__ void __launch_bounds__(kThreads) views_kernel(const __grid_constant__ StepParams P, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w, const uint8_t* __restrict__ occ, float* __restrict__ cx, float* __restrict__ cy, float* __restrict__ cz, float* __restrict__ vm, float* __restrict__ wx, float* __restrict__ wy,
                                                          float* __restrict__ wz, float* __restrict__ wm, float* __restrict__ div, uint32_t groups) {
    pdl_begin();
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n) return;
    int x, y, z;
    cell_xyz(P, q, x, y, z);
    if (groups & kViewsVelocity) {
        const float a = centred<0>(u, x, y, z, P);
        const float b = centred<1>(v, x, y, z, P);
        const float c = centred<2>(w, x, y, z, P);
        cx[q] = a;
        cy[q] = b;
        cz[q] = c;
        vm[q] = sqrtf(a * a + b * b + c * c);
    }
    if (!(groups & kViewsVorticity)) return;
    if (occ[q] != 0) {
        wx[q] = wy[q] = wz[q] = wm[q] = 0.0f;
        div[q] = 0.0f;
        return;
    }
    const float4 o = vorticity_at(u, v, w, x, y, z, P);
    wx[q] = o.x;
    wy[q] = o.y;
    wz[q] = o.z;
    wm[q] = o.w;
    div[q] = (u[fidx<0>(P, x + 1, y, z)] - u[fidx<0>(P, x, y, z)] + v[fidx<1>(P, x, y + 1, z)] - v[fidx<1>(P, x, y, z)] + w[fidx<2>(P, x, y, z + 1)] - w[fidx<2>(P, x, y, z)]) * P.inv_h;
}

// ------------------------------------------------------------------------------------------ occupancy-derived
__global__ void occupancy_float_kernel(uint32_t n, const uint8_t* __restrict__ occ, float* __restrict__ out) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) out[q] = static_cast<float>(occ[q]);
}

__global__ void set_int_kernel(int32_t* p, int32_t v) { *p = v; }

// anchor = smallest fluid cell index (:1292-1302); warp minimum first, one atomic per warp.
__global__ void anchor_kernel(uint32_t n, const uint8_t* __restrict__ occ, int32_t* anchor) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t v = (q < n && occ[q] == 0) ? static_cast<int32_t>(q) : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v != 0x7fffffff) atomicMin(anchor, v);
}

// Row code of the Poisson operator (:1343-1412): solid or anchor rows are identity (diag 1, no neighbours);
// a fluid row's diagonal counts fluid neighbours (anchor included, periodic wrap, repeats counted) plus OUTFLOW
// domain faces, at least 1; neighbour bits mark distinct fluid non-anchor neighbours other than the cell itself.
__global__ void __launch_bounds__(kThreads) stencil_code_kernel(const __grid_constant__ StepParams P, const uint8_t* __restrict__ occ, const int32_t* __restrict__ anchor_ptr, uint16_t* __restrict__ codes) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n) return;
    const int32_t anchor = *anchor_ptr;
    if (occ[q] != 0 || static_cast<int32_t>(q) == anchor) {
        codes[q] = static_cast<uint16_t>(1u << 8);
        return;
    }
    int c[3];
    cell_xyz(P, q, c[0], c[1], c[2]);
    const int n[3] = {P.nx, P.ny, P.nz};
    uint32_t diag = 0, mask = 0;
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        const int a = e >> 1;
        int d[3] = {c[0], c[1], c[2]};
        d[a] += (e & 1) ? 1 : -1;
        if (d[a] < 0 || d[a] >= n[a]) {
            if (!P.fper[a]) {
                if (P.flow[e].type == kFlowOutflow) ++diag;
                continue;
            }
            d[a] = wrapi(d[a], n[a]);
        }
        const uint32_t nb = cidx(P, d[0], d[1], d[2]);
        if (occ[nb] != 0) continue;
        ++diag;
        if (static_cast<int32_t>(nb) == anchor || nb == q) continue;
        if ((e & 1) && n[a] == 2 && P.fper[a]) continue;  // same cell as the -a neighbour, kept once
        mask |= 1u << e;
    }
    if (diag == 0) diag = 1;
    codes[q] = static_cast<uint16_t>(mask | (diag << 8) | kCodeActive);
}

// Nearest-fluid source of each solid cell (:1243-1290): first Chebyshev shell (radius 1, 2, ...) holding a fluid
// cell, smallest squared distance in it, first in (dz, dy, dx) scan order on ties, density periodicity. Only the
// shell surface is enumerated, in the same order as a full-cube scan.
__global__ void __launch_bounds__(kThreads) fill_build_kernel(const __grid_constant__ StepParams P, const uint8_t* __restrict__ occ, const int32_t* __restrict__ anchor_ptr, FillEntry* __restrict__ list, uint32_t* __restrict__ count) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n || occ[q] == 0) return;
    int32_t best = -1;
    if (*anchor_ptr < static_cast<int32_t>(P.n)) {  // at least one fluid cell exists
        int x, y, z;
        cell_xyz(P, q, x, y, z);
        const int max_radius = imax(P.nx, imax(P.ny, P.nz));
        for (int r = 1; r <= max_radius && best < 0; ++r) {
            int best_d2 = 0x7fffffff;
            for (int dz = -r; dz <= r; ++dz) {
                for (int dy = -r; dy <= r; ++dy) {
                    const bool full_row = (dz == -r || dz == r || dy == -r || dy == r);
                    const int step = full_row ? 1 : 2 * r;
                    for (int dx = -r; dx <= r; dx += step) {
                        int c[3] = {x + dx, y + dy, z + dz};
                        const int nn[3] = {P.nx, P.ny, P.nz};
                        bool ok = true;
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            if (P.dper[a]) c[a] = wrapi(c[a], nn[a]);
                            ok = ok && c[a] >= 0 && c[a] < nn[a];
                        }
                        if (!ok) continue;
                        const uint32_t nb = cidx(P, c[0], c[1], c[2]);
                        if (occ[nb] != 0) continue;
                        const int d2 = dx * dx + dy * dy + dz * dz;
                        if (d2 < best_d2) {
                            best_d2 = d2;
                            best = static_cast<int32_t>(nb);
                        }
                    }
                }
            }
        }
    }
    const uint32_t slot = atomicAdd(count, 1u);
    list[slot] = FillEntry{q, best};
}

__global__ void fill_value_kernel(float* __restrict__ dst, float value, uint64_t count) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) dst[i] = value;
}

}  // namespace

StepParams make_params(const SmokeSimulationConfig& cfg) {
    StepParams P{};
    P.nx = cfg.nx;
    P.ny = cfg.ny;
    P.nz = cfg.nz;
    P.h = cfg.cell_size;
    P.dt = cfg.dt;
    P.ambient = cfg.ambient_temperature;
    P.alpha = cfg.buoyancy_density_factor;
    P.beta = cfg.buoyancy_temperature_factor;
    P.epsilon = cfg.vorticity_confinement;
    P.cubic = cfg.scalar_advection_mode == SMOKE_SIMULATION_SCALAR_ADVECTION_MONOTONIC_CUBIC;
    const SmokeSimulationFlowBoundaryFaceDesc* fb = &cfg.flow_boundary.x_minus;
    const SmokeSimulationScalarBoundaryFaceDesc* db = &cfg.density_boundary.x_minus;
    const SmokeSimulationScalarBoundaryFaceDesc* tb = &cfg.temperature_boundary.x_minus;
    for (int e = 0; e < 6; ++e) {
        P.flow[e] = fb[e];
        P.den[e] = db[e];
        P.tem[e] = tb[e];
    }
    for (int a = 0; a < 3; ++a) {
        P.fper[a] = fb[2 * a].type == kFlowPeriodic && fb[2 * a + 1].type == kFlowPeriodic;
        P.dper[a] = db[2 * a].type == kScalarPeriodic && db[2 * a + 1].type == kScalarPeriodic;
        P.tper[a] = tb[2 * a].type == kScalarPeriodic && tb[2 * a + 1].type == kScalarPeriodic;
    }
    const uint32_t nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
    P.n = nx * ny * nz;
    P.nu = (nx + 1) * ny * nz;
    P.nv = nx * (ny + 1) * nz;
    P.nw = nx * ny * (nz + 1);
    P.inv_h = 1.0f / cfg.cell_size;
    {  // a normal power of two with a normal reciprocal: x * inv_h == x / h for every float x
        int e = 0;
        P.h_pow2 = std::isnormal(cfg.cell_size) && std::isnormal(P.inv_h) && std::frexp(cfg.cell_size, &e) == 0.5f && P.inv_h * cfg.cell_size == 1.0f;
    }
    P.dt_over_h64 = static_cast<double>(cfg.dt) / static_cast<double>(cfg.cell_size);
    P.div_nx = FastDiv(nx);
    P.div_ny = FastDiv(ny);
    P.div_slab = FastDiv(nx * ny);
    for (int a = 0; a < 3; ++a) {
        P.div_fx[a] = FastDiv(nx + (a == 0));
        P.div_fy[a] = FastDiv(ny + (a == 1));
    }
    set_advect_tile(P, 0);
    return P;
}

bool set_advect_tile(StepParams& P, int code) {
    if (code < 0 || code >= kAdvectTileCount) return false;
    for (int a = 0; a < 3; ++a) P.tile[a] = kAdvectTiles[code][a];
    return true;
}

cudaError_t launch_vorticity(const StepParams& P, ConstFaces vel, const uint8_t* occ, float* wx, float* wy, float* wz, float* wmag, cudaStream_t s) {
    vorticity_kernel<<<blocks_for(P.n), kThreads, 0, s>>>(P, vel.u, vel.v, vel.w, occ, wx, wy, wz, wmag);
    return cudaGetLastError();
}

cudaError_t launch_cell_force(const StepParams& P, const float* wx, const float* wy, const float* wz, const float* wmag, const float* density, const float* temperature, const float* ufx, const float* ufy, const float* ufz, const uint8_t* occ, float* fx, float* fy, float* fz, cudaStream_t s, const ScalarSources& S) {
    launch_pdl(cell_force_kernel, dim3(blocks_for(P.n)), dim3(kThreads), 0, s, P, wx, wy, wz, wmag, density, temperature, ufx, ufy, ufz, occ, fx, fy, fz, S);
    return cudaGetLastError();
}

cudaError_t launch_face_force(const StepParams& P, ConstFaces in, const float* fx, const float* fy, const float* fz, const uint8_t* occ, ConstFaces solid, Faces out, cudaStream_t s, Faces pad) {
    const unsigned bu = blocks_for(P.nu), bv = blocks_for(P.nv), bw = blocks_for(P.nw);
    launch_pdl(face_force_kernel, dim3(bu + bv + bw), dim3(kThreads), 0, s, P, in.u, in.v, in.w, fx, fy, fz, occ, solid.u, solid.v, solid.w, out.u, out.v, out.w, pad.u, pad.v, pad.w, bu, bv);
    return cudaGetLastError();
}

// Padded copy descriptor of field KIND stored at `pad`.
PadField pad_field(const StepParams& P, int kind, const float* raw, const float* pad) {
    const uint32_t fx = P.nx + (kind == 0), fy = P.ny + (kind == 1);
    PadField F{};
    F.p = pad;
    F.raw = raw;
    F.px = fx + 2 * kPad;
    F.pxy = F.px * (fy + 2 * kPad);
    return F;
}

size_t pad_count(const StepParams& P, int kind) {
    return static_cast<size_t>(P.nx + (kind == 0) + 2 * kPad) * (P.ny + (kind == 1) + 2 * kPad) * (P.nz + (kind == 2) + 2 * kPad);
}

cudaError_t launch_pads(const StepParams& P, int count, const int* kinds, const float* const* fields, float* const* pads, cudaStream_t s, int ghost_only) {
    if (count < 1 || count > 3) return cudaErrorInvalidValue;
    PadJob J{};
    J.count = count;
    J.pz_blocks = (P.nz + 1 + 2 * kPad + kPadPlanes - 1) / kPadPlanes;
    for (int c = 0; c < count; ++c) {
        J.f[c] = fields[c];
        J.out[c] = pads[c];
        J.kind[c] = kinds[c];
    }
    if (ghost_only) {  // the largest shell of the fields (faces of the x, y or z axis have one more layer)
        const uint32_t px = P.nx + 1 + 2 * kPad, py = P.ny + 1 + 2 * kPad, pz = P.nz + 1 + 2 * kPad;
        const uint64_t most = static_cast<uint64_t>(px) * py * pz - static_cast<uint64_t>(P.nx) * P.ny * P.nz;
        launch_pdl(pad_ghost_kernel, dim3(static_cast<unsigned>((most + 255) / 256), count), dim3(256), 0, s, P, J);
        return cudaGetLastError();
    }
    const dim3 grid((P.nx + 1 + 2 * kPad + 31) / 32, (P.ny + 1 + 2 * kPad + 7) / 8, J.pz_blocks * count);
    pad_kernel<<<grid, dim3(32, 8), 0, s>>>(P, J);
    return cudaGetLastError();
}

// The advection kernel instance <CUBIC, TILED, POW2> of P, from the 8 given in that binary order.
template <class K>
K pick_advect(const StepParams& P, K k000, K k001, K k010, K k011, K k100, K k101, K k110, K k111) {
    const K all[8] = {k000, k001, k010, k011, k100, k101, k110, k111};
    return all[(P.cubic ? 4 : 0) + (P.tile[0] >= 0 ? 2 : 0) + (P.h_pow2 ? 1 : 0)];
}

// The device's global nanosecond timer into *slot (one thread).
__global__ void time_stamp_kernel(unsigned long long* slot) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *slot = t;
}

cudaError_t launch_time_stamp(unsigned long long* slot, cudaStream_t s) {
    time_stamp_kernel<<<1, 1, 0, s>>>(slot);
    return cudaGetLastError();
}

cudaError_t launch_advect_velocity(const StepParams& P, ConstFaces in, ConstFaces pad, const uint8_t* occ, ConstFaces solid, Faces out, cudaStream_t s) {
    const unsigned bu = advect_blocks(P, P.nx + 1, P.ny, P.nz), bv = advect_blocks(P, P.nx, P.ny + 1, P.nz), bw = advect_blocks(P, P.nx, P.ny, P.nz + 1);
    const PadField u = pad_field(P, 0, in.u, pad.u), v = pad_field(P, 1, in.v, pad.v), w = pad_field(P, 2, in.w, pad.w);
    auto kernel = pick_advect(P, advect_velocity_kernel<false, false, false>, advect_velocity_kernel<false, false, true>, advect_velocity_kernel<false, true, false>, advect_velocity_kernel<false, true, true>, advect_velocity_kernel<true, false, false>,
                              advect_velocity_kernel<true, false, true>, advect_velocity_kernel<true, true, false>, advect_velocity_kernel<true, true, true>);
    launch_pdl(kernel, dim3(bu + bv + bw), dim3(kThreads), 0, s, P, u, v, w, occ, solid.u, solid.v, solid.w, out.u, out.v, out.w, bu, bv);
    return cudaGetLastError();
}

cudaError_t launch_rhs(const StepParams& P, ConstFaces vel, const uint8_t* occ, const int32_t* anchor, float* rhs, cudaStream_t s) {
    launch_pdl(rhs_kernel, dim3(blocks_for(P.n)), dim3(kThreads), 0, s, P, vel.u, vel.v, vel.w, occ, anchor, rhs);
    return cudaGetLastError();
}

cudaError_t launch_project(const StepParams& P, ConstFaces in, const float* pressure, const double* pressure64, const uint8_t* occ, ConstFaces solid, Faces out, cudaStream_t s, Faces pad) {
    const unsigned bu = blocks_for(P.nu), bv = blocks_for(P.nv), bw = blocks_for(P.nw);
    launch_pdl(project_kernel, dim3(bu + bv + bw), dim3(kThreads), 0, s, P, in.u, in.v, in.w, pressure, pressure64, occ, solid.u, solid.v, solid.w, out.u, out.v, out.w, pad.u, pad.v, pad.w, bu, bv);
    return cudaGetLastError();
}

cudaError_t launch_advect_scalars(const StepParams& P, ConstFaces vel, ConstFaces vel_pad, const uint8_t* occ, const float* t_tmp, const float* t_pad, const float* d_tmp, const float* d_pad, const float* solid_temperature, float* temperature, float* density, cudaStream_t s) {
    const PadField u = pad_field(P, 0, vel.u, vel_pad.u), v = pad_field(P, 1, vel.v, vel_pad.v), w = pad_field(P, 2, vel.w, vel_pad.w);
    const PadField t = pad_field(P, 4, t_tmp, t_pad), d = pad_field(P, 3, d_tmp, d_pad);
    auto kernel = pick_advect(P, advect_scalars_kernel<false, false, false>, advect_scalars_kernel<false, false, true>, advect_scalars_kernel<false, true, false>, advect_scalars_kernel<false, true, true>, advect_scalars_kernel<true, false, false>,
                              advect_scalars_kernel<true, false, true>, advect_scalars_kernel<true, true, false>, advect_scalars_kernel<true, true, true>);
    launch_pdl(kernel, dim3(advect_blocks(P, P.nx, P.ny, P.nz)), dim3(kThreads), 0, s, P, u, v, w, occ, t, d, solid_temperature, temperature, density);
    return cudaGetLastError();
}

cudaError_t launch_density_fill(const FillEntry* list, const uint32_t* count, float* density, int max_blocks, cudaStream_t s) {
    launch_pdl(density_fill_kernel, dim3(max_blocks), dim3(kThreads), 0, s, list, count, density);
    return cudaGetLastError();
}

cudaError_t launch_views(const StepParams& P, ConstFaces vel, const uint8_t* occ, float* cx, float* cy, float* cz, float* vmag, float* wx, float* wy, float* wz, float* wmag, float* div, uint32_t groups, cudaStream_t s) {
    views_kernel<<<blocks_for(P.n), kThreads, 0, s>>>(P, vel.u, vel.v, vel.w, occ, cx, cy, cz, vmag, wx, wy, wz, wmag, div, groups);
    return cudaGetLastError();
}

cudaError_t launch_occupancy_float(const StepParams& P, const uint8_t* occ, float* out, cudaStream_t s) {
    occupancy_float_kernel<<<blocks_for(P.n), kThreads, 0, s>>>(P.n, occ, out);
    return cudaGetLastError();
}

cudaError_t launch_anchor(const StepParams& P, const uint8_t* occ, int32_t* anchor, cudaStream_t s) {
    set_int_kernel<<<1, 1, 0, s>>>(anchor, static_cast<int32_t>(P.n));
    anchor_kernel<<<blocks_for(P.n), kThreads, 0, s>>>(P.n, occ, anchor);
    return cudaGetLastError();
}

cudaError_t launch_stencil_codes(const StepParams& P, const uint8_t* occ, const int32_t* anchor, uint16_t* codes, cudaStream_t s) {
    stencil_code_kernel<<<blocks_for(P.n), kThreads, 0, s>>>(P, occ, anchor, codes);
    return cudaGetLastError();
}

cudaError_t launch_fill_build(const StepParams& P, const uint8_t* occ, const int32_t* anchor, FillEntry* list, uint32_t* count, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    fill_build_kernel<<<blocks_for(P.n), kThreads, 0, s>>>(P, occ, anchor, list, count);
    return cudaGetLastError();
}

cudaError_t launch_fill_value(float* dst, float value, uint64_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const uint64_t want = (count + kThreads - 1) / kThreads;
    const unsigned grid = static_cast<unsigned>(want < 4096 ? want : 4096);
    fill_value_kernel<<<grid, kThreads, 0, s>>>(dst, value, count);
    return cudaGetLastError();
}

}  // namespace smoke_b200
