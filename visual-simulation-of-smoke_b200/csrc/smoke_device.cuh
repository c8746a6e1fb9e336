// Device-side building blocks of the B200 smoke step: launch parameters, index arithmetic, the reference's
// boundary "ghost" rules, trilinear / monotone-cubic samplers and the RK2 back-trace.
//
// Behaviour follows the reference (backend-cuda.cu:121-838); the structure does not: every rule is
// written once and specialised by template on the field kind, and each sampler first tests whether its whole
// tap box lies inside the array, in which case it gathers without any boundary logic (the common case).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "visual-simulation-of-smoke-3d.h"

namespace smoke_b200 {

constexpr uint32_t kFlowNoSlip = SMOKE_SIMULATION_FLOW_BOUNDARY_NO_SLIP_WALL;
constexpr uint32_t kFlowFreeSlip = SMOKE_SIMULATION_FLOW_BOUNDARY_FREE_SLIP_WALL;
constexpr uint32_t kFlowOutflow = SMOKE_SIMULATION_FLOW_BOUNDARY_OUTFLOW;
constexpr uint32_t kFlowPeriodic = SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC;
constexpr uint32_t kScalarFixed = SMOKE_SIMULATION_SCALAR_BOUNDARY_FIXED_VALUE;
constexpr uint32_t kScalarZeroFlux = SMOKE_SIMULATION_SCALAR_BOUNDARY_ZERO_FLUX;
constexpr uint32_t kScalarPeriodic = SMOKE_SIMULATION_SCALAR_BOUNDARY_PERIODIC;

// Unsigned division by a runtime constant d >= 1, exact for every 32-bit numerator
// (Granlund & Montgomery 1994, "round-up" multiplier with the add-and-shift fix-up).
struct FastDiv {
    uint32_t d = 1, m = 0, s = 0;
    FastDiv() = default;
    explicit FastDiv(uint32_t divisor) : d(divisor) {
        uint32_t l = 0;
        while ((1ull << l) < d) ++l;
        m = static_cast<uint32_t>(((1ull << 32) * ((1ull << l) - d)) / d + 1);
        s = l;
    }
#if defined(__CUDACC__)
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        if (d == 1) return n;
        const uint32_t t = __umulhi(n, m);
        return (t + ((n - t) >> 1)) >> (s - 1);
    }
#endif
};

// Everything a step kernel needs, passed by value (__grid_constant__) to every launch.
struct StepParams {
    int nx, ny, nz;
    float h, dt;
    float ambient, alpha, beta, epsilon;
    int cubic;          // scalar_advection_mode == MONOTONIC_CUBIC (applies to velocity and scalars)
    int fper[3];        // flow periodic per axis
    int dper[3];        // density periodic per axis
    int tper[3];        // temperature periodic per axis
    SmokeSimulationFlowBoundaryFaceDesc flow[6];   // x-, x+, y-, y+, z-, z+
    SmokeSimulationScalarBoundaryFaceDesc den[6];
    SmokeSimulationScalarBoundaryFaceDesc tem[6];
    uint32_t n, nu, nv, nw; // cell and face counts
    FastDiv div_nx, div_ny, div_slab;            // cells: x fastest
    FastDiv div_fx[3], div_fy[3];                // faces of axis a: row length and rows per slab
    float inv_h;                                 // 1 / h (grid coordinates of sample positions)
    double dt_over_h64;                          // dt / h in FP64 (gradient of the refined FP64 pressure)
    int tile[3];                                 // advection blocks: log2 extents (x, y, z) of the box of faces or
                                                 // cells one block covers (sum 8); tile[0] < 0: 256 consecutive ones
    int h_pow2;                                  // h and 1 / h are normal powers of two (see over_h)
};

#if defined(__CUDACC__)

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return imin(imax(v, lo), hi); }
__device__ __forceinline__ int wrapi(int v, int n) {
    v %= n;
    return v < 0 ? v + n : v;
}

// Cell (x,y,z) -> linear index, x fastest.
__device__ __forceinline__ uint32_t cidx(const StepParams& P, int x, int y, int z) {
    return (static_cast<uint32_t>(z) * P.ny + y) * P.nx + x;
}
// Face of axis A: extents (nx + [A==0]) x (ny + [A==1]) x (nz + [A==2]).
template <int A>
__device__ __forceinline__ int fsx(const StepParams& P) { return P.nx + (A == 0); }
template <int A>
__device__ __forceinline__ int fsy(const StepParams& P) { return P.ny + (A == 1); }
template <int A>
__device__ __forceinline__ int fsz(const StepParams& P) { return P.nz + (A == 2); }
template <int A>
__device__ __forceinline__ uint32_t fidx(const StepParams& P, int i, int j, int k) {
    return (static_cast<uint32_t>(k) * fsy<A>(P) + j) * fsx<A>(P) + i;
}

__device__ __forceinline__ float face_comp(const SmokeSimulationFlowBoundaryFaceDesc& f, int c) {
    return c == 0 ? f.velocity_x : (c == 1 ? f.velocity_y : f.velocity_z);
}

__device__ __forceinline__ int axis_n(const StepParams& P, int a) { return a == 0 ? P.nx : (a == 1 ? P.ny : P.nz); }

// ---------------------------------------------------------------------------------------------- taps
// Face component A at integer index (i,j,k), with the reference's ghost rule outside the array
// (backend-cuda.cu:276-376): along A, OUTFLOW -> interior, otherwise 2*wall - interior; across A,
// OUTFLOW and FREE_SLIP -> interior, otherwise 2*wall - interior; periodic axes wrap. Axes are resolved
// in x, y, z order and the interior sample clamps the remaining coordinates.
template <int A>
__device__ inline float face_tap_slow(const float* __restrict__ f, int i, int j, int k, const StepParams& P) {
    int c[3] = {i, j, k};
    const int ext[3] = {fsx<A>(P) - 1, fsy<A>(P) - 1, fsz<A>(P) - 1};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (c[a] < 0 || c[a] > ext[a]) {
            if (P.fper[a]) {
                c[a] = wrapi(c[a], axis_n(P, a));
            } else {
                const SmokeSimulationFlowBoundaryFaceDesc face = P.flow[2 * a + (c[a] < 0 ? 0 : 1)];
                int q[3];
#pragma unroll
                for (int b = 0; b < 3; ++b) q[b] = (b == a) ? (c[a] < 0 ? 0 : ext[a]) : clampi(c[b], 0, ext[b]);
                const float interior = f[fidx<A>(P, q[0], q[1], q[2])];
                if (face.type == kFlowOutflow) return interior;
                if (a != A && face.type == kFlowFreeSlip) return interior;
                return 2.0f * face_comp(face, A) - interior;
            }
        }
    }
    return f[fidx<A>(P, c[0], c[1], c[2])];
}

// Cell-centred scalar tap with the scalar rule (backend-cuda.cu:166-200): PERIODIC wraps, ZERO_FLUX clamps,
// FIXED_VALUE returns the face value.
__device__ inline float scalar_tap_slow(const float* __restrict__ f, int x, int y, int z, const StepParams& P, const SmokeSimulationScalarBoundaryFaceDesc* bc, const int* per) {
    int c[3] = {x, y, z};
    const int n[3] = {P.nx, P.ny, P.nz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (c[a] < 0 || c[a] >= n[a]) {
            const SmokeSimulationScalarBoundaryFaceDesc face = bc[2 * a + (c[a] < 0 ? 0 : 1)];
            if (per[a]) c[a] = wrapi(c[a], n[a]);
            else if (face.type == kScalarZeroFlux) c[a] = c[a] < 0 ? 0 : n[a] - 1;
            else return face.value;
        }
    }
    return f[cidx(P, c[0], c[1], c[2])];
}

// ---------------------------------------------------------------------------------------------- samplers
// Hermite cubic with central slopes, slopes zeroed where they disagree in sign with the secant or the secant
// is below 1e-6 (backend-cuda.cu:378-392). Every operation is spelled out (IEEE single, round to nearest), so that
// the two-lane form below, which the padded samplers use, gives the same bits as this scalar form.
struct HermiteW {
    float h00, h10, h01, h11;  // weights of p1, m1, p2, m2
};
__device__ __forceinline__ HermiteW hermite_weights(float t) {
    const float t2 = __fmul_rn(t, t);
    const float t3 = __fmul_rn(t2, t);
    HermiteW w;
    w.h00 = __fmaf_rn(2.0f, t3, __fmaf_rn(-3.0f, t2, 1.0f));  // 2t^3 - 3t^2 + 1
    w.h10 = __fadd_rn(t3, __fmaf_rn(-2.0f, t2, t));            // t^3 - 2t^2 + t
    w.h01 = __fmaf_rn(-2.0f, t3, __fmul_rn(3.0f, t2));         // -2t^3 + 3t^2
    w.h11 = __fsub_rn(t3, t2);                                  // t^3 - t^2
    return w;
}
__device__ __forceinline__ float mono_cubic(float p0, float p1, float p2, float p3, const HermiteW& w) {
    const float delta = __fsub_rn(p2, p1);
    float m1 = __fmul_rn(0.5f, __fsub_rn(p2, p0));
    float m2 = __fmul_rn(0.5f, __fsub_rn(p3, p1));
    const bool flat = fabsf(delta) < 1.0e-6f;
    if (flat || __fmul_rn(m1, delta) <= 0.0f) m1 = 0.0f;
    if (flat || __fmul_rn(m2, delta) <= 0.0f) m2 = 0.0f;
    float r = __fmul_rn(w.h00, p1);
    r = __fmaf_rn(w.h10, m1, r);
    r = __fmaf_rn(w.h01, p2, r);
    return __fmaf_rn(w.h11, m2, r);
}
__device__ __forceinline__ float mono_cubic(float p0, float p1, float p2, float p3, float t) { return mono_cubic(p0, p1, p2, p3, hermite_weights(t)); }

// Two lanes of FP32 in one 64-bit register, for sm_100's paired FP32 instructions (add/sub/mul/fma .rn.f32x2): two
// IEEE single operations per instruction, each lane rounded exactly as the scalar instruction rounds it.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
struct HermiteW2 {
    f32x2 h00, h10, h01, h11;
};
__device__ __forceinline__ HermiteW2 hermite_pair(const HermiteW& a, const HermiteW& b) {
    return HermiteW2{f2_pack(a.h00, b.h00), f2_pack(a.h10, b.h10), f2_pack(a.h01, b.h01), f2_pack(a.h11, b.h11)};
}
// Two monotone cubics at once (lane by lane the scalar mono_cubic, same operations in the same order): the slope and
// polynomial arithmetic in paired instructions, the limiter's tests per lane.
__device__ __forceinline__ f32x2 mono_cubic2(f32x2 p0, f32x2 p1, f32x2 p2, f32x2 p3, const HermiteW2& w) {
    const f32x2 half = f2_pack(0.5f, 0.5f);
    const f32x2 delta = f2_sub(p2, p1);
    const f32x2 m1 = f2_mul(half, f2_sub(p2, p0));
    const f32x2 m2 = f2_mul(half, f2_sub(p3, p1));
    const f32x2 s1 = f2_mul(m1, delta), s2 = f2_mul(m2, delta);
    float d0, d1, a0, a1, b0, b1, m10, m11, m20, m21;
    f2_unpack(delta, d0, d1);
    f2_unpack(s1, a0, a1);
    f2_unpack(s2, b0, b1);
    f2_unpack(m1, m10, m11);
    f2_unpack(m2, m20, m21);
    const bool flat0 = fabsf(d0) < 1.0e-6f, flat1 = fabsf(d1) < 1.0e-6f;
    if (flat0 || a0 <= 0.0f) m10 = 0.0f;
    if (flat1 || a1 <= 0.0f) m11 = 0.0f;
    if (flat0 || b0 <= 0.0f) m20 = 0.0f;
    if (flat1 || b1 <= 0.0f) m21 = 0.0f;
    f32x2 r = f2_mul(w.h00, p1);
    r = f2_fma(w.h10, f2_pack(m10, m11), r);
    r = f2_fma(w.h01, p2, r);
    return f2_fma(w.h11, f2_pack(m20, m21), r);
}

__device__ __forceinline__ float wrap_pos(float p, int n, float h) {
    const float extent = static_cast<float>(n) * h;
    p = fmodf(p, extent);
    if (p < 0.0f) p += extent;
    return p;
}

// x / h exactly as the IEEE division computes it. For a power-of-two h (P.h_pow2, with 1 / h exact and normal) the
// product x * (1 / h) rounds the same real number x * 2^-k once, so it is the identical float; __fmul_rn keeps the
// product out of FMA contraction with a following add, which would skip that rounding.
template <bool POW2>
__device__ __forceinline__ float over_h(float x, const StepParams& P) {
    if constexpr (POW2) return __fmul_rn(x, P.inv_h);
    else return x / P.h;
}

// Field kinds: 0,1,2 = MAC face component of that axis; 3 = density; 4 = temperature.
template <int KIND>
__device__ __forceinline__ bool periodic_axis(const StepParams& P, int a) {
    if constexpr (KIND < 3) return P.fper[a] != 0;
    else if constexpr (KIND == 3) return P.dper[a] != 0;
    else return P.tper[a] != 0;
}

// Boundary-aware taps and interpolation with a runtime field kind. Only reached when some tap of a sample lies
// outside the array (near the domain edge), so it is kept out of line: inlining the ghost rules into every tap of
// every sampler made the advection kernels miss in the instruction cache.
__device__ __noinline__ inline float tap_rt(const float* __restrict__ f, int kind, int i, int j, int k, const StepParams& P) {
    switch (kind) {
    case 0: return face_tap_slow<0>(f, i, j, k, P);
    case 1: return face_tap_slow<1>(f, i, j, k, P);
    case 2: return face_tap_slow<2>(f, i, j, k, P);
    case 3: return scalar_tap_slow(f, i, j, k, P, P.den, P.dper);
    default: return scalar_tap_slow(f, i, j, k, P, P.tem, P.tper);
    }
}

__device__ __noinline__ inline float sample_edge(const float* __restrict__ f, int kind, int cubic, int x0, int y0, int z0, float tx, float ty, float tz, const StepParams& P) {
    if (!cubic) {
        const float c000 = tap_rt(f, kind, x0, y0, z0, P), c100 = tap_rt(f, kind, x0 + 1, y0, z0, P);
        const float c010 = tap_rt(f, kind, x0, y0 + 1, z0, P), c110 = tap_rt(f, kind, x0 + 1, y0 + 1, z0, P);
        const float c001 = tap_rt(f, kind, x0, y0, z0 + 1, P), c101 = tap_rt(f, kind, x0 + 1, y0, z0 + 1, P);
        const float c011 = tap_rt(f, kind, x0, y0 + 1, z0 + 1, P), c111 = tap_rt(f, kind, x0 + 1, y0 + 1, z0 + 1, P);
        const float c00 = c000 + (c100 - c000) * tx;
        const float c10 = c010 + (c110 - c010) * tx;
        const float c01 = c001 + (c101 - c001) * tx;
        const float c11 = c011 + (c111 - c011) * tx;
        const float c0 = c00 + (c10 - c00) * ty;
        const float c1 = c01 + (c11 - c01) * ty;
        return c0 + (c1 - c0) * tz;
    }
    float zs[4];
#pragma unroll 1
    for (int dz = 0; dz < 4; ++dz) {
        float ys[4];
#pragma unroll 1
        for (int dy = 0; dy < 4; ++dy) {
            const int yy = y0 + dy - 1, zz = z0 + dz - 1;
            ys[dy] = mono_cubic(tap_rt(f, kind, x0 - 1, yy, zz, P), tap_rt(f, kind, x0, yy, zz, P), tap_rt(f, kind, x0 + 1, yy, zz, P), tap_rt(f, kind, x0 + 2, yy, zz, P), tx);
        }
        zs[dz] = mono_cubic(ys[0], ys[1], ys[2], ys[3], ty);
    }
    return mono_cubic(zs[0], zs[1], zs[2], zs[3], tz);
}

// ---------------------------------------------------------------------------------------------- padded fields
// A sampled field copied with kPad ghost cells on every side, each ghost cell holding exactly the boundary tap of
// its index (face_tap_slow / scalar_tap_slow), so that a sample whose taps all lie within kPad cells of the array
// is one plain tensor of loads with no per-tap test. Samples of points inside the domain always qualify; `raw` (the
// unpadded field) serves the rare sample reaching further out, through sample_edge.
constexpr int kPad = 2;
struct PadField {
    const float* p;    // padded array, index (k + kPad) * pxy + (j + kPad) * px + (i + kPad)
    const float* raw;  // the field itself
    uint32_t px, pxy;  // padded row and slab pitch
};

// Tensor monotone cubic of the 4 x 4 x 4 taps at f (x fastest; row pitch sy, slab pitch sz): 16 cubics along x, 4 along
// y, 1 along z, the scalar mono_cubic's arithmetic. The x cubics run two rows per paired instruction, the y cubics two
// slabs per instruction.
__device__ __forceinline__ float cubic_taps(const float* __restrict__ f, uint32_t sy, uint32_t sz, float tx, float ty, float tz) {
    const HermiteW wx = hermite_weights(tx), wy = hermite_weights(ty);
    const HermiteW2 wx2 = hermite_pair(wx, wx), wy2 = hermite_pair(wy, wy);
    float ys[4][4];
#pragma unroll
    for (int dz = 0; dz < 4; ++dz)
#pragma unroll
        for (int dy = 0; dy < 4; dy += 2) {
            const float* r0 = f + dz * sz + dy * sy;
            const float* r1 = r0 + sy;
            const f32x2 c = mono_cubic2(f2_pack(__ldg(r0), __ldg(r1)), f2_pack(__ldg(r0 + 1), __ldg(r1 + 1)), f2_pack(__ldg(r0 + 2), __ldg(r1 + 2)), f2_pack(__ldg(r0 + 3), __ldg(r1 + 3)), wx2);
            f2_unpack(c, ys[dz][dy], ys[dz][dy + 1]);
        }
    float zs[4];
#pragma unroll
    for (int dz = 0; dz < 4; dz += 2) {
        const f32x2 c = mono_cubic2(f2_pack(ys[dz][0], ys[dz + 1][0]), f2_pack(ys[dz][1], ys[dz + 1][1]), f2_pack(ys[dz][2], ys[dz + 1][2]), f2_pack(ys[dz][3], ys[dz + 1][3]), wy2);
        f2_unpack(c, zs[dz], zs[dz + 1]);
    }
    return mono_cubic(zs[0], zs[1], zs[2], zs[3], tz);
}

// The same tensor cubic for two fields with the same tap box (lane 0: f, lane 1: g), every cubic one paired
// instruction stream for both.
__device__ __forceinline__ void cubic_taps_pair(const float* __restrict__ f, const float* __restrict__ g, uint32_t sy, uint32_t sz, float tx, float ty, float tz, float& out_f, float& out_g) {
    const HermiteW wx = hermite_weights(tx), wy = hermite_weights(ty), wz = hermite_weights(tz);
    const HermiteW2 wx2 = hermite_pair(wx, wx), wy2 = hermite_pair(wy, wy), wz2 = hermite_pair(wz, wz);
    f32x2 zs[4];
#pragma unroll
    for (int dz = 0; dz < 4; ++dz) {
        f32x2 ys[4];
#pragma unroll
        for (int dy = 0; dy < 4; ++dy) {
            const uint32_t o = dz * sz + dy * sy;
            ys[dy] = mono_cubic2(f2_pack(__ldg(f + o), __ldg(g + o)), f2_pack(__ldg(f + o + 1), __ldg(g + o + 1)), f2_pack(__ldg(f + o + 2), __ldg(g + o + 2)), f2_pack(__ldg(f + o + 3), __ldg(g + o + 3)), wx2);
        }
        zs[dz] = mono_cubic2(ys[0], ys[1], ys[2], ys[3], wy2);
    }
    f2_unpack(mono_cubic2(zs[0], zs[1], zs[2], zs[3], wz2), out_f, out_g);
}

// Samples field KIND at world position (x,y,z): periodic wrap of the position, conversion to grid coordinates
// (cell-centred axes offset by -0.5, backend-cuda.cu:413-415, 505-507), then trilinear (8 taps) or tensor monotone
// cubic (64 taps) from the padded copy; a tap box reaching beyond the padding goes through sample_edge.
template <int KIND, bool CUBIC, bool POW2>
__device__ __forceinline__ float sample_pad(const PadField& F, float x, float y, float z, const StepParams& P) {
    if (periodic_axis<KIND>(P, 0)) x = wrap_pos(x, P.nx, P.h);
    if (periodic_axis<KIND>(P, 1)) y = wrap_pos(y, P.ny, P.h);
    if (periodic_axis<KIND>(P, 2)) z = wrap_pos(z, P.nz, P.h);
    const float gx = KIND == 0 ? over_h<POW2>(x, P) : over_h<POW2>(x, P) - 0.5f;
    const float gy = KIND == 1 ? over_h<POW2>(y, P) : over_h<POW2>(y, P) - 0.5f;
    const float gz = KIND == 2 ? over_h<POW2>(z, P) : over_h<POW2>(z, P) - 0.5f;
    const int x0 = static_cast<int>(floorf(gx));
    const int y0 = static_cast<int>(floorf(gy));
    const int z0 = static_cast<int>(floorf(gz));
    const float tx = gx - static_cast<float>(x0);
    const float ty = gy - static_cast<float>(y0);
    const float tz = gz - static_cast<float>(z0);
    const int ex = P.nx + (KIND == 0) - 1, ey = P.ny + (KIND == 1) - 1, ez = P.nz + (KIND == 2) - 1;  // last indices
    const uint32_t sy = F.px, sz = F.pxy;
    if constexpr (!CUBIC) {
        // taps x0 .. x0+1 within [-kPad, ex+kPad]; written so that saturated conversions cannot overflow the test
        if (!(x0 >= -kPad && x0 < ex + kPad && y0 >= -kPad && y0 < ey + kPad && z0 >= -kPad && z0 < ez + kPad)) return sample_edge(F.raw, KIND, 0, x0, y0, z0, tx, ty, tz, P);
        const uint32_t b = static_cast<uint32_t>(z0 + kPad) * sz + static_cast<uint32_t>(y0 + kPad) * sy + static_cast<uint32_t>(x0 + kPad);
        const float* f = F.p;
        const float c000 = __ldg(f + b), c100 = __ldg(f + b + 1);
        const float c010 = __ldg(f + b + sy), c110 = __ldg(f + b + sy + 1);
        const float c001 = __ldg(f + b + sz), c101 = __ldg(f + b + sz + 1);
        const float c011 = __ldg(f + b + sz + sy), c111 = __ldg(f + b + sz + sy + 1);
        const float c00 = c000 + (c100 - c000) * tx;
        const float c10 = c010 + (c110 - c010) * tx;
        const float c01 = c001 + (c101 - c001) * tx;
        const float c11 = c011 + (c111 - c011) * tx;
        const float c0 = c00 + (c10 - c00) * ty;
        const float c1 = c01 + (c11 - c01) * ty;
        return c0 + (c1 - c0) * tz;
    } else {
        // taps x0-1 .. x0+2 within [-kPad, ex+kPad]
        if (!(x0 >= 1 - kPad && x0 <= ex + kPad - 2 && y0 >= 1 - kPad && y0 <= ey + kPad - 2 && z0 >= 1 - kPad && z0 <= ez + kPad - 2)) return sample_edge(F.raw, KIND, 1, x0, y0, z0, tx, ty, tz, P);
        const uint32_t base = static_cast<uint32_t>(z0 - 1 + kPad) * sz + static_cast<uint32_t>(y0 - 1 + kPad) * sy + static_cast<uint32_t>(x0 - 1 + kPad);
        return cubic_taps(F.p + base, sy, sz, tx, ty, tz);
    }
}

// Temperature (KIND 4) and density (KIND 3) at the same world position, as sample_pad<4> and sample_pad<3> give them.
// Both are cell-centred with padded copies of the same shape, so when their periodic axes agree and the cubic tap box
// lies within the padding, one tap box serves both and the cubic runs with the fields in the two lanes.
template <bool CUBIC, bool POW2>
__device__ __forceinline__ void sample_pad_scalars(const PadField& T, const PadField& D, float x, float y, float z, const StepParams& P, float& out_t, float& out_d) {
    if (CUBIC && (P.tper[0] != 0) == (P.dper[0] != 0) && (P.tper[1] != 0) == (P.dper[1] != 0) && (P.tper[2] != 0) == (P.dper[2] != 0) && T.px == D.px && T.pxy == D.pxy) {
        float px = x, py = y, pz = z;
        if (P.dper[0]) px = wrap_pos(px, P.nx, P.h);
        if (P.dper[1]) py = wrap_pos(py, P.ny, P.h);
        if (P.dper[2]) pz = wrap_pos(pz, P.nz, P.h);
        const float gx = over_h<POW2>(px, P) - 0.5f, gy = over_h<POW2>(py, P) - 0.5f, gz = over_h<POW2>(pz, P) - 0.5f;
        const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
        const int ex = P.nx - 1, ey = P.ny - 1, ez = P.nz - 1;
        if (x0 >= 1 - kPad && x0 <= ex + kPad - 2 && y0 >= 1 - kPad && y0 <= ey + kPad - 2 && z0 >= 1 - kPad && z0 <= ez + kPad - 2) {
            const uint32_t base = static_cast<uint32_t>(z0 - 1 + kPad) * D.pxy + static_cast<uint32_t>(y0 - 1 + kPad) * D.px + static_cast<uint32_t>(x0 - 1 + kPad);
            cubic_taps_pair(T.p + base, D.p + base, D.px, D.pxy, gx - static_cast<float>(x0), gy - static_cast<float>(y0), gz - static_cast<float>(z0), out_t, out_d);
            return;
        }
    }
    out_t = sample_pad<4, CUBIC, POW2>(T, x, y, z, P);
    out_d = sample_pad<3, CUBIC, POW2>(D, x, y, z, P);
}

// Trilinear sample of field KIND at the start of a back-trace: the centre of face (i, j, k) of axis START (0-2) or of
// cell (i, j, k) (START = 3), for a power-of-two cell size. Its grid coordinate is then exact on every axis, with
// fraction 1/2 where exactly one of "START is this axis" and "KIND is this axis" holds and 0 otherwise, so only the
// taps of nonzero weight are read (1, 2 or 4 of 8) and every tap lies inside the padded copy. The blends are those of
// sample_pad; a tap of weight 0 enters there as c + (d - c) * 0, which is c for finite values (a zero may change sign,
// which the position arithmetic p - dt * v it feeds cannot see), so the sample is sample_pad's.
template <int KIND, int START>
__device__ __forceinline__ float start_sample(const PadField& F, int i, int j, int k) {
    constexpr bool hx = (START == 0) != (KIND == 0), hy = (START == 1) != (KIND == 1), hz = (START == 2) != (KIND == 2);
    const int x0 = (START == 0 && KIND != 0) ? i - 1 : i;
    const int y0 = (START == 1 && KIND != 1) ? j - 1 : j;
    const int z0 = (START == 2 && KIND != 2) ? k - 1 : k;
    const uint32_t sy = F.px, sz = F.pxy;
    const float* f = F.p + static_cast<uint32_t>(z0 + kPad) * sz + static_cast<uint32_t>(y0 + kPad) * sy + static_cast<uint32_t>(x0 + kPad);
    const float c000 = __ldg(f);
    float c00 = c000, c10 = 0.0f, c01 = 0.0f, c11 = 0.0f;
    if constexpr (hx) c00 = c000 + (__ldg(f + 1) - c000) * 0.5f;
    if constexpr (hy) {
        const float c010 = __ldg(f + sy);
        c10 = hx ? c010 + (__ldg(f + sy + 1) - c010) * 0.5f : c010;
    }
    if constexpr (hz) {
        const float c001 = __ldg(f + sz);
        c01 = hx ? c001 + (__ldg(f + sz + 1) - c001) * 0.5f : c001;
        if constexpr (hy) {
            const float c011 = __ldg(f + sz + sy);
            c11 = hx ? c011 + (__ldg(f + sz + sy + 1) - c011) * 0.5f : c011;
        }
    }
    const float c0 = hy ? c00 + (c10 - c00) * 0.5f : c00;
    if constexpr (!hz) return c0;
    const float c1 = hy ? c01 + (c11 - c01) * 0.5f : c01;
    return c0 + (c1 - c0) * 0.5f;
}

// The boundary tap of field KIND at any integer index (the value a ghost cell of the padded copy holds).
template <int KIND>
__device__ __forceinline__ float boundary_tap(const float* __restrict__ f, int i, int j, int k, const StepParams& P) {
    if constexpr (KIND < 3) return face_tap_slow<KIND>(f, i, j, k, P);
    else if constexpr (KIND == 3) return scalar_tap_slow(f, i, j, k, P, P.den, P.dper);
    else return scalar_tap_slow(f, i, j, k, P, P.tem, P.tper);
}

// ---------------------------------------------------------------------------------------------- trace
// End-point / probe test of the back-trace (backend-cuda.cu:781-812): outside [0, n*h] on a non-periodic
// axis, or inside a solid cell.
template <bool POW2>
__device__ __forceinline__ bool blocked(float x, float y, float z, const uint8_t* __restrict__ occ, const StepParams& P) {
    if (P.fper[0]) x = wrap_pos(x, P.nx, P.h);
    if (P.fper[1]) y = wrap_pos(y, P.ny, P.h);
    if (P.fper[2]) z = wrap_pos(z, P.nz, P.h);
    if (x < 0.0f || x > static_cast<float>(P.nx) * P.h || y < 0.0f || y > static_cast<float>(P.ny) * P.h || z < 0.0f || z > static_cast<float>(P.nz) * P.h) return true;
    int cx = static_cast<int>(floorf(over_h<POW2>(x, P)));
    int cy = static_cast<int>(floorf(over_h<POW2>(y, P)));
    int cz = static_cast<int>(floorf(over_h<POW2>(z, P)));
    if (cx == P.nx) cx = P.nx - 1;
    if (cy == P.ny) cy = P.ny - 1;
    if (cz == P.nz) cz = P.nz - 1;
    if (cx < 0 || cx >= P.nx || cy < 0 || cy >= P.ny || cz < 0 || cz >= P.nz) return true;
    return occ[cidx(P, cx, cy, cz)] != 0;
}

// Bisection of a blocked back-trace end point towards the start, 10 steps (backend-cuda.cu:760-838).
template <bool POW2>
__device__ __noinline__ float3 bisect_blocked(float sx, float sy, float sz, float tx, float ty, float tz, const uint8_t* __restrict__ occ, const StepParams& P) {
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 10; ++it) {
        const float mid = 0.5f * (lo + hi);
        if (blocked<POW2>(sx + (tx - sx) * mid, sy + (ty - sy) * mid, sz + (tz - sz) * mid, occ, P)) hi = mid;
        else lo = mid;
    }
    return make_float3(sx + (tx - sx) * lo, sy + (ty - sy) * lo, sz + (tz - sz) * lo);
}

// Midpoint RK2 back-trace through the face velocities (padded copies of u, v, w), trilinear samples; a blocked end
// point is pulled back towards the start by bisection (backend-cuda.cu:760-838). (sx, sy, sz) is the centre of face
// (i, j, k) of axis START, or of cell (i, j, k) for START = 3; with a power-of-two cell size the start samples use
// start_sample.
template <bool POW2, int START>
__device__ __forceinline__ float3 trace_rk2(float sx, float sy, float sz, int i, int j, int k, const PadField& u, const PadField& v, const PadField& w, const uint8_t* __restrict__ occ, const StepParams& P) {
    const float dt = P.dt;
    const float a0 = POW2 ? start_sample<0, START>(u, i, j, k) : sample_pad<0, false, POW2>(u, sx, sy, sz, P);
    const float b0 = POW2 ? start_sample<1, START>(v, i, j, k) : sample_pad<1, false, POW2>(v, sx, sy, sz, P);
    const float c0 = POW2 ? start_sample<2, START>(w, i, j, k) : sample_pad<2, false, POW2>(w, sx, sy, sz, P);
    const float mx = sx - 0.5f * dt * a0, my = sy - 0.5f * dt * b0, mz = sz - 0.5f * dt * c0;
    const float a1 = sample_pad<0, false, POW2>(u, mx, my, mz, P);
    const float b1 = sample_pad<1, false, POW2>(v, mx, my, mz, P);
    const float c1 = sample_pad<2, false, POW2>(w, mx, my, mz, P);
    const float tx = sx - dt * a1, ty = sy - dt * b1, tz = sz - dt * c1;
    if (!blocked<POW2>(tx, ty, tz, occ, P)) return make_float3(tx, ty, tz);
    return bisect_blocked<POW2>(sx, sy, sz, tx, ty, tz, occ, P);
}

// ---------------------------------------------------------------------------------------------- centred velocity
// Face -> cell average of component C at an in-range cell (backend-cuda.cu:859-868).
template <int C>
__device__ __forceinline__ float centred(const float* __restrict__ f, int x, int y, int z, const StepParams& P) {
    const uint32_t a = fidx<C>(P, x, y, z);
    const uint32_t step = C == 0 ? 1u : (C == 1 ? static_cast<uint32_t>(P.nx) : static_cast<uint32_t>(P.nx) * P.ny);
    return 0.5f * (__ldg(f + a) + __ldg(f + a + step));
}

// Centred component C at any cell index, with the ghost rule of backend-cuda.cu:228-274: across a wall,
// 2*wall - interior; OUTFLOW and FREE_SLIP-tangential -> interior; periodic wraps.
template <int C>
__device__ inline float centred_tap(const float* __restrict__ f, int x, int y, int z, const StepParams& P) {
    int c[3] = {x, y, z};
    const int n[3] = {P.nx, P.ny, P.nz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (c[a] < 0 || c[a] >= n[a]) {
            if (P.fper[a]) {
                c[a] = wrapi(c[a], n[a]);
            } else {
                int q[3];
#pragma unroll
                for (int b = 0; b < 3; ++b) q[b] = (b == a) ? (c[a] < 0 ? 0 : n[a] - 1) : clampi(c[b], 0, n[b] - 1);
                const float interior = centred<C>(f, q[0], q[1], q[2], P);
                const SmokeSimulationFlowBoundaryFaceDesc face = P.flow[2 * a + (c[a] < 0 ? 0 : 1)];
                if (face.type == kFlowOutflow) return interior;
                if (face.type == kFlowFreeSlip && C != a) return interior;
                return 2.0f * face_comp(face, C) - interior;
            }
        }
    }
    return centred<C>(f, c[0], c[1], c[2], P);
}

// Vorticity of the centred velocity at an in-range fluid cell: central differences / h (backend-cuda.cu:885-900).
// A cell one cell or more inside every wall reads its 12 centred values directly; others go through the ghost rules.
__device__ __forceinline__ float4 vorticity_at(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w, int x, int y, int z, const StepParams& P) {
    if (x > 0 && x < P.nx - 1 && y > 0 && y < P.ny - 1 && z > 0 && z < P.nz - 1) {
        const float hh = 0.5f * P.inv_h;
        const float dvz_dy = hh * (centred<2>(w, x, y + 1, z, P) - centred<2>(w, x, y - 1, z, P));
        const float dvy_dz = hh * (centred<1>(v, x, y, z + 1, P) - centred<1>(v, x, y, z - 1, P));
        const float dvx_dz = hh * (centred<0>(u, x, y, z + 1, P) - centred<0>(u, x, y, z - 1, P));
        const float dvz_dx = hh * (centred<2>(w, x + 1, y, z, P) - centred<2>(w, x - 1, y, z, P));
        const float dvy_dx = hh * (centred<1>(v, x + 1, y, z, P) - centred<1>(v, x - 1, y, z, P));
        const float dvx_dy = hh * (centred<0>(u, x, y + 1, z, P) - centred<0>(u, x, y - 1, z, P));
        const float wx = dvz_dy - dvy_dz, wy = dvx_dz - dvz_dx, wz = dvy_dx - dvx_dy;
        return make_float4(wx, wy, wz, sqrtf(wx * wx + wy * wy + wz * wz));
    }
    const float hh = 0.5f * P.inv_h;
    const float dvz_dy = hh * (centred_tap<2>(w, x, y + 1, z, P) - centred_tap<2>(w, x, y - 1, z, P));
    const float dvy_dz = hh * (centred_tap<1>(v, x, y, z + 1, P) - centred_tap<1>(v, x, y, z - 1, P));
    const float dvx_dz = hh * (centred_tap<0>(u, x, y, z + 1, P) - centred_tap<0>(u, x, y, z - 1, P));
    const float dvz_dx = hh * (centred_tap<2>(w, x + 1, y, z, P) - centred_tap<2>(w, x - 1, y, z, P));
    const float dvy_dx = hh * (centred_tap<1>(v, x + 1, y, z, P) - centred_tap<1>(v, x - 1, y, z, P));
    const float dvx_dy = hh * (centred_tap<0>(u, x, y + 1, z, P) - centred_tap<0>(u, x, y - 1, z, P));
    const float wx = dvz_dy - dvy_dz;
    const float wy = dvx_dz - dvz_dx;
    const float wz = dvy_dx - dvx_dy;
    return make_float4(wx, wy, wz, sqrtf(wx * wx + wy * wy + wz * wz));
}

// Cell coordinates of linear cell index q.
__device__ __forceinline__ void cell_xyz(const StepParams& P, uint32_t q, int& x, int& y, int& z) {
    const uint32_t zz = P.div_slab.div(q);
    const uint32_t rem = q - zz * static_cast<uint32_t>(P.nx) * P.ny;
    const uint32_t yy = P.div_nx.div(rem);
    x = static_cast<int>(rem - yy * P.nx);
    y = static_cast<int>(yy);
    z = static_cast<int>(zz);
}

// Face coordinates of linear face index q of axis A.
template <int A>
__device__ __forceinline__ void face_ijk(const StepParams& P, uint32_t q, int& i, int& j, int& k) {
    const uint32_t sx = fsx<A>(P), sy = fsy<A>(P);
    const uint32_t row = P.div_fx[A].div(q);
    const uint32_t kk = P.div_fy[A].div(row);
    i = static_cast<int>(q - row * sx);
    j = static_cast<int>(row - kk * sy);
    k = static_cast<int>(kk);
}

#endif  // __CUDACC__

}  // namespace smoke_b200
