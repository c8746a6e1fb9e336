// Asynchronous z-marching ("2.5D") traversal used by the multigrid solver (mgpcg.cu).
//
// Same decomposition as march.cuh (32x8-cell columns, one own cell per thread, 84 in-plane halo slots, balanced
// column-plane ranges per block), but the inputs of each plane are copied global -> shared memory with cp.async
// into a ring of NS + 1 stages, NS - 1 planes ahead of the plane being computed. Registers then hold only the
// stencil values of three planes, so the look-ahead (and with it the number of loads in flight per SM) is set by
// shared memory, not by the register file.
//
// Per step (plane z of a column segment [za, zb)):
//   1. issue the copies of plane z + NS - 1 (one commit group per plane, empty when past zb);
//   2. wait until plane z + 2 has landed (cp.async.wait_group NS - 3), then __syncthreads;
//   3. compute the stencil value u of plane z + 2 for the own and the halo slot into ring[(z + 2) % 4];
//   4. run the own-cell callback of plane z, whose in-plane neighbours come from ring[z % 4] (written two steps
//      earlier) and whose -z/+z neighbours are registers.
// A stage is rewritten two steps after its plane was last read (NS + 1 stages), and the ring slot written in
// step 3 was last read two steps earlier, so one barrier per step orders every reuse. Stage entries written by a
// thread's cp.async are read only by that thread, except the pass's shared "extra" words (read after the barrier).
#pragma once

#include "launch.h"

namespace smoke_b200 {
namespace amarch {

constexpr int kThreads = 256;
constexpr int CX = 32, CY = 8;
constexpr int PX = CX + 2, PY = CY + 2;
constexpr int kPlane = PX * PY;
constexpr int kHalo = kPlane - CX * CY;  // 84
constexpr int kRing = 4;
static_assert(CX * CY == kThreads, "one column cell per thread");
static_assert(kHalo <= kThreads, "one halo slot per thread at most");

// 4-byte asynchronous copy global -> shared; ok == false zero-fills the destination without reading `src`.
__device__ __forceinline__ void cp4(void* dst, const void* src, bool ok) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(src), "r"(ok ? 4 : 0) : "memory");
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait_pending() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Extents and periodic axes of the grid being marched.
struct Geom {
    int nx, ny, nz;
    int per[3];
};

struct Columns {
    int ncx, ncy;
    uint32_t total;  // column-planes: ncx * ncy * nz
};

__host__ __device__ inline Columns columns_of(int nx, int ny, int nz) {
    Columns c;
    c.ncx = (nx + CX - 1) / CX;
    c.ncy = (ny + CY - 1) / CY;
    c.total = static_cast<uint32_t>(c.ncx) * c.ncy * nz;
    return c;
}

__device__ __forceinline__ bool wrap_axis(int& v, int n, int periodic) {
    if (v >= 0 && v < n) return true;
    if (!periodic) return false;
    v = wrapi(v, n);
    return true;
}

// This thread's slots in the current column: the own cell and (threads < kHalo) one halo cell. Coordinates are
// unwrapped (a halo slot across a periodic edge has x = -1 or x = nx); offsets are of the wrapped cell.
struct Slots {
    int x0, y0;
    int ox, oy, hx, hy;
    uint32_t ooff, hoff;  // in-plane offsets y * nx + x (valid when loaded)
    int oslot, hslot;     // ring positions
    bool oout;            // own cell inside the domain: produces output
    bool oload, hload;    // slot maps to a cell (possibly across a periodic edge)
    bool halo;            // this thread carries a halo slot
};

__device__ __forceinline__ Slots slots_of(const Geom& P, int x0, int y0) {
    Slots s;
    s.x0 = x0;
    s.y0 = y0;
    const int tx = threadIdx.x % CX, ty = threadIdx.x / CX;
    s.ox = x0 + tx;
    s.oy = y0 + ty;
    s.oslot = (ty + 1) * PX + tx + 1;
    s.oout = s.ox < P.nx && s.oy < P.ny;
    int wx = s.ox, wy = s.oy;
    s.oload = wrap_axis(wx, P.nx, P.per[0]) && wrap_axis(wy, P.ny, P.per[1]);
    s.ooff = s.oload ? static_cast<uint32_t>(wy) * P.nx + wx : 0u;
    s.halo = threadIdx.x < kHalo;
    s.hx = 0;
    s.hy = 0;
    s.hslot = 0;
    s.hload = false;
    s.hoff = 0;
    if (s.halo) {
        const int h = threadIdx.x;
        int hx, hy;
        if (h < PX) {
            hx = h - 1;
            hy = -1;
        } else if (h < 2 * PX) {
            hx = h - PX - 1;
            hy = CY;
        } else if (h < 2 * PX + CY) {
            hx = -1;
            hy = h - 2 * PX;
        } else {
            hx = CX;
            hy = h - 2 * PX - CY;
        }
        s.hslot = (hy + 1) * PX + hx + 1;
        s.hx = x0 + hx;
        s.hy = y0 + hy;
        int lx = s.hx, ly = s.hy;
        s.hload = wrap_axis(lx, P.nx, P.per[0]) && wrap_axis(ly, P.ny, P.per[1]);
        s.hoff = s.hload ? static_cast<uint32_t>(ly) * P.nx + lx : 0u;
    }
    return s;
}

// Offset of plane z (wrapped across a periodic edge); false outside the domain.
__device__ __forceinline__ bool plane_base(const Geom& P, int z, uint32_t& base) {
    if (!wrap_axis(z, P.nz, P.per[2])) return false;
    base = static_cast<uint32_t>(z) * static_cast<uint32_t>(P.nx) * P.ny;
    return true;
}

// The 16-bit operator code of cell q, from the 4-byte word holding it that was copied into shared memory
// (code arrays are read as aligned pairs and carry one spare element at the end).
__device__ __forceinline__ const void* code_word(const uint16_t* code, uint32_t q) { return code + (q & ~1u); }
__device__ __forceinline__ uint16_t code_of(uint32_t word, uint32_t q) { return static_cast<uint16_t>((q & 1u) ? (word >> 16) : (word & 0xffffu)); }

// March over every column segment of this block (see the file comment). NS >= 3 planes are in flight.
//   issue(s, stage, z, zok, base)           issue this thread's copies of plane z (unwrapped) into `stage`;
//                                           zok: the plane exists, base: its offset
//   value(s, stage, z, base, halo) -> float stencil value of the own (halo = false) or halo slot of plane z
//                                           (base: the plane's offset, 0 outside the domain)
//   own(s, stage, z, q, um1, u0, u1, plane, last)   plane z for the own cell; called by every thread (q is valid
//                                           when s.oout); `plane` is the ring plane of z; last: z + 1 == zb
template <int NS, class Issue, class Value, class Own>
__device__ __forceinline__ void march(const Geom& P, const Columns& C, float (*ring)[kPlane], Issue&& issue, Value&& value, Own&& own) {
    static_assert(NS >= 3, "at least three planes in flight");
    constexpr int NST = NS + 1;
    const uint32_t a = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x) * C.total) / gridDim.x);
    const uint32_t b = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x + 1) * C.total) / gridDim.x);
    const int nz = P.nz;
    uint32_t L = a;
    while (L < b) {
        const int col = static_cast<int>(L / static_cast<uint32_t>(nz));
        const int za = static_cast<int>(L - static_cast<uint32_t>(col) * nz);
        const int zb = za + static_cast<int>(min(static_cast<uint32_t>(nz - za), b - L));
        L += static_cast<uint32_t>(zb - za);
        const Slots s = slots_of(P, (col % C.ncx) * CX, (col / C.ncx) * CY);
        // plane z = za - 1 + rel lives in stage rel % NST and ring slot rel % kRing
        auto put = [&](int rel) {
            const int z = za - 1 + rel;
            if (z <= zb) {
                uint32_t base = 0;
                const bool zok = plane_base(P, z, base);
                issue(s, rel % NST, z, zok, base);
            }
            commit();
        };
        auto val = [&](int st, int z, bool halo) {
            uint32_t base = 0;
            plane_base(P, z, base);
            return value(s, st, z, base, halo);
        };
        for (int rel = 0; rel < NS; ++rel) put(rel);
        wait_pending<NS - 3>();
        __syncthreads();
        float um1 = val(0, za - 1, false);
        float u0 = val(1, za, false);
        float u1 = val(2, za + 1, false);
        ring[0][s.oslot] = um1;
        ring[1][s.oslot] = u0;
        ring[2][s.oslot] = u1;
        if (s.halo) {
            ring[0][s.hslot] = val(0, za - 1, true);
            ring[1][s.hslot] = val(1, za, true);
            ring[2][s.hslot] = val(2, za + 1, true);
        }
        for (int z = za; z < zb; ++z) {
            const int rel = z - za + 1;
            put(rel + NS - 1);
            wait_pending<NS - 3>();
            __syncthreads();
            float u2 = 0.0f;
            if (z + 2 <= zb) {
                const int st = (rel + 2) % NST, rs = (rel + 2) % kRing;
                u2 = val(st, z + 2, false);
                ring[rs][s.oslot] = u2;
                if (s.halo) ring[rs][s.hslot] = val(st, z + 2, true);
            }
            uint32_t q = 0;
            if (s.oout) {
                uint32_t base = 0;
                plane_base(P, z, base);
                q = base + s.ooff;
            }
            own(s, rel % NST, z, q, um1, u0, u1, ring[rel % kRing], z + 1 == zb);
            um1 = u0;
            u0 = u1;
            u1 = u2;
        }
        wait_pending<0>();
        __syncthreads();
    }
}

}  // namespace amarch
}  // namespace smoke_b200
