// z-marching ("2.5D") traversal shared by the persistent solver kernels (pcg.cu).
//
// The grid is cut into 32x8-cell columns; each block owns a fixed, balanced range of column-planes and walks each
// of its column segments in z. Every thread owns one (x, y) cell of the column, so one plane step costs one
// address add; the -z/+z neighbours of the stencil stay in registers and only the in-plane halo (84 slots around
// the 32x8 plane) goes through a three-plane ring in shared memory. Loads of plane z+2 are issued before plane z is
// computed. Halo cells across a periodic edge are loaded from the opposite side.
#pragma once

#include "launch.h"

namespace smoke_b200 {
namespace zmarch {

constexpr int kThreads = 256;
constexpr int CX = 32, CY = 8;
constexpr int PX = CX + 2, PY = CY + 2;
constexpr int kPlane = PX * PY;
constexpr int kHaloSlots = kPlane - CX * CY;
static_assert(kHaloSlots <= kThreads, "one halo slot per thread at most");
static_assert(CX * CY == kThreads, "one column cell per thread");

// Extents and periodic axes of the grid being marched.
struct MarchGeom {
    int nx, ny, nz;
    int per[3];
};

__host__ __device__ inline MarchGeom geom_of(int nx, int ny, int nz, const int* per) {
    MarchGeom g{nx, ny, nz, {per[0], per[1], per[2]}};
    return g;
}

__host__ inline uint32_t column_planes(const MarchGeom& g, int* ncx = nullptr, int* ncy = nullptr) {
    const int cx = (g.nx + CX - 1) / CX, cy = (g.ny + CY - 1) / CY;
    if (ncx) *ncx = cx;
    if (ncy) *ncy = cy;
    return static_cast<uint32_t>(cx) * cy * g.nz;
}

struct Columns {
    int ncx, ncy;
    uint32_t total;  // column-planes: ncx * ncy * nz
};

__device__ __forceinline__ bool wrap_axis(int& v, int n, int periodic) {
    if (v >= 0 && v < n) return true;
    if (!periodic) return false;
    v = wrapi(v, n);
    return true;
}

// Per-thread geometry of one column: the thread's own slot, and (threads < kHaloSlots) one halo slot of the ring.
struct ColumnGeo {
    uint32_t own_off, halo_off;  // in-plane offsets (y * nx + x) of the cells loaded into the slots
    int own_slot, halo_slot;
    int own_x, own_y, halo_x, halo_y;  // in-plane coordinates of those cells (wrapped)
    bool own_out;                // the own cell is inside the domain and produces output
    bool own_load, halo_load;    // the slot maps to a cell (possibly across a periodic edge)
};

__device__ __forceinline__ ColumnGeo column_geo(const MarchGeom& P, int x0, int y0) {
    ColumnGeo g;
    const int tx = threadIdx.x % CX, ty = threadIdx.x / CX;
    int gx = x0 + tx, gy = y0 + ty;
    g.own_slot = (ty + 1) * PX + tx + 1;
    g.own_out = gx < P.nx && gy < P.ny;
    g.own_load = wrap_axis(gx, P.nx, P.per[0]) && wrap_axis(gy, P.ny, P.per[1]);
    g.own_off = g.own_load ? static_cast<uint32_t>(gy) * P.nx + gx : 0u;
    g.own_x = gx;
    g.own_y = gy;
    g.halo_x = 0;
    g.halo_y = 0;
    g.halo_load = false;
    g.halo_slot = 0;
    g.halo_off = 0;
    if (threadIdx.x < kHaloSlots) {
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
        g.halo_slot = (hy + 1) * PX + hx + 1;
        int lx = x0 + hx, ly = y0 + hy;
        g.halo_load = wrap_axis(lx, P.nx, P.per[0]) && wrap_axis(ly, P.ny, P.per[1]);
        g.halo_off = g.halo_load ? static_cast<uint32_t>(ly) * P.nx + lx : 0u;
        g.halo_x = lx;
        g.halo_y = ly;
    }
    return g;
}

// Offset of plane z (wrapped across a periodic edge, z updated); false outside the domain.
__device__ __forceinline__ bool plane_base(const MarchGeom& P, int& z, uint32_t& base) {
    if (!wrap_axis(z, P.nz, P.per[2])) return false;
    base = static_cast<uint32_t>(z) * static_cast<uint32_t>(P.nx) * P.ny;
    return true;
}

// March over every column segment of this block. For each plane z of a segment [za, zb):
//   load(ok, q, own, x, y, z) -> Data      loads one slot's inputs (zero Data when !ok); (x, y, z) is the cell
//   ufn(Data) -> V                          the value whose stencil is taken
//   own(q, Data, um1, u0, u1, plane, slot, x, y, z)   the own cell's work at plane z (um1/u1: its -z/+z values)
// Planes of the ring are (z mod 3). One __syncthreads per plane step.
template <typename V, typename Data, class Load, class UFn, class Own>
__device__ __forceinline__ void march(const MarchGeom& P, const Columns& C, V (*ring)[kPlane], Load&& load, UFn&& ufn, Own&& own) {
    const uint32_t a = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x) * C.total) / gridDim.x);
    const uint32_t b = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x + 1) * C.total) / gridDim.x);
    const int nz = P.nz;
    uint32_t L = a;
    while (L < b) {
        const int col = static_cast<int>(L / static_cast<uint32_t>(nz));
        const int za = static_cast<int>(L - static_cast<uint32_t>(col) * nz);
        const int zb = za + static_cast<int>(min(static_cast<uint32_t>(nz - za), b - L));
        L += static_cast<uint32_t>(zb - za);
        const ColumnGeo g = column_geo(P, (col % C.ncx) * CX, (col / C.ncx) * CY);
        const bool halo = threadIdx.x < kHaloSlots;
        auto fetch = [&](int z, Data& own_d, Data& halo_d) {
            uint32_t base = 0;
            const bool pz = plane_base(P, z, base);
            own_d = load(pz && g.own_load, base + g.own_off, true, g.own_x, g.own_y, z);
            if (halo) halo_d = load(pz && g.halo_load, base + g.halo_off, false, g.halo_x, g.halo_y, z);
        };
        Data om1, o0, o1, o2, h0, h1, h2, hm1;
        fetch(za - 1, om1, hm1);
        fetch(za, o0, h0);
        fetch(za + 1, o1, h1);
        V um1 = ufn(om1);
        V u0 = ufn(o0);
        ring[za % 3][g.own_slot] = u0;
        if (halo) ring[za % 3][g.halo_slot] = ufn(h0);
        for (int z = za; z < zb; ++z) {
            if (z + 2 <= zb) fetch(z + 2, o2, h2);
            const V u1 = ufn(o1);
            ring[(z + 1) % 3][g.own_slot] = u1;
            if (halo) ring[(z + 1) % 3][g.halo_slot] = ufn(h1);
            __syncthreads();
            if (g.own_out) {
                uint32_t base = 0;
                int zz = z;
                plane_base(P, zz, base);
                own(base + g.own_off, o0, um1, u0, u1, ring[z % 3], g.own_slot, g.own_x, g.own_y, z);
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


}  // namespace zmarch
}  // namespace smoke_b200
