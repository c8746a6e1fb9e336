/*
 * TEST INFRASTRUCTURE -- the oracle. A plain-C restatement of the reference smoke step
 * (Xayah-Graphics/visual-simulation-of-smoke, backend-cuda.cu) used only by tests/, by the smoke() check
 * and by bench.py's CPU-baseline leg. The product library never links or calls it.
 *
 * One source, two builds: REAL=float ("mirror": same arithmetic type as the reference) and REAL=double
 * ("truth": the same algorithm in FP64). Each function names the reference lines whose behaviour it
 * restates. Where the reference kernels race (a domain face copying a neighbour face that another thread
 * of the same kernel writes, backend-cuda.cu:1023-1024 vs :1047-1063), this restatement uses the
 * sequential order "interior and solid faces first, then domain faces from the settled neighbour".
 *
 * Reductions (dot products) are accumulated in double over fixed z-slabs and summed in slab order, so a
 * result does not depend on the number of OpenMP threads.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "visual-simulation-of-smoke-3d.h"

#ifdef ORACLE_DOUBLE
typedef double real;
#define RFLOOR floor
#define RFMOD fmod
#define RSQRT sqrt
#define RFABS fabs
#define ORACLE_FN(name) oracle64_##name
#else
typedef float real;
#define RFLOOR floorf
#define RFMOD fmodf
#define RSQRT sqrtf
#define RFABS fabsf
#define ORACLE_FN(name) oracle32_##name
#endif
#define K(x) ((real)(x))

#define FLOW_NO_SLIP SMOKE_SIMULATION_FLOW_BOUNDARY_NO_SLIP_WALL
#define FLOW_FREE_SLIP SMOKE_SIMULATION_FLOW_BOUNDARY_FREE_SLIP_WALL
#define FLOW_OUTFLOW SMOKE_SIMULATION_FLOW_BOUNDARY_OUTFLOW
#define FLOW_PERIODIC SMOKE_SIMULATION_FLOW_BOUNDARY_PERIODIC
#define SCALAR_FIXED SMOKE_SIMULATION_SCALAR_BOUNDARY_FIXED_VALUE
#define SCALAR_ZERO_FLUX SMOKE_SIMULATION_SCALAR_BOUNDARY_ZERO_FLUX
#define SCALAR_PERIODIC SMOKE_SIMULATION_SCALAR_BOUNDARY_PERIODIC

typedef SmokeSimulationFlowBoundaryConfig FlowBC;
typedef SmokeSimulationScalarBoundaryConfig ScalarBC;
typedef SmokeSimulationFlowBoundaryFaceDesc FlowFace;

/* All state the step reads or writes. Arrays use the reference layouts (backend-cuda.cu:121-135). */
typedef struct OracleFields {
    real* u;
    real* v;
    real* w;
    real* temp_u;
    real* temp_v;
    real* temp_w;
    real* density;
    real* temperature;
    const real* density_source;
    const real* temperature_source;
    const real* force_x;
    const real* force_y;
    const real* force_z;
    const real* solid_velocity_x;
    const real* solid_velocity_y;
    const real* solid_velocity_z;
    const real* solid_temperature;
    const uint8_t* occupancy;
    real* pressure;
    real* pressure_rhs;
    real* centered_x;
    real* centered_y;
    real* centered_z;
    real* velocity_magnitude;
    real* vorticity_x;
    real* vorticity_y;
    real* vorticity_z;
    real* vorticity_magnitude;
    real* divergence;
} OracleFields;

enum { SOLVER_FIXED_CG = 0, SOLVER_JACOBI_PCG = 1 };

typedef struct OracleSolver {
    int32_t mode;            /* SOLVER_FIXED_CG (reference) or SOLVER_JACOBI_PCG */
    int32_t max_iterations;  /* FIXED_CG: ignored (config.pressure_iterations); PCG: cap */
    double tolerance;        /* PCG: relative residual target */
    int32_t iterations;      /* out */
    int32_t reserved;
    double relative_residual; /* out: recurrence residual at exit */
} OracleSolver;

/* ------------------------------------------------------------------ indexing, backend-cuda.cu:121-166 */
static inline size_t idx_c(int x, int y, int z, int nx, int ny) { return ((size_t)z * (size_t)ny + (size_t)y) * (size_t)nx + (size_t)x; }
static inline size_t idx_u(int i, int j, int k, int nx, int ny) { return ((size_t)k * (size_t)ny + (size_t)j) * (size_t)(nx + 1) + (size_t)i; }
static inline size_t idx_v(int i, int j, int k, int nx, int ny) { return ((size_t)k * (size_t)(ny + 1) + (size_t)j) * (size_t)nx + (size_t)i; }
static inline size_t idx_w(int i, int j, int k, int nx, int ny) { return ((size_t)k * (size_t)ny + (size_t)j) * (size_t)nx + (size_t)i; }

static inline int wrap(int value, int size) {
    if (size <= 0) return 0;
    value %= size;
    if (value < 0) value += size;
    return value;
}
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int in_bounds(int x, int y, int z, int nx, int ny, int nz) { return x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz; }
static inline int flow_periodic(FlowFace a, FlowFace b) { return a.type == FLOW_PERIODIC && b.type == FLOW_PERIODIC; }
static inline int scalar_periodic(SmokeSimulationScalarBoundaryFaceDesc a, SmokeSimulationScalarBoundaryFaceDesc b) { return a.type == SCALAR_PERIODIC && b.type == SCALAR_PERIODIC; }

typedef struct Grid {
    int nx, ny, nz;
    real h;
    FlowBC fb;
    int px, py, pz; /* flow periodic per axis */
} Grid;

/* resolve_cell_coordinates :146-151 */
static inline int resolve_flow(int* x, int* y, int* z, const Grid* g) {
    if (g->px && g->nx > 0) *x = wrap(*x, g->nx);
    if (g->py && g->ny > 0) *y = wrap(*y, g->ny);
    if (g->pz && g->nz > 0) *z = wrap(*z, g->nz);
    return in_bounds(*x, *y, *z, g->nx, g->ny, g->nz);
}

/* resolve_scalar_cell_coordinates :153-158 */
static inline int resolve_scalar(int* x, int* y, int* z, const Grid* g, const ScalarBC* sb) {
    if (scalar_periodic(sb->x_minus, sb->x_plus) && g->nx > 0) *x = wrap(*x, g->nx);
    if (scalar_periodic(sb->y_minus, sb->y_plus) && g->ny > 0) *y = wrap(*y, g->ny);
    if (scalar_periodic(sb->z_minus, sb->z_plus) && g->nz > 0) *z = wrap(*z, g->nz);
    return in_bounds(*x, *y, *z, g->nx, g->ny, g->nz);
}

/* load_occupancy :160-164: cells outside a non-periodic domain count as solid */
static inline int occupied(const uint8_t* occ, int x, int y, int z, const Grid* g) {
    if (occ == NULL) return 0;
    if (!resolve_flow(&x, &y, &z, g)) return 1;
    return occ[idx_c(x, y, z, g->nx, g->ny)] != 0;
}

/* load_scalar :166-200: FIXED -> value, ZERO_FLUX -> clamp, PERIODIC (both faces) -> wrap */
static real load_scalar(const real* f, int x, int y, int z, const Grid* g, const ScalarBC* sb) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    if (x < 0 || x >= nx) {
        SmokeSimulationScalarBoundaryFaceDesc face = x < 0 ? sb->x_minus : sb->x_plus;
        if (scalar_periodic(sb->x_minus, sb->x_plus) && nx > 0) x = wrap(x, nx);
        else if (face.type == SCALAR_ZERO_FLUX && nx > 0) x = x < 0 ? 0 : nx - 1;
        else return K(face.value);
    }
    if (y < 0 || y >= ny) {
        SmokeSimulationScalarBoundaryFaceDesc face = y < 0 ? sb->y_minus : sb->y_plus;
        if (scalar_periodic(sb->y_minus, sb->y_plus) && ny > 0) y = wrap(y, ny);
        else if (face.type == SCALAR_ZERO_FLUX && ny > 0) y = y < 0 ? 0 : ny - 1;
        else return K(face.value);
    }
    if (z < 0 || z >= nz) {
        SmokeSimulationScalarBoundaryFaceDesc face = z < 0 ? sb->z_minus : sb->z_plus;
        if (scalar_periodic(sb->z_minus, sb->z_plus) && nz > 0) z = wrap(z, nz);
        else if (face.type == SCALAR_ZERO_FLUX && nz > 0) z = z < 0 ? 0 : nz - 1;
        else return K(face.value);
    }
    return f[idx_c(x, y, z, nx, ny)];
}

/* load_flow_cell :202-226: clamp, or wrap on periodic axes */
static real load_flow_cell(const real* f, int x, int y, int z, const Grid* g) {
    if (x < 0 || x >= g->nx) x = (g->px && g->nx > 0) ? wrap(x, g->nx) : (x < 0 ? 0 : g->nx - 1);
    if (y < 0 || y >= g->ny) y = (g->py && g->ny > 0) ? wrap(y, g->ny) : (y < 0 ? 0 : g->ny - 1);
    if (z < 0 || z >= g->nz) z = (g->pz && g->nz > 0) ? wrap(z, g->nz) : (z < 0 ? 0 : g->nz - 1);
    return f[idx_c(x, y, z, g->nx, g->ny)];
}

static inline real face_component(FlowFace f, int axis) { return axis == 0 ? K(f.velocity_x) : (axis == 1 ? K(f.velocity_y) : K(f.velocity_z)); }

/* load_center_velocity_component :228-274: ghost = interior (OUTFLOW, or FREE_SLIP tangential),
 * else 2*prescribed - interior; the interior sample clamps the other coordinates */
static real load_center(const real* f, int axis, int x, int y, int z, const Grid* g) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    if (x < 0 || x >= nx) {
        FlowFace face = x < 0 ? g->fb.x_minus : g->fb.x_plus;
        if (g->px && nx > 0) x = wrap(x, nx);
        else {
            real interior = f[idx_c(x < 0 ? 0 : nx - 1, clampi(y, 0, ny - 1), clampi(z, 0, nz - 1), nx, ny)];
            if (face.type == FLOW_OUTFLOW) return interior;
            if (face.type == FLOW_FREE_SLIP && axis != 0) return interior;
            return K(2.0) * face_component(face, axis) - interior;
        }
    }
    if (y < 0 || y >= ny) {
        FlowFace face = y < 0 ? g->fb.y_minus : g->fb.y_plus;
        if (g->py && ny > 0) y = wrap(y, ny);
        else {
            real interior = f[idx_c(clampi(x, 0, nx - 1), y < 0 ? 0 : ny - 1, clampi(z, 0, nz - 1), nx, ny)];
            if (face.type == FLOW_OUTFLOW) return interior;
            if (face.type == FLOW_FREE_SLIP && axis != 1) return interior;
            return K(2.0) * face_component(face, axis) - interior;
        }
    }
    if (z < 0 || z >= nz) {
        FlowFace face = z < 0 ? g->fb.z_minus : g->fb.z_plus;
        if (g->pz && nz > 0) z = wrap(z, nz);
        else {
            real interior = f[idx_c(clampi(x, 0, nx - 1), clampi(y, 0, ny - 1), z < 0 ? 0 : nz - 1, nx, ny)];
            if (face.type == FLOW_OUTFLOW) return interior;
            if (face.type == FLOW_FREE_SLIP && axis != 2) return interior;
            return K(2.0) * face_component(face, axis) - interior;
        }
    }
    return f[idx_c(x, y, z, nx, ny)];
}

/* load_velocity_{x,y,z} :276-376. `axis` is the face-normal axis of the component. Along its own axis the
 * index range is [0, n]; a ghost is interior for OUTFLOW, else 2*prescribed - interior. Along the other two
 * axes the range is [0, n-1]; a ghost is interior for OUTFLOW and FREE_SLIP, else 2*prescribed - interior. */
static real load_face(const real* f, int axis, int i, int j, int k, const Grid* g) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const int sx = nx + (axis == 0), sy = ny + (axis == 1); /* array extents */
    int ext[3] = {nx + (axis == 0) - 1, ny + (axis == 1) - 1, nz + (axis == 2) - 1}; /* max valid index */
    int c[3] = {i, j, k};
    const int per[3] = {g->px, g->py, g->pz};
    const int n[3] = {nx, ny, nz};
    const FlowFace lo[3] = {g->fb.x_minus, g->fb.y_minus, g->fb.z_minus};
    const FlowFace hi[3] = {g->fb.x_plus, g->fb.y_plus, g->fb.z_plus};
    for (int a = 0; a < 3; ++a) {
        if (c[a] < 0 || c[a] > ext[a]) {
            FlowFace face = c[a] < 0 ? lo[a] : hi[a];
            if (per[a] && n[a] > 0) {
                c[a] = wrap(c[a], n[a]);
            } else {
                int q[3];
                for (int b = 0; b < 3; ++b) q[b] = (b == a) ? (c[a] < 0 ? 0 : ext[a]) : clampi(c[b], 0, ext[b]);
                real interior = f[((size_t)q[2] * (size_t)sy + (size_t)q[1]) * (size_t)sx + (size_t)q[0]];
                if (face.type == FLOW_OUTFLOW) return interior;
                if (a != axis && face.type == FLOW_FREE_SLIP) return interior;
                return K(2.0) * face_component(face, axis) - interior;
            }
        }
    }
    return f[((size_t)c[2] * (size_t)sy + (size_t)c[1]) * (size_t)sx + (size_t)c[0]];
}

/* monotonic_cubic_1d :378-392 */
static real mcubic(real p0, real p1, real p2, real p3, real t) {
    const real delta = p2 - p1;
    real m1 = K(0.5) * (p2 - p0);
    real m2 = K(0.5) * (p3 - p1);
    if (RFABS(delta) < K(1.0e-6)) {
        m1 = K(0.0);
        m2 = K(0.0);
    } else {
        if (m1 * delta <= K(0.0)) m1 = K(0.0);
        if (m2 * delta <= K(0.0)) m2 = K(0.0);
    }
    const real t2 = t * t;
    const real t3 = t2 * t;
    return (K(2.0) * t3 - K(3.0) * t2 + K(1.0)) * p1 + (t3 - K(2.0) * t2 + t) * m1 + (K(-2.0) * t3 + K(3.0) * t2) * p2 + (t3 - t2) * m2;
}

static inline real wrap_pos(real p, int n, real h) {
    const real extent = (real)n * h;
    p = RFMOD(p, extent);
    if (p < K(0.0)) p += extent;
    return p;
}

/* Generic sampler. kind: 0..2 = face component on that axis (load_velocity_*), 3 = cell-centred scalar.
 * Positions are wrapped on periodic axes of `pflags` first (:394-411, :486-503), then converted to grid
 * coordinates with an offset of -0.5 on cell-centred axes (:413-415, :505-507). cubic: tensor monotone
 * cubic over 4x4x4 taps (:443-484), else trilinear over 8 taps (:412-439). */
typedef struct Sampler {
    const real* f;
    int kind;
    const Grid* g;
    const ScalarBC* sb;
    int pflags[3];
} Sampler;

static inline real tap(const Sampler* s, int i, int j, int k) {
    if (s->kind == 3) return load_scalar(s->f, i, j, k, s->g, s->sb);
    return load_face(s->f, s->kind, i, j, k, s->g);
}

static real sample(const Sampler* s, real x, real y, real z, int cubic) {
    const Grid* g = s->g;
    if (s->pflags[0] && g->nx > 0) x = wrap_pos(x, g->nx, g->h);
    if (s->pflags[1] && g->ny > 0) y = wrap_pos(y, g->ny, g->h);
    if (s->pflags[2] && g->nz > 0) z = wrap_pos(z, g->nz, g->h);
    const real gx = (s->kind == 0) ? x / g->h : x / g->h - K(0.5);
    const real gy = (s->kind == 1) ? y / g->h : y / g->h - K(0.5);
    const real gz = (s->kind == 2) ? z / g->h : z / g->h - K(0.5);
    const int x0 = (int)RFLOOR(gx), y0 = (int)RFLOOR(gy), z0 = (int)RFLOOR(gz);
    const real tx = gx - (real)x0, ty = gy - (real)y0, tz = gz - (real)z0;
    if (!cubic) {
        const real c000 = tap(s, x0, y0, z0), c100 = tap(s, x0 + 1, y0, z0);
        const real c010 = tap(s, x0, y0 + 1, z0), c110 = tap(s, x0 + 1, y0 + 1, z0);
        const real c001 = tap(s, x0, y0, z0 + 1), c101 = tap(s, x0 + 1, y0, z0 + 1);
        const real c011 = tap(s, x0, y0 + 1, z0 + 1), c111 = tap(s, x0 + 1, y0 + 1, z0 + 1);
        const real c00 = c000 + (c100 - c000) * tx;
        const real c10 = c010 + (c110 - c010) * tx;
        const real c01 = c001 + (c101 - c001) * tx;
        const real c11 = c011 + (c111 - c011) * tx;
        const real c0 = c00 + (c10 - c00) * ty;
        const real c1 = c01 + (c11 - c01) * ty;
        return c0 + (c1 - c0) * tz;
    }
    real zs[4];
    for (int dz = 0; dz < 4; ++dz) {
        real ys[4];
        for (int dy = 0; dy < 4; ++dy) {
            const int yy = y0 + dy - 1, zz = z0 + dz - 1;
            ys[dy] = mcubic(tap(s, x0 - 1, yy, zz), tap(s, x0, yy, zz), tap(s, x0 + 1, yy, zz), tap(s, x0 + 2, yy, zz), tx);
        }
        zs[dz] = mcubic(ys[0], ys[1], ys[2], ys[3], ty);
    }
    return mcubic(zs[0], zs[1], zs[2], zs[3], tz);
}

static Sampler face_sampler(const real* f, int axis, const Grid* g) {
    Sampler s = {f, axis, g, NULL, {g->px, g->py, g->pz}};
    return s;
}

/* sample_velocity :756-758 (always trilinear) */
static void sample_velocity(const real* u, const real* v, const real* w, real x, real y, real z, const Grid* g, real out[3]) {
    Sampler su = face_sampler(u, 0, g), sv = face_sampler(v, 1, g), sw = face_sampler(w, 2, g);
    out[0] = sample(&su, x, y, z, 0);
    out[1] = sample(&sv, x, y, z, 0);
    out[2] = sample(&sw, x, y, z, 0);
}

/* The end-point / bisection-probe test of trace_particle_rk2 :781-812: outside [0, n*h] or in a solid cell */
static int hits_solid(real x, real y, real z, const uint8_t* occ, const Grid* g) {
    if (g->px && g->nx > 0) x = wrap_pos(x, g->nx, g->h);
    if (g->py && g->ny > 0) y = wrap_pos(y, g->ny, g->h);
    if (g->pz && g->nz > 0) z = wrap_pos(z, g->nz, g->h);
    int hit = x < K(0.0) || x > (real)g->nx * g->h || y < K(0.0) || y > (real)g->ny * g->h || z < K(0.0) || z > (real)g->nz * g->h;
    if (!hit && occ != NULL) {
        int cx = (int)RFLOOR(x / g->h), cy = (int)RFLOOR(y / g->h), cz = (int)RFLOOR(z / g->h);
        if (cx == g->nx) cx = g->nx - 1;
        if (cy == g->ny) cy = g->ny - 1;
        if (cz == g->nz) cz = g->nz - 1;
        hit = !in_bounds(cx, cy, cz, g->nx, g->ny, g->nz) || occ[idx_c(cx, cy, cz, g->nx, g->ny)] != 0;
    }
    return hit;
}

/* trace_particle_rk2 :760-838: midpoint RK2 back-trace; a blocked end point is pulled back by 10 bisection steps */
static void trace(real sx, real sy, real sz, const real* u, const real* v, const real* w, const uint8_t* occ, real dt, const Grid* g, real out[3]) {
    real v0[3], v1[3];
    sample_velocity(u, v, w, sx, sy, sz, g, v0);
    const real mx = sx - K(0.5) * dt * v0[0], my = sy - K(0.5) * dt * v0[1], mz = sz - K(0.5) * dt * v0[2];
    sample_velocity(u, v, w, mx, my, mz, g, v1);
    const real tx = sx - dt * v1[0], ty = sy - dt * v1[1], tz = sz - dt * v1[2];
    if (!hits_solid(tx, ty, tz, occ, g)) {
        out[0] = tx;
        out[1] = ty;
        out[2] = tz;
        return;
    }
    real lo = K(0.0), hi = K(1.0);
    for (int it = 0; it < 10; ++it) {
        const real mid = K(0.5) * (lo + hi);
        const real px = sx + (tx - sx) * mid, py = sy + (ty - sy) * mid, pz = sz + (tz - sz) * mid;
        if (hits_solid(px, py, pz, occ, g)) hi = mid;
        else lo = mid;
    }
    out[0] = sx + (tx - sx) * lo;
    out[1] = sy + (ty - sy) * lo;
    out[2] = sz + (tz - sz) * lo;
}

/* ------------------------------------------------------------------ per-stage restatement */
typedef struct Ctx {
    const SmokeSimulationConfig* cfg;
    Grid g;
    size_t n, nu, nv, nw;
} Ctx;

static Ctx make_ctx(const SmokeSimulationConfig* cfg) {
    Ctx c;
    c.cfg = cfg;
    c.g.nx = cfg->nx;
    c.g.ny = cfg->ny;
    c.g.nz = cfg->nz;
    c.g.h = K(cfg->cell_size);
    c.g.fb = cfg->flow_boundary;
    c.g.px = flow_periodic(cfg->flow_boundary.x_minus, cfg->flow_boundary.x_plus);
    c.g.py = flow_periodic(cfg->flow_boundary.y_minus, cfg->flow_boundary.y_plus);
    c.g.pz = flow_periodic(cfg->flow_boundary.z_minus, cfg->flow_boundary.z_plus);
    c.n = (size_t)cfg->nx * cfg->ny * cfg->nz;
    c.nu = (size_t)(cfg->nx + 1) * cfg->ny * cfg->nz;
    c.nv = (size_t)cfg->nx * (cfg->ny + 1) * cfg->nz;
    c.nw = (size_t)cfg->nx * cfg->ny * (cfg->nz + 1);
    return c;
}

/* apply_solid_temperature_kernel :1235-1241 */
static void apply_solid_temperature(const Ctx* c, OracleFields* f) {
    const real ambient = K(c->cfg->ambient_temperature);
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < (long long)c->n; ++q) {
        if (f->occupancy[q] == 0) continue;
        f->temperature[q] = f->solid_temperature ? f->solid_temperature[q] : ambient;
    }
}

/* compute_center_velocity_kernel :859-868 */
static void center_velocity(const Ctx* c, const real* u, const real* v, const real* w, real* cx, real* cy, real* cz) {
    const int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                cx[q] = K(0.5) * (u[idx_u(x, y, z, nx, ny)] + u[idx_u(x + 1, y, z, nx, ny)]);
                cy[q] = K(0.5) * (v[idx_v(x, y, z, nx, ny)] + v[idx_v(x, y + 1, z, nx, ny)]);
                cz[q] = K(0.5) * (w[idx_w(x, y, z, nx, ny)] + w[idx_w(x, y, z + 1, nx, ny)]);
            }
}

/* compute_vorticity_kernel :870-900 */
static void vorticity(const Ctx* c, const uint8_t* occ, const real* cx, const real* cy, const real* cz, real* wx, real* wy, real* wz, real* wm) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const real h = g->h;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                if (occupied(occ, x, y, z, g)) {
                    wx[q] = wy[q] = wz[q] = wm[q] = K(0.0);
                    continue;
                }
                const real dvz_dy = K(0.5) * (load_center(cz, 2, x, y + 1, z, g) - load_center(cz, 2, x, y - 1, z, g)) / h;
                const real dvy_dz = K(0.5) * (load_center(cy, 1, x, y, z + 1, g) - load_center(cy, 1, x, y, z - 1, g)) / h;
                const real dvx_dz = K(0.5) * (load_center(cx, 0, x, y, z + 1, g) - load_center(cx, 0, x, y, z - 1, g)) / h;
                const real dvz_dx = K(0.5) * (load_center(cz, 2, x + 1, y, z, g) - load_center(cz, 2, x - 1, y, z, g)) / h;
                const real dvy_dx = K(0.5) * (load_center(cy, 1, x + 1, y, z, g) - load_center(cy, 1, x - 1, y, z, g)) / h;
                const real dvx_dy = K(0.5) * (load_center(cx, 0, x, y + 1, z, g) - load_center(cx, 0, x, y - 1, z, g)) / h;
                const real a = dvz_dy - dvy_dz, b = dvx_dz - dvz_dx, d = dvy_dx - dvx_dy;
                wx[q] = a;
                wy[q] = b;
                wz[q] = d;
                wm[q] = RSQRT(a * a + b * b + d * d);
            }
}

/* solid_velocity_value :1007-1012 */
static real solid_velocity_value(const real* sv, const uint8_t* occ, int x, int y, int z, const Grid* g) {
    if (sv == NULL || occ == NULL) return K(0.0);
    if (!resolve_flow(&x, &y, &z, g)) return K(0.0);
    const size_t q = idx_c(x, y, z, g->nx, g->ny);
    if (occ[q] == 0) return K(0.0);
    return sv[q];
}

/* enforce_velocity_{x,y,z}_boundaries_kernel :1014-1168 and sync_periodic_velocity_* :1170-1189, for the
 * face component normal to `axis`. Interior faces touching a solid cell take the mean solid velocity of the
 * solid neighbours; non-periodic domain faces take the prescribed normal velocity, or for OUTFLOW the value the
 * adjacent interior face had when the kernel started (:1023-1024, :1030-1031: in the reference the copy and the
 * neighbour's solid rule run in the same kernel, and on B200 the copying thread reads first); then on periodic
 * axes face n copies face 0. */
static void enforce(const Ctx* c, real* f, int axis, const uint8_t* occ, const real* solid_v) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const int sx = nx + (axis == 0), sy = ny + (axis == 1), sz = nz + (axis == 2);
    const size_t total = (size_t)sx * sy * sz;
    real* before = (real*)malloc(total * sizeof(real));
    memcpy(before, f, total * sizeof(real));
    const int n_axis = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const FlowFace lo = axis == 0 ? g->fb.x_minus : (axis == 1 ? g->fb.y_minus : g->fb.z_minus);
    const FlowFace hi = axis == 0 ? g->fb.x_plus : (axis == 1 ? g->fb.y_plus : g->fb.z_plus);
    const int periodic = axis == 0 ? g->px : (axis == 1 ? g->py : g->pz);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < sz; ++k)
        for (int j = 0; j < sy; ++j)
            for (int i = 0; i < sx; ++i) {
                const int a = axis == 0 ? i : (axis == 1 ? j : k);
                if ((a == 0 && lo.type != FLOW_PERIODIC) || (a == n_axis && hi.type != FLOW_PERIODIC)) continue;
                if (occ == NULL) continue;
                int l[3] = {i, j, k}, r[3] = {i, j, k};
                l[axis] -= 1;
                const int has_l = resolve_flow(&l[0], &l[1], &l[2], g);
                const int has_r = resolve_flow(&r[0], &r[1], &r[2], g);
                const int lo_occ = has_l && occ[idx_c(l[0], l[1], l[2], nx, ny)] != 0;
                const int hi_occ = has_r && occ[idx_c(r[0], r[1], r[2], nx, ny)] != 0;
                if (!lo_occ && !hi_occ) continue;
                real value = K(0.0), weight = K(0.0);
                if (lo_occ) {
                    value += solid_velocity_value(solid_v, occ, l[0], l[1], l[2], g);
                    weight += K(1.0);
                }
                if (hi_occ) {
                    value += solid_velocity_value(solid_v, occ, r[0], r[1], r[2], g);
                    weight += K(1.0);
                }
                f[((size_t)k * sy + j) * sx + i] = weight > K(0.0) ? value / weight : K(0.0);
            }
    /* domain faces: OUTFLOW copies the adjacent face's value from before this pass */
#pragma omp parallel for schedule(static)
    for (int k = 0; k < sz; ++k)
        for (int j = 0; j < sy; ++j)
            for (int i = 0; i < sx; ++i) {
                const int a = axis == 0 ? i : (axis == 1 ? j : k);
                if (a != 0) continue;
                const size_t stride = axis == 0 ? 1 : (axis == 1 ? (size_t)sx : (size_t)sx * sy);
                const size_t base = ((size_t)k * sy + j) * sx + i;
                const size_t first = base, last = base + (size_t)n_axis * stride;
                real v_lo = f[first], v_hi = f[last];
                if (lo.type != FLOW_PERIODIC) v_lo = (lo.type == FLOW_OUTFLOW && n_axis > 0) ? before[first + stride] : face_component(lo, axis);
                if (hi.type != FLOW_PERIODIC) v_hi = (hi.type == FLOW_OUTFLOW && n_axis > 0) ? before[last - stride] : face_component(hi, axis);
                f[first] = v_lo;
                f[last] = v_hi;
                if (periodic) f[last] = f[first];
            }
    free(before);
}

/* Forces, backend-cuda.cu:2001-2018 (apply_solid_temperature, centre velocity, vorticity, seed_force,
 * add_buoyancy :910-918, add_confinement :920-948, add_center_forces_to_velocity_* :950-1005, enforce) */
static void stage_forces(const Ctx* c, OracleFields* f) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const SmokeSimulationConfig* cfg = c->cfg;
    const size_t n = c->n;
    apply_solid_temperature(c, f);
    center_velocity(c, f->u, f->v, f->w, f->centered_x, f->centered_y, f->centered_z);
    vorticity(c, f->occupancy, f->centered_x, f->centered_y, f->centered_z, f->vorticity_x, f->vorticity_y, f->vorticity_z, f->vorticity_magnitude);
    real* fx = (real*)malloc(n * sizeof(real));
    real* fy = (real*)malloc(n * sizeof(real));
    real* fz = (real*)malloc(n * sizeof(real));
    const real alpha = K(cfg->buoyancy_density_factor), beta = K(cfg->buoyancy_temperature_factor);
    const real ambient = K(cfg->ambient_temperature), eps = K(cfg->vorticity_confinement), h = g->h;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                fx[q] = f->force_x ? f->force_x[q] : K(0.0);
                fy[q] = f->force_y ? f->force_y[q] : K(0.0);
                fz[q] = f->force_z ? f->force_z[q] : K(0.0);
                if (occupied(f->occupancy, x, y, z, g)) continue;
                fy[q] += -alpha * f->density[q] + beta * (f->temperature[q] - ambient);
            }
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                if (occupied(f->occupancy, x, y, z, g)) continue;
                const real* m = f->vorticity_magnitude;
                const real gx = K(0.5) * (load_flow_cell(m, x + 1, y, z, g) - load_flow_cell(m, x - 1, y, z, g)) / h;
                const real gy = K(0.5) * (load_flow_cell(m, x, y + 1, z, g) - load_flow_cell(m, x, y - 1, z, g)) / h;
                const real gz = K(0.5) * (load_flow_cell(m, x, y, z + 1, g) - load_flow_cell(m, x, y, z - 1, g)) / h;
                const real gm = RSQRT(gx * gx + gy * gy + gz * gz);
                if (gm < K(1.0e-6)) continue;
                const real inv = K(1.0) / gm;
                const real nxv = gx * inv, nyv = gy * inv, nzv = gz * inv;
                const size_t q = idx_c(x, y, z, nx, ny);
                const real wx = f->vorticity_x[q], wy = f->vorticity_y[q], wz = f->vorticity_z[q];
                fx[q] += eps * h * (nyv * wz - nzv * wy);
                fy[q] += eps * h * (nzv * wx - nxv * wz);
                fz[q] += eps * h * (nxv * wy - nyv * wx);
            }
    const real dt = K(cfg->dt);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                real sum = K(0.0), wgt = K(0.0);
                if (i > 0) { sum += fx[idx_c(i - 1, j, k, nx, ny)]; wgt += K(1.0); }
                if (i < nx) { sum += fx[idx_c(i, j, k, nx, ny)]; wgt += K(1.0); }
                if (wgt > K(0.0)) f->u[idx_u(i, j, k, nx, ny)] += dt * (sum / wgt);
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i < nx; ++i) {
                real sum = K(0.0), wgt = K(0.0);
                if (j > 0) { sum += fy[idx_c(i, j - 1, k, nx, ny)]; wgt += K(1.0); }
                if (j < ny) { sum += fy[idx_c(i, j, k, nx, ny)]; wgt += K(1.0); }
                if (wgt > K(0.0)) f->v[idx_v(i, j, k, nx, ny)] += dt * (sum / wgt);
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                real sum = K(0.0), wgt = K(0.0);
                if (k > 0) { sum += fz[idx_c(i, j, k - 1, nx, ny)]; wgt += K(1.0); }
                if (k < nz) { sum += fz[idx_c(i, j, k, nx, ny)]; wgt += K(1.0); }
                if (wgt > K(0.0)) f->w[idx_w(i, j, k, nx, ny)] += dt * (sum / wgt);
            }
    free(fx);
    free(fy);
    free(fz);
    enforce(c, f->u, 0, f->occupancy, f->solid_velocity_x);
    enforce(c, f->v, 1, f->occupancy, f->solid_velocity_y);
    enforce(c, f->w, 2, f->occupancy, f->solid_velocity_z);
}

/* advect_velocity_{x,y,z}_kernel :1191-1219 then enforce :2025-2030 */
static void stage_advect_velocity(const Ctx* c, OracleFields* f) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const real h = g->h, dt = K(c->cfg->dt);
    const int cubic = c->cfg->scalar_advection_mode == SMOKE_SIMULATION_SCALAR_ADVECTION_MONOTONIC_CUBIC;
    real* dst[3] = {f->temp_u, f->temp_v, f->temp_w};
    const real* src[3] = {f->u, f->v, f->w};
    for (int axis = 0; axis < 3; ++axis) {
        const int sx = nx + (axis == 0), sy = ny + (axis == 1), sz = nz + (axis == 2);
        Sampler s = face_sampler(src[axis], axis, g);
#pragma omp parallel for schedule(dynamic, 1)
        for (int k = 0; k < sz; ++k)
            for (int j = 0; j < sy; ++j)
                for (int i = 0; i < sx; ++i) {
                    const real px = axis == 0 ? (real)i * h : ((real)i + K(0.5)) * h;
                    const real py = axis == 1 ? (real)j * h : ((real)j + K(0.5)) * h;
                    const real pz = axis == 2 ? (real)k * h : ((real)k + K(0.5)) * h;
                    real p[3];
                    trace(px, py, pz, f->u, f->v, f->w, f->occupancy, dt, g, p);
                    dst[axis][((size_t)k * sy + j) * sx + i] = sample(&s, p[0], p[1], p[2], cubic);
                }
    }
    enforce(c, f->temp_u, 0, f->occupancy, f->solid_velocity_x);
    enforce(c, f->temp_v, 1, f->occupancy, f->solid_velocity_y);
    enforce(c, f->temp_w, 2, f->occupancy, f->solid_velocity_z);
}

/* ------------------------------------------------------------------ pressure */
/* find_pressure_anchor :1292-1302: the smallest fluid cell index, or n when there is none */
static size_t pressure_anchor(const Ctx* c, const uint8_t* occ) {
    for (size_t q = 0; q < c->n; ++q)
        if (occ == NULL || occ[q] == 0) return q;
    return c->n;
}

/* Row structure of the Poisson operator, build_pressure_matrix_kernel :1343-1412 with the CSR pattern of
 * initialize_pressure_system :1688-1733: solid or anchor rows are identity; a fluid row has
 * diagonal = #fluid neighbours (anchor included, periodic wrap, duplicates counted) + #OUTFLOW domain faces
 * (at least 1) and -1 for each distinct fluid, non-anchor neighbour other than itself. */
typedef struct Row {
    real diag;
    int count;
    size_t nb[6];
} Row;

static void build_rows(const Ctx* c, const uint8_t* occ, size_t anchor, Row* rows) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                Row r;
                r.diag = K(0.0);
                r.count = 0;
                const int special = (occ != NULL && occ[q] != 0) || q == anchor;
                if (special) {
                    r.diag = K(1.0);
                    rows[q] = r;
                    continue;
                }
                const int d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
                for (int e = 0; e < 6; ++e) {
                    int a = e / 2;
                    int p[3] = {x + d[e][0], y + d[e][1], z + d[e][2]};
                    const int n3[3] = {nx, ny, nz};
                    const int per[3] = {g->px, g->py, g->pz};
                    if (p[a] < 0 || p[a] >= n3[a]) {
                        if (per[a]) {
                            p[a] = wrap(p[a], n3[a]);
                        } else {
                            const FlowFace lo = a == 0 ? g->fb.x_minus : (a == 1 ? g->fb.y_minus : g->fb.z_minus);
                            const FlowFace hi = a == 0 ? g->fb.x_plus : (a == 1 ? g->fb.y_plus : g->fb.z_plus);
                            const FlowFace face = p[a] < 0 ? lo : hi;
                            if (face.type == FLOW_OUTFLOW) r.diag += K(1.0);
                            continue;
                        }
                    }
                    const size_t nb = idx_c(p[0], p[1], p[2], nx, ny);
                    if (occ != NULL && occ[nb] != 0) continue;
                    r.diag += K(1.0);
                    if (nb == anchor) continue;
                    int dup = 0;
                    for (int t = 0; t < r.count; ++t) dup |= r.nb[t] == nb;
                    if (dup) continue;
                    r.nb[r.count++] = nb;
                }
                if (r.diag <= K(0.0)) r.diag = K(1.0);
                /* a neighbour equal to the row itself (periodic axis of length 1) only feeds the diagonal */
                int keep = 0;
                for (int t = 0; t < r.count; ++t)
                    if (r.nb[t] != q) r.nb[keep++] = r.nb[t];
                r.count = keep;
                rows[q] = r;
            }
}

static void apply_rows(const Ctx* c, const Row* rows, const real* p, real* out) {
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < (long long)c->n; ++q) {
        const Row* r = &rows[q];
        real acc = r->diag * p[q];
        for (int t = 0; t < r->count; ++t) acc -= p[r->nb[t]];
        out[q] = acc;
    }
}

/* Deterministic dot product: double partials per z-slab, summed in slab order. */
static double dot(const Ctx* c, const real* a, const real* b) {
    const int nz = c->g.nz;
    const size_t slab = (size_t)c->g.nx * c->g.ny;
    double* part = (double*)malloc((size_t)nz * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z) {
        double s = 0.0;
        const size_t base = (size_t)z * slab;
        for (size_t q = 0; q < slab; ++q) s += (double)a[base + q] * (double)b[base + q];
        part[z] = s;
    }
    double total = 0.0;
    for (int z = 0; z < nz; ++z) total += part[z];
    free(part);
    return total;
}

/* compute_pressure_rhs_kernel :1304-1328 */
static void pressure_rhs(const Ctx* c, const OracleFields* f, size_t anchor, real* rhs) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const real h = g->h, dt = K(c->cfg->dt);
    const FlowBC* b = &g->fb;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                if (q == anchor || (f->occupancy != NULL && f->occupancy[q] != 0)) {
                    rhs[q] = K(0.0);
                    continue;
                }
                const real div = (f->temp_u[idx_u(x + 1, y, z, nx, ny)] - f->temp_u[idx_u(x, y, z, nx, ny)] + f->temp_v[idx_v(x, y + 1, z, nx, ny)] - f->temp_v[idx_v(x, y, z, nx, ny)] + f->temp_w[idx_w(x, y, z + 1, nx, ny)] -
                                     f->temp_w[idx_w(x, y, z, nx, ny)]) /
                                 h;
                real bsum = K(0.0);
                if (x == 0 && b->x_minus.type == FLOW_OUTFLOW) bsum += K(b->x_minus.pressure);
                if (x == nx - 1 && b->x_plus.type == FLOW_OUTFLOW) bsum += K(b->x_plus.pressure);
                if (y == 0 && b->y_minus.type == FLOW_OUTFLOW) bsum += K(b->y_minus.pressure);
                if (y == ny - 1 && b->y_plus.type == FLOW_OUTFLOW) bsum += K(b->y_plus.pressure);
                if (z == 0 && b->z_minus.type == FLOW_OUTFLOW) bsum += K(b->z_minus.pressure);
                if (z == nz - 1 && b->z_plus.type == FLOW_OUTFLOW) bsum += K(b->z_plus.pressure);
                rhs[q] = -(h * h / dt) * div + bsum;
            }
}

/* solve_pressure_cg :1788-1824: x0 = 0, z = r, exactly `iterations` steps, ratios guarded by |den| > 1e-20 */
static void solve_fixed_cg(const Ctx* c, const Row* rows, const real* b, real* x, int iterations, OracleSolver* s) {
    const size_t n = c->n;
    real* r = (real*)malloc(n * sizeof(real));
    real* p = (real*)malloc(n * sizeof(real));
    real* q = (real*)malloc(n * sizeof(real));
    memset(x, 0, n * sizeof(real));
    memcpy(r, b, n * sizeof(real));
    memcpy(p, r, n * sizeof(real));
    real rz = (real)dot(c, r, r);
    for (int it = 0; it < iterations; ++it) {
        apply_rows(c, rows, p, q);
        const real pq = (real)dot(c, p, q);
        const real alpha = RFABS(pq) > K(1.0e-20) ? rz / pq : K(0.0);
#pragma omp parallel for schedule(static)
        for (long long t = 0; t < (long long)n; ++t) {
            x[t] += alpha * p[t];
            r[t] += -alpha * q[t];
        }
        const real rr = (real)dot(c, r, r);
        const real beta = RFABS(rz) > K(1.0e-20) ? rr / rz : K(0.0);
#pragma omp parallel for schedule(static)
        for (long long t = 0; t < (long long)n; ++t) p[t] = r[t] + beta * p[t];
        rz = rr;
    }
    const double bb = dot(c, b, b);
    s->iterations = iterations;
    s->relative_residual = bb > 0.0 ? sqrt(dot(c, r, r) / bb) : 0.0;
    free(r);
    free(p);
    free(q);
}

/* Jacobi-preconditioned CG to ||r|| <= tol ||b|| (FP64 scalars) -- the library's JACOBI_PCG mode. */
static void solve_jacobi_pcg(const Ctx* c, const Row* rows, const real* b, real* x, int max_it, double tol, OracleSolver* s) {
    const size_t n = c->n;
    real* r = (real*)malloc(n * sizeof(real));
    real* p = (real*)malloc(n * sizeof(real));
    real* q = (real*)malloc(n * sizeof(real));
    real* zv = (real*)malloc(n * sizeof(real));
    memset(x, 0, n * sizeof(real));
    memcpy(r, b, n * sizeof(real));
    const double bb = dot(c, b, b);
    int it = 0;
    double rr = bb;
    if (bb > 0.0) {
#pragma omp parallel for schedule(static)
        for (long long t = 0; t < (long long)n; ++t) zv[t] = r[t] / rows[t].diag;
        memcpy(p, zv, n * sizeof(real));
        double rz = dot(c, r, zv);
        while (it < max_it && rr > tol * tol * bb) {
            apply_rows(c, rows, p, q);
            const double pq = dot(c, p, q);
            const double alpha = fabs(pq) > 1.0e-300 ? rz / pq : 0.0;
#pragma omp parallel for schedule(static)
            for (long long t = 0; t < (long long)n; ++t) {
                x[t] = (real)((double)x[t] + alpha * (double)p[t]);
                r[t] = (real)((double)r[t] - alpha * (double)q[t]);
                zv[t] = r[t] / rows[t].diag;
            }
            ++it;
            rr = dot(c, r, r);
            const double rz_new = dot(c, r, zv);
            const double beta = fabs(rz) > 1.0e-300 ? rz_new / rz : 0.0;
#pragma omp parallel for schedule(static)
            for (long long t = 0; t < (long long)n; ++t) p[t] = (real)((double)zv[t] + beta * (double)p[t]);
            rz = rz_new;
        }
    }
    s->iterations = it;
    s->relative_residual = bb > 0.0 ? sqrt(rr / bb) : 0.0;
    free(r);
    free(p);
    free(q);
    free(zv);
}

static void stage_pressure(const Ctx* c, OracleFields* f, OracleSolver* s) {
    const size_t anchor = pressure_anchor(c, f->occupancy);
    Row* rows = (Row*)malloc(c->n * sizeof(Row));
    build_rows(c, f->occupancy, anchor, rows);
    pressure_rhs(c, f, anchor, f->pressure_rhs);
    if (s->mode == SOLVER_JACOBI_PCG) solve_jacobi_pcg(c, rows, f->pressure_rhs, f->pressure, s->max_iterations, s->tolerance, s);
    else solve_fixed_cg(c, rows, f->pressure_rhs, f->pressure, c->cfg->pressure_iterations, s);
    free(rows);
}

/* project_velocity_{x,y,z}_kernel :1425-1600 (interior faces; the domain faces are settled by the enforce
 * pass that follows, :2035-2040), then temp velocity -> velocity (:2041-2043) */
static void project_axis(const Ctx* c, real* f, int axis, const real* p, const uint8_t* occ, const real* solid_v) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const int sx = nx + (axis == 0), sy = ny + (axis == 1), sz = nz + (axis == 2);
    const int n_axis = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const FlowFace lo = axis == 0 ? g->fb.x_minus : (axis == 1 ? g->fb.y_minus : g->fb.z_minus);
    const FlowFace hi = axis == 0 ? g->fb.x_plus : (axis == 1 ? g->fb.y_plus : g->fb.z_plus);
    const real h = g->h, dt = K(c->cfg->dt);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < sz; ++k)
        for (int j = 0; j < sy; ++j)
            for (int i = 0; i < sx; ++i) {
                const int a = axis == 0 ? i : (axis == 1 ? j : k);
                if ((a == 0 && lo.type != FLOW_PERIODIC) || (a == n_axis && hi.type != FLOW_PERIODIC)) continue;
                int l[3] = {i, j, k}, r[3] = {i, j, k};
                l[axis] -= 1;
                const int has_l = resolve_flow(&l[0], &l[1], &l[2], g);
                const int has_r = resolve_flow(&r[0], &r[1], &r[2], g);
                const int lo_occ = has_l && occ != NULL && occ[idx_c(l[0], l[1], l[2], nx, ny)] != 0;
                const int hi_occ = has_r && occ != NULL && occ[idx_c(r[0], r[1], r[2], nx, ny)] != 0;
                real* face = &f[((size_t)k * sy + j) * sx + i];
                if (lo_occ || hi_occ) {
                    real value = K(0.0), weight = K(0.0);
                    if (lo_occ) { value += solid_velocity_value(solid_v, occ, l[0], l[1], l[2], g); weight += K(1.0); }
                    if (hi_occ) { value += solid_velocity_value(solid_v, occ, r[0], r[1], r[2], g); weight += K(1.0); }
                    *face = weight > K(0.0) ? value / weight : K(0.0);
                    continue;
                }
                if (has_l && has_r) {
                    const real pr = p[idx_c(r[0], r[1], r[2], nx, ny)];
                    const real pl = p[idx_c(l[0], l[1], l[2], nx, ny)];
                    *face -= dt * (pr - pl) / h;
                }
            }
}

static void stage_project(const Ctx* c, OracleFields* f) {
    project_axis(c, f->temp_u, 0, f->pressure, f->occupancy, f->solid_velocity_x);
    project_axis(c, f->temp_v, 1, f->pressure, f->occupancy, f->solid_velocity_y);
    project_axis(c, f->temp_w, 2, f->pressure, f->occupancy, f->solid_velocity_z);
    enforce(c, f->temp_u, 0, f->occupancy, f->solid_velocity_x);
    enforce(c, f->temp_v, 1, f->occupancy, f->solid_velocity_y);
    enforce(c, f->temp_w, 2, f->occupancy, f->solid_velocity_z);
    memcpy(f->u, f->temp_u, c->nu * sizeof(real));
    memcpy(f->v, f->temp_v, c->nv * sizeof(real));
    memcpy(f->w, f->temp_w, c->nw * sizeof(real));
}

/* advect_scalar_kernel :1221-1233: solid cells -> 0, else trace from the cell centre with the flow BCs and
 * sample the scalar with its own BCs */
static void advect_scalar(const Ctx* c, const OracleFields* f, const real* src, real* dst, const ScalarBC* sb) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const real h = g->h, dt = K(c->cfg->dt);
    const int cubic = c->cfg->scalar_advection_mode == SMOKE_SIMULATION_SCALAR_ADVECTION_MONOTONIC_CUBIC;
    Sampler s = {src, 3, g, sb, {scalar_periodic(sb->x_minus, sb->x_plus), scalar_periodic(sb->y_minus, sb->y_plus), scalar_periodic(sb->z_minus, sb->z_plus)}};
#pragma omp parallel for schedule(dynamic, 1)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                if (occupied(f->occupancy, x, y, z, g)) {
                    dst[q] = K(0.0);
                    continue;
                }
                real p[3];
                trace(((real)x + K(0.5)) * h, ((real)y + K(0.5)) * h, ((real)z + K(0.5)) * h, f->u, f->v, f->w, f->occupancy, dt, g, p);
                dst[q] = sample(&s, p[0], p[1], p[2], cubic);
            }
}

/* boundary_fill_density_kernel :1243-1290: a solid cell takes the value of the fluid cell with the smallest
 * squared distance in the first non-empty Chebyshev shell (first in dz, dy, dx scan order on ties), else 0 */
static void fill_density(const Ctx* c, const uint8_t* occ, const real* src, real* dst, const ScalarBC* sb) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    int max_radius = nx;
    if (ny > max_radius) max_radius = ny;
    if (nz > max_radius) max_radius = nz;
#pragma omp parallel for schedule(dynamic, 1)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                if (occ == NULL || occ[q] == 0) {
                    dst[q] = src[q];
                    continue;
                }
                real out = K(0.0);
                for (int radius = 1; radius <= max_radius; ++radius) {
                    int found = 0, best_d2 = 0;
                    real best = K(0.0);
                    for (int dz = -radius; dz <= radius; ++dz)
                        for (int dy = -radius; dy <= radius; ++dy)
                            for (int dx = -radius; dx <= radius; ++dx) {
                                int sr = abs(dx);
                                if (abs(dy) > sr) sr = abs(dy);
                                if (abs(dz) > sr) sr = abs(dz);
                                if (sr != radius) continue;
                                int px = x + dx, py = y + dy, pz = z + dz;
                                if (!resolve_scalar(&px, &py, &pz, g, sb)) continue;
                                const size_t nb = idx_c(px, py, pz, nx, ny);
                                if (occ[nb] != 0) continue;
                                const int d2 = dx * dx + dy * dy + dz * dz;
                                if (!found || d2 < best_d2) {
                                    found = 1;
                                    best_d2 = d2;
                                    best = src[nb];
                                }
                            }
                    if (found) {
                        out = best;
                        break;
                    }
                }
                dst[q] = out;
            }
}

/* Scalars, backend-cuda.cu:2044-2052: temperature (source, advect, solid temperature), then density
 * (source, advect, nearest-fluid fill of solid cells) */
static void stage_scalars(const Ctx* c, OracleFields* f) {
    const size_t n = c->n;
    const real dt = K(c->cfg->dt);
    real* tmp = (real*)malloc(n * sizeof(real));
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < (long long)n; ++q) tmp[q] = f->temperature[q] + dt * (f->temperature_source ? f->temperature_source[q] : K(0.0));
    advect_scalar(c, f, tmp, f->temperature, &c->cfg->temperature_boundary);
    apply_solid_temperature(c, f);
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < (long long)n; ++q) tmp[q] = f->density[q] + dt * (f->density_source ? f->density_source[q] : K(0.0));
    advect_scalar(c, f, tmp, f->density, &c->cfg->density_boundary);
    fill_density(c, f->occupancy, f->density, tmp, &c->cfg->density_boundary);
    memcpy(f->density, tmp, n * sizeof(real));
    free(tmp);
}

/* Views, backend-cuda.cu:2053-2057: centre velocity, vorticity, divergence (:1330-1341), |u| (:1602-1609) */
static void stage_views(const Ctx* c, OracleFields* f) {
    const Grid* g = &c->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const real h = g->h;
    center_velocity(c, f->u, f->v, f->w, f->centered_x, f->centered_y, f->centered_z);
    vorticity(c, f->occupancy, f->centered_x, f->centered_y, f->centered_z, f->vorticity_x, f->vorticity_y, f->vorticity_z, f->vorticity_magnitude);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t q = idx_c(x, y, z, nx, ny);
                if (f->occupancy != NULL && f->occupancy[q] != 0) {
                    f->divergence[q] = K(0.0);
                    continue;
                }
                f->divergence[q] = (f->u[idx_u(x + 1, y, z, nx, ny)] - f->u[idx_u(x, y, z, nx, ny)] + f->v[idx_v(x, y + 1, z, nx, ny)] - f->v[idx_v(x, y, z, nx, ny)] + f->w[idx_w(x, y, z + 1, nx, ny)] - f->w[idx_w(x, y, z, nx, ny)]) / h;
            }
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < (long long)c->n; ++q) {
        const real a = f->centered_x[q], b = f->centered_y[q], d = f->centered_z[q];
        f->velocity_magnitude[q] = RSQRT(a * a + b * b + d * d);
    }
}

/* ------------------------------------------------------------------ exported entry points */
/* Runs stages first..last of one step (0 forces, 1 velocity advection, 2 pressure, 3 projection, 4 scalars,
 * 5 views). The reference runs all six in this order (backend-cuda.cu:2000-2057). */
int ORACLE_FN(step)(const SmokeSimulationConfig* cfg, OracleFields* f, OracleSolver* solver, int first, int last) {
    if (cfg == NULL || f == NULL || solver == NULL) return 1;
    Ctx c = make_ctx(cfg);
    for (int stage = first; stage <= last; ++stage) {
        switch (stage) {
        case 0: stage_forces(&c, f); break;
        case 1: stage_advect_velocity(&c, f); break;
        case 2: stage_pressure(&c, f, solver); break;
        case 3: stage_project(&c, f); break;
        case 4: stage_scalars(&c, f); break;
        case 5: stage_views(&c, f); break;
        default: return 2;
        }
    }
    return 0;
}

/* out = A x with the operator of the pressure stage (for residual checks of any solver's output). */
void ORACLE_FN(apply_pressure_operator)(const SmokeSimulationConfig* cfg, const uint8_t* occ, const real* x, real* out) {
    Ctx c = make_ctx(cfg);
    const size_t anchor = pressure_anchor(&c, occ);
    Row* rows = (Row*)malloc(c.n * sizeof(Row));
    build_rows(&c, occ, anchor, rows);
    apply_rows(&c, rows, x, out);
    free(rows);
}

/* Diagonal of the operator (1 on identity rows) and the anchor index. */
long long ORACLE_FN(pressure_diagonal)(const SmokeSimulationConfig* cfg, const uint8_t* occ, real* diag) {
    Ctx c = make_ctx(cfg);
    const size_t anchor = pressure_anchor(&c, occ);
    Row* rows = (Row*)malloc(c.n * sizeof(Row));
    build_rows(&c, occ, anchor, rows);
    for (size_t q = 0; q < c.n; ++q) diag[q] = rows[q].diag;
    free(rows);
    return (long long)anchor;
}

/* Solve A x = b on its own (mode/tolerance from `solver`), for standalone pressure-solve checks. */
void ORACLE_FN(solve_pressure)(const SmokeSimulationConfig* cfg, const uint8_t* occ, const real* b, real* x, OracleSolver* s) {
    Ctx c = make_ctx(cfg);
    const size_t anchor = pressure_anchor(&c, occ);
    Row* rows = (Row*)malloc(c.n * sizeof(Row));
    build_rows(&c, occ, anchor, rows);
    if (s->mode == SOLVER_JACOBI_PCG) solve_jacobi_pcg(&c, rows, b, x, s->max_iterations, s->tolerance, s);
    else solve_fixed_cg(&c, rows, b, x, cfg->pressure_iterations, s);
    free(rows);
}

/* Single samples, for unit tests of the interpolation rules. kind 0..2 = face component, 3 = scalar. */
double ORACLE_FN(sample)(const SmokeSimulationConfig* cfg, const real* field, int kind, int cubic, int use_density_bc, double x, double y, double z) {
    Ctx c = make_ctx(cfg);
    const ScalarBC* sb = use_density_bc ? &cfg->density_boundary : &cfg->temperature_boundary;
    Sampler s;
    if (kind == 3) {
        Sampler t = {field, 3, &c.g, sb, {scalar_periodic(sb->x_minus, sb->x_plus), scalar_periodic(sb->y_minus, sb->y_plus), scalar_periodic(sb->z_minus, sb->z_plus)}};
        s = t;
    } else {
        s = face_sampler(field, kind, &c.g);
    }
    return (double)sample(&s, (real)x, (real)y, (real)z, cubic);
}

double ORACLE_FN(monotonic_cubic)(double p0, double p1, double p2, double p3, double t) { return (double)mcubic((real)p0, (real)p1, (real)p2, (real)p3, (real)t); }

int ORACLE_FN(real_bytes)(void) { return (int)sizeof(real); }
