// Mask builders on the device: the node grid (type, BCs, node values) of a
// domain built from its geometric description instead of being uploaded.
//
//   Shape3D  (Grid3D::Build, Grid3D.cpp:854-898): every cell NODE_IN, the
//            triangles of the shapes rasterised as NODE_BOUND
//            (RasterPolygon :710-788 and RasterLine on each edge :790-809), the
//            outside found by a flood fill from cell (0,0,0) (FloodFill
//            :811-852), then NODE_IN / NODE_OUT cells get no-slip, v = 0,
//            T = baseT.  NODE_BOUND cells keep their previous BCs and values.
//   SeaNetCDF (Grid3D::Prepare3D_NetCDF, Grid3D.cpp:966-1075): water columns
//            from a depth map, the water next to land or air turned into
//            no-slip walls, and the two far faces into inflow/outflow valves.
//   Shape2D  (FluidSolver2D::Grid2D::Build, Grid2D.cpp:231-266): a 2D node grid
//            from polylines (moving ones as valves, fixed ones as walls) and a
//            flood fill; and Grid3D::Prepare2D (Grid3D.cpp:608-665): a 2D node
//            grid extruded in depth with a curved bottom.
//
// The arithmetic is the reference's FTYPE = float arithmetic step for step:
// every operation is an explicitly rounded intrinsic (no contraction into FMA,
// and the file is compiled with --fmad=false as well), sqrt and division are the
// IEEE-rounded ones, and float -> int conversions reproduce the x86-64
// truncating conversion the reference is compiled to (NaN and out-of-range
// values give INT_MIN).  The resulting masks are bit-identical to the
// reference's on the same input.
//
// Parallel structure.  Rasterisation runs one warp per triangle: the scanline
// walk (a running float sum, hence sequential) is computed by all lanes alike and
// the cells of each scanline span are split over the lanes; every write stores
// the same value (NODE_BOUND), so concurrent writers agree.  2D polylines write
// data that differ per cell, so there the last write in the reference's order is
// found first (a claim pass) and then carried out.  The flood fill is a
// fixed-point iteration of line scans along X, Y and Z, each of which turns a
// NODE_IN run into NODE_OUT when one of its ends touches a NODE_OUT cell; the fixed
// point is the connected component the reference's breadth-first search finds.
//
// Loops whose trip count the reference leaves to float arithmetic (a scanline
// walk that stops advancing, a span walked away from its end, a huge line) are
// bounded here; reaching a bound, or a write outside the grid, is reported in a
// status word instead of being carried out (in the reference those cases do not
// terminate or write outside the node array).
#include "adi_internal.cuh"

#include <climits>

namespace adi {

namespace {

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// (int)f as the reference's x86-64 build computes it (cvttss2si / cvttsd2si).
__device__ __forceinline__ int to_int(float f)
{
    return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : INT_MIN;
}
__device__ __forceinline__ int to_int(double f)
{
    return (f > -2147483649.0 && f < 2147483648.0) ? __double2int_rz(f) : INT_MIN;
}
// std::max(a, b) = (a < b) ? b : a, including its NaN behaviour
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

struct F2 {
    float x, y;
};
struct F3 {
    float x, y, z;
};

constexpr double COMP_EPS = 1e-8;   // Geometry.h:23

// GetIntersectHorizon (Grid3D.cpp:678-688): the point of segment p1-p2 at height p.y.
__device__ __forceinline__ F2 horizon(F2 p1, F2 p2, F2 p)
{
    F2 r;
    r.y = p.y;
    if ((double)fabsf(fsub(p1.y, p2.y)) < COMP_EPS) r.x = p.x;
    else r.x = fadd(p1.x, fdiv(fmul(fsub(p2.x, p1.x), fsub(r.y, p1.y)), fsub(p2.y, p1.y)));
    return r;
}

enum : int { ST_OUTSIDE = 0, ST_BOUNDED = 1 };

struct Grid {
    uint8_t *type;
    int nx, ny, nz;
    int *status;   // [0]: writes outside the grid skipped, [1]: loops stopped at their bound
};

__device__ __forceinline__ void set_bound(const Grid &g, int x, int y, int z)
{
    if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) {
        atomicAdd(&g.status[ST_OUTSIDE], 1);
        return;
    }
    g.type[((long long)x * g.ny + y) * g.nz + z] = NODE_BOUND;
}

// ProjectPointOnPolygon (Grid3D.cpp:690-708): the cell of the triangle's plane
// above point (i, j) of the projection plane.
__device__ __forceinline__ void project(const Grid &g, int dir, int i, int j, F2 t, F3 n, float d)
{
    const float nd = -d;
    if (dir == 0) {
        const int k = to_int(fdiv(fsub(nd, fadd(fmul(t.x, n.y), fmul(t.y, n.z))), n.x));
        if (k >= 0 && k < g.nx) set_bound(g, k, i, j);
    } else if (dir == 1) {
        const int k = to_int(fdiv(fsub(nd, fadd(fmul(t.x, n.x), fmul(t.y, n.z))), n.y));
        if (k >= 0 && k < g.ny) set_bound(g, i, k, j);
    } else {
        const int k = to_int(fdiv(fsub(nd, fadd(fmul(t.x, n.x), fmul(t.y, n.y))), n.z));
        if (k >= 0 && k < g.nz) set_bound(g, i, j, k);
    }
}

// Loop bounds: a walk of `steps` increments gets 2 * steps + 8 iterations, and
// no walk or span longer than this.
constexpr long long MAX_WALK = 1ll << 22;

// One scanline part of RasterPolygon (Grid3D.cpp:760-787): while p.y < ytop,
// project the span from p.x to the edge e1-e2 at p.y, then p += dp.
__device__ void scan_part(const Grid &g, int dir, F3 n, float d, F2 &p, F2 dp, float ytop, F2 e1, F2 e2, int di,
                          int steps, int lane)
{
    long long cap = 2ll * (steps > 0 ? steps : 0) + 8;
    if (cap > MAX_WALK) cap = MAX_WALK;
    long long it = 0;
    for (; p.y < ytop; it++) {
        if (it >= cap) {
            if (lane == 0) atomicAdd(&g.status[ST_BOUNDED], 1);
            return;
        }
        const int j = to_int(p.y);
        const int i0 = to_int(p.x);
        const int last = to_int(horizon(e1, e2, p).x);
        // for (i = i0; i != last + di; i += di): (last - i0) * di + 1 iterations
        // when that is >= 0; otherwise the reference's loop runs through the
        // whole int range.
        const long long cnt = ((long long)last - i0) * di + 1;
        if (cnt < 0 || cnt > MAX_WALK) {
            if (lane == 0) atomicAdd(&g.status[ST_BOUNDED], 1);
        } else {
            for (long long c = lane; c < cnt; c += 32) {
                const int i = i0 + (int)c * di;
                project(g, dir, i, j, F2{__int2float_rn(i), p.y}, n, d);
            }
        }
        p.x = fadd(p.x, dp.x);
        p.y = fadd(p.y, dp.y);
    }
}

// RasterLine (Grid3D.cpp:790-809) by one warp: the walk is computed by every
// lane, lane q writes the points q, q + 32, ...
__device__ void raster_line(const Grid &g, F3 p1, F3 p2, int lane)
{
    const F3 dv{fsub(p2.x, p1.x), fsub(p2.y, p1.y), fsub(p2.z, p1.z)};
    const int steps = to_int(smax(fabsf(dv.x), smax(fabsf(dv.y), fabsf(dv.z)))) + 1;
    if (steps > MAX_WALK) {
        if (lane == 0) atomicAdd(&g.status[ST_BOUNDED], 1);
        return;
    }
    const float s = fdiv(1.0f, __int2float_rn(steps));   // Vec3D::operator/ multiplies by 1/t
    const F3 dp{fmul(dv.x, s), fmul(dv.y, s), fmul(dv.z, s)};
    F3 p = p1;
    for (int i = 0; i <= steps; i++) {
        if ((i & 31) == lane) set_bound(g, to_int(p.x), to_int(p.y), to_int(p.z));
        p.x = fadd(p.x, dp.x);
        p.y = fadd(p.y, dp.y);
        p.z = fadd(p.z, dp.z);
    }
}

__device__ __forceinline__ bool near_equal(F3 a, F3 b)   // Vec3D::equal (Geometry.h:135-140)
{
    return (double)fabsf(fsub(a.x, b.x)) < COMP_EPS && (double)fabsf(fsub(a.y, b.y)) < COMP_EPS &&
           (double)fabsf(fsub(a.z, b.z)) < COMP_EPS;
}

// RasterPolygon (Grid3D.cpp:710-788) by one warp.
__device__ void raster_polygon(const Grid &g, F3 p1, F3 p2, F3 p3, int lane)
{
    if (near_equal(p1, p2) && near_equal(p1, p3)) return;
    // normal (p2 - p1) x (p3 - p1), normalised by 1 / length
    const F3 a{fsub(p2.x, p1.x), fsub(p2.y, p1.y), fsub(p2.z, p1.z)};
    const F3 b{fsub(p3.x, p1.x), fsub(p3.y, p1.y), fsub(p3.z, p1.z)};
    F3 n{fsub(fmul(a.y, b.z), fmul(a.z, b.y)), fsub(fmul(a.z, b.x), fmul(a.x, b.z)),
         fsub(fmul(a.x, b.y), fmul(a.y, b.x))};
    const float len = __fsqrt_rn(fadd(fadd(fmul(n.x, n.x), fmul(n.y, n.y)), fmul(n.z, n.z)));
    const float t = fdiv(1.0f, len);
    n.x = fmul(n.x, t);
    n.y = fmul(n.y, t);
    n.z = fmul(n.z, t);
    const float d = -fadd(fadd(fmul(p1.x, n.x), fmul(p1.y, n.y)), fmul(p1.z, n.z));

    // dominant axis of the normal; later axes win ties as in the reference
    const float maxv = smax(fabsf(n.x), smax(fabsf(n.y), fabsf(n.z)));
    int dir = -1;
    if ((double)fabsf(fsub(maxv, fabsf(n.x))) < COMP_EPS) dir = 0;
    if ((double)fabsf(fsub(maxv, fabsf(n.y))) < COMP_EPS) dir = 1;
    if ((double)fabsf(fsub(maxv, fabsf(n.z))) < COMP_EPS) dir = 2;
    // A degenerate triangle (collinear corners) has a NaN normal and no axis;
    // the reference then reads an unset axis.  Its edges are still rasterised.
    if (dir < 0) return;

    F2 q1, q2, q3;
    if (dir == 0) { q1 = F2{p1.y, p1.z}; q2 = F2{p2.y, p2.z}; q3 = F2{p3.y, p3.z}; }
    else if (dir == 1) { q1 = F2{p1.x, p1.z}; q2 = F2{p2.x, p2.z}; q3 = F2{p3.x, p3.z}; }
    else { q1 = F2{p1.x, p1.y}; q2 = F2{p2.x, p2.y}; q3 = F2{p3.x, p3.y}; }

    F2 m;
    if (q3.y < q2.y) { m = q3; q3 = q2; q2 = m; }
    if (q1.y > q2.y) { m = q1; q1 = q2; q2 = m; }
    if (q3.y < q2.y) { m = q3; q3 = q2; q2 = m; }

    const F2 mid = horizon(q1, q3, q2);
    const F2 d1{fsub(mid.x, q1.x), fsub(mid.y, q1.y)};
    const F2 d2{fsub(q3.x, mid.x), fsub(q3.y, mid.y)};
    const int steps1 = to_int(smax(fabsf(d1.x), fabsf(d1.y))) + 1;
    const int steps2 = to_int(smax(fabsf(d2.x), fabsf(d2.y))) + 1;
    const F2 dp1{fdiv(d1.x, __int2float_rn(steps1)), fdiv(d1.y, __int2float_rn(steps1))};
    const F2 dp2{fdiv(d2.x, __int2float_rn(steps2)), fdiv(d2.y, __int2float_rn(steps2))};
    F2 p = q1;
    const int di = (mid.x < q2.x) ? 1 : -1;
    scan_part(g, dir, n, d, p, dp1, mid.y, q1, q2, di, steps1, lane);
    scan_part(g, dir, n, d, p, dp2, q3.y, q2, q3, di, steps2, lane);
}

__global__ void __launch_bounds__(256) raster_triangles_kernel(Grid g, const float *__restrict__ verts,
                                                               const int *__restrict__ tris, int ntris, int nverts)
{
    const int tri = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (tri >= ntris) return;
    const int i1 = tris[3 * tri], i2 = tris[3 * tri + 1], i3 = tris[3 * tri + 2];
    if (i1 < 0 || i1 >= nverts || i2 < 0 || i2 >= nverts || i3 < 0 || i3 >= nverts) return;   // checked on the host
    const F3 v1{verts[3 * i1], verts[3 * i1 + 1], verts[3 * i1 + 2]};
    const F3 v2{verts[3 * i2], verts[3 * i2 + 1], verts[3 * i2 + 2]};
    const F3 v3{verts[3 * i3], verts[3 * i3 + 1], verts[3 * i3 + 2]};
    raster_polygon(g, v1, v2, v3, lane);
    // additionally rasterise the edges (Grid3D.cpp:869-872)
    raster_line(g, v1, v2, lane);
    raster_line(g, v1, v3, lane);
    raster_line(g, v3, v2, lane);
}

__global__ void fill_types_kernel(uint8_t *type, long long n, uint8_t v)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        type[c] = v;
}

// One flood-fill scan along direction DIR.  Each line is cut into chunks of
// `chunk` cells; one thread walks one chunk forward and another walks it backward
// (threads of neighbouring lines are neighbours, so X and Y scans coalesce).  A
// NODE_IN cell reached from a NODE_OUT cell through NODE_IN cells becomes NODE_OUT;
// a walk starts reached when the cell just before its chunk (in its direction) is
// NODE_OUT.  Cells only ever turn from NODE_IN to NODE_OUT, so walks that meet
// agree, and the passes repeat until one changes nothing: the fixed point is the
// connected component of the reference's breadth-first search.  Each walk reads
// U cells ahead (independent loads) before applying the sequential rule to them.
template <int DIR>
__global__ void flood_scan_kernel(uint8_t *type, int nx, int ny, int nz, int chunk, int *changed)
{
    const long long nlines = DIR == 0 ? (long long)ny * nz : (DIR == 1 ? (long long)nx * nz : (long long)nx * ny);
    const int len = DIR == 0 ? nx : (DIR == 1 ? ny : nz);
    const int nch = (len + chunk - 1) / chunk;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= nlines * nch * 2) return;
    const long long line = idx % nlines;
    const long long rest = idx / nlines;
    const int ch = (int)(rest % nch);
    const bool bwd = rest >= nch;
    long long base, stride;
    if (DIR == 0) { base = line; stride = (long long)ny * nz; }                               // (j, k)
    else if (DIR == 1) { base = (line / nz) * (long long)ny * nz + line % nz; stride = nz; }  // (i, k)
    else { base = line * nz; stride = 1; }                                                   // (i, j)
    const int p_lo = ch * chunk, p_hi = min(len, p_lo + chunk) - 1;
    constexpr int U = 8;
    uint8_t *row = type + base;
    bool any = false;
    if (!bwd) {
        bool reach = p_lo > 0 && row[(long long)(p_lo - 1) * stride] == NODE_OUT;
        for (int p0 = p_lo; p0 <= p_hi; p0 += U) {
            uint8_t t[U];
#pragma unroll
            for (int u = 0; u < U; u++) t[u] = (p0 + u <= p_hi) ? row[(long long)(p0 + u) * stride] : (uint8_t)NODE_BOUND;
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (t[u] == NODE_OUT) reach = true;
                else if (t[u] == NODE_IN) {
                    if (reach) { row[(long long)(p0 + u) * stride] = NODE_OUT; any = true; }
                } else reach = false;
            }
        }
    } else {
        bool reach = p_hi < len - 1 && row[(long long)(p_hi + 1) * stride] == NODE_OUT;
        for (int p1 = p_hi; p1 >= p_lo; p1 -= U) {
            uint8_t t[U];
#pragma unroll
            for (int u = 0; u < U; u++) t[u] = (p1 - u >= p_lo) ? row[(long long)(p1 - u) * stride] : (uint8_t)NODE_BOUND;
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (t[u] == NODE_OUT) reach = true;
                else if (t[u] == NODE_IN) {
                    if (reach) { row[(long long)(p1 - u) * stride] = NODE_OUT; any = true; }
                } else reach = false;
            }
        }
    }
    if (any) *changed = 1;
}

// The end of Grid3D::Build (Grid3D.cpp:880-897): NODE_IN and NODE_OUT cells get
// no-slip BCs, v = 0 and T = baseT; NODE_BOUND cells keep their BCs and values.
// The node values also become the initial state (cur).
template <typename R>
__global__ void shape_install_kernel(const uint8_t *__restrict__ type, uint8_t *code, Layer<R> nv, Layer<R> cur,
                                     long long n, R baseT)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const uint8_t t = type[c];
        if (t == NODE_BOUND) {
            code[c] = (uint8_t)(NODE_BOUND | (code[c] & (CODE_VEL_FREE | CODE_TEMP_FREE)));
        } else {
            code[c] = t;
            nv.f[0][c] = R(0);
            nv.f[1][c] = R(0);
            nv.f[2][c] = R(0);
            nv.f[3][c] = baseT;
        }
#pragma unroll
        for (int v = 0; v < 4; v++) cur.f[v][c] = nv.f[v][c];
    }
}

// ---------------------------------------------------------------------------
// SeaNetCDF
// ---------------------------------------------------------------------------

template <typename R>
__device__ __forceinline__ void set_node(uint8_t *code, Layer<R> nv, long long c, uint8_t type, float vx, float vy,
                                         float vz, float T)
{
    code[c] = type;   // both BCs no-slip in every write of the sea builder
    nv.f[0][c] = (R)vx;
    nv.f[1][c] = (R)vy;
    nv.f[2][c] = (R)vz;
    nv.f[3][c] = (R)T;
}

// Grid3D.cpp:968-977: every cell NODE_OUT with no-slip, v = 0, T = baseT.
template <typename R>
__global__ void sea_columns_kernel(uint8_t *code, Layer<R> nv, long long n, float baseT)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        set_node<R>(code, nv, c, NODE_OUT, 0.0f, 0.0f, 0.0f, baseT);
}

// Grid3D.cpp:979-997: the cells k = 1 .. bound_k - 1 of each water column
// NODE_IN.  The NODE_IN writes use the flat index i*ny*nz + j*nz + k as the
// reference does (a bound_k beyond nz reaches into the next columns); writes past
// the array are skipped and counted.
__global__ void sea_water_kernel(uint8_t *code, int nx, int ny, int nz, const float *__restrict__ depth, int dnx,
                                 int dny, float zmin, int *status)
{
    const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (col >= (long long)nx * ny) return;
    const int i = (int)(col / ny), j = (int)(col % ny);
    const int di = (int)((long long)i * dnx / nx);
    const int dj = (int)((long long)j * dny / ny);
    const float z = depth[dj + (long long)di * dny];
    if (!(z < 0.0f)) return;
    const int bound_k = to_int(fdiv(fmul(__int2float_rn(nz), z), zmin));
    const long long n = (long long)nx * ny * nz;
    const long long base = col * nz;
    if ((long long)bound_k - 1 > MAX_WALK) {
        atomicAdd(&status[ST_BOUNDED], 1);
        return;
    }
    for (int k = 1; k < bound_k; k++) {
        if (base + k >= n) {
            atomicAdd(&status[ST_OUTSIDE], 1);
            return;
        }
        code[base + k] = NODE_IN;   // the type only; the data stay those of the first pass
    }
}

// Grid3D.cpp:999-1013: interior NODE_IN cells with a NODE_OUT neighbour become
// no-slip walls (in place: the test reads NODE_OUT, which this pass never writes).
template <typename R>
__global__ void sea_wall_in_kernel(uint8_t *code, Layer<R> nv, int nx, int ny, int nz, float baseT)
{
    const long long n = (long long)nx * ny * nz;
    const long long sx = (long long)ny * nz, sy = nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c / sx), j = (int)((c / sy) % ny), k = (int)(c % nz);
        if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) continue;
        if ((code[c] & CODE_TYPE) != NODE_IN) continue;
        auto out = [&](long long q) { return (code[q] & CODE_TYPE) == NODE_OUT; };
        if (out(c - sx) || out(c + sx) || out(c - sy) || out(c + sy) || out(c - 1) || out(c + 1))
            set_node<R>(code, nv, c, NODE_BOUND, 0.0f, 0.0f, 0.0f, baseT);
    }
}

// Grid3D.cpp:1015-1034: interior NODE_OUT cells with a NODE_BOUND neighbour become
// walls; the reference collects them first, so the test reads a snapshot.
template <typename R>
__global__ void sea_wall_out_kernel(const uint8_t *__restrict__ snap, uint8_t *code, Layer<R> nv, int nx, int ny,
                                    int nz, float baseT)
{
    const long long n = (long long)nx * ny * nz;
    const long long sx = (long long)ny * nz, sy = nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c / sx), j = (int)((c / sy) % ny), k = (int)(c % nz);
        if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) continue;
        if ((snap[c] & CODE_TYPE) != NODE_OUT) continue;
        auto bnd = [&](long long q) { return (snap[q] & CODE_TYPE) == NODE_BOUND; };
        if (bnd(c - sx) || bnd(c + sx) || bnd(c - sy) || bnd(c + sy) || bnd(c - 1) || bnd(c + 1))
            set_node<R>(code, nv, c, NODE_BOUND, 0.0f, 0.0f, 0.0f, baseT);
    }
}

// Grid3D.cpp:1036-1074: the NODE_IN cells of the face line j = ny-1 (FACE 1, one
// thread per i) or i = nx-1 (FACE 0, one thread per j) become valves: inflow
// (bcInVel, bcInT) below the middle of the line's water, outflow (-bcInVel,
// 2 - bcInT) above it.
template <typename R, int FACE>
__global__ void sea_face_kernel(uint8_t *code, Layer<R> nv, int nx, int ny, int nz, float vx, float vy, float vz,
                                float T_in)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (FACE == 1 ? nx : ny)) return;
    const long long base = FACE == 1 ? ((long long)q * ny + (ny - 1)) * nz : ((long long)(nx - 1) * ny + q) * nz;
    int start = -1, end = 0;
    for (int k = 0; k < nz; k++)
        if ((code[base + k] & CODE_TYPE) == NODE_IN) {
            if (start < 0) start = k;
            end = k;
        }
    if (start < 0) return;
    const int half = (start + end) / 2;
    for (int k = 0; k < nz; k++)
        if ((code[base + k] & CODE_TYPE) == NODE_IN) {
            if (k < half) set_node<R>(code, nv, base + k, NODE_VALVE, vx, vy, vz, T_in);
            else set_node<R>(code, nv, base + k, NODE_VALVE, fsub(0.0f, vx), fsub(0.0f, vy), fsub(0.0f, vz),
                             fsub(2.0f, T_in));
        }
}

// ---------------------------------------------------------------------------
// Shape2D extrusion (Grid3D::Prepare2D, Grid3D.cpp:608-665), one thread per
// column: the column is cleared (memset: NODE_IN, no-slip, zeros) and written in
// the reference's order.  The host checks 2 <= active_nz <= nz; a bottom that
// would reach outside the column is counted in the status word and clipped.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void set_full(uint8_t *code, Layer<R> nv, long long c, uint8_t type, int bcv, int bct,
                                         float vx, float vy, float vz, float T)
{
    code[c] = (uint8_t)(type | (bcv == BC_FREE ? CODE_VEL_FREE : 0) | (bct == BC_FREE ? CODE_TEMP_FREE : 0));
    nv.f[0][c] = (R)vx;
    nv.f[1][c] = (R)vy;
    nv.f[2][c] = (R)vz;
    nv.f[3][c] = (R)T;
}

template <typename R>
__global__ void extrude2d_kernel(uint8_t *code, Layer<R> nv, Layer<R> cur, int nx, int ny, int nz,
                                 const uint8_t *__restrict__ t2, const float *__restrict__ v2,
                                 const float *__restrict__ T2, int active_nz, double depth_var, float baseT,
                                 int *status)
{
    const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (col >= (long long)nx * ny) return;
    const int i = (int)(col / ny), j = (int)(col % ny);
    const long long base = col * nz;
    for (int k = 0; k < nz; k++) set_full<R>(code, nv, base + k, NODE_IN, BC_NOSLIP, BC_NOSLIP, 0.f, 0.f, 0.f, 0.f);
    const uint8_t t = t2[col];
    if (t == NODE_OUT) {
        for (int k = 0; k < nz; k++) code[base + k] = NODE_OUT;
    } else {
        // top: constant height
        for (int k = active_nz - 1; k < nz; k++) code[base + k] = (uint8_t)(NODE_OUT | (code[base + k] & ~CODE_TYPE));
        set_full<R>(code, nv, base + active_nz - 2, NODE_BOUND, BC_NOSLIP, BC_FREE, 0.f, 0.f, 0.f, baseT);
        // bottom with a perturbation (double arithmetic, Grid3D.cpp:633-637)
        const int height = max(active_nz - 2 - 2, 0);
        const double x = __dadd_rn(-1.0, __ddiv_rn(__dmul_rn(2.0, (double)i), (double)nx));
        const double y = __dadd_rn(-1.0, __ddiv_rn(__dmul_rn(2.0, (double)j), (double)ny));
        const double z = __dsub_rn(1.0, __dmul_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), 0.5));
        int bottom = 1 + to_int(__dmul_rn(__dmul_rn(depth_var, z), (double)height));
        if (bottom > nz - 1 || bottom < -1) {   // the reference would write into a neighbouring column
            atomicAdd(&status[ST_OUTSIDE], 1);
            bottom = bottom < -1 ? -1 : nz - 1;
        }
        code[base] = (uint8_t)(NODE_OUT | (code[base] & ~CODE_TYPE));
        for (int k = 1; k <= bottom; k++)
            set_full<R>(code, nv, base + k, NODE_BOUND, BC_NOSLIP, BC_FREE, 0.f, 0.f, 0.f, baseT);
        const float vx = v2[2 * col], vy = v2[2 * col + 1], T = T2[col];
        for (int k = bottom + 1; k < active_nz - 2; k++) {
            const long long c = base + k;
            if (t == NODE_BOUND) {
                set_full<R>(code, nv, c, NODE_BOUND, BC_NOSLIP, BC_FREE, vx, vy, 0.f, T);
            } else if (t == NODE_VALVE) {
                if (vx == 0.0f && vy == 0.0f) set_full<R>(code, nv, c, NODE_VALVE, BC_FREE, BC_FREE, vx, vy, 0.f, T);
                else set_full<R>(code, nv, c, NODE_VALVE, BC_NOSLIP, BC_NOSLIP, vx, vy, 0.f, T);
            } else {   // NODE_IN: the type and T (Grid3D.cpp:657-660)
                code[c] = (uint8_t)(NODE_IN | (code[c] & ~CODE_TYPE));
                nv.f[3][c] = (R)baseT;
            }
        }
    }
    for (int k = 0; k < nz; k++)
#pragma unroll
        for (int v = 0; v < 4; v++) cur.f[v][base + k] = nv.f[v][base + k];
}

template <typename R>
__global__ void copy_state_kernel(Layer<R> nv, Layer<R> cur, long long n)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int v = 0; v < 4; v++) cur.f[v][c] = nv.f[v][c];
}

// ---------------------------------------------------------------------------
// Shape2D (FluidSolver2D::Grid2D::Build, Grid2D.cpp:231-266): a 2D node grid from
// polylines.  Every cell NODE_IN; the segments of the moving shapes rasterised as
// NODE_VALVE, then those of the fixed shapes as NODE_BOUND (RasterLine,
// Grid2D.cpp:109-141, the no-slip form: the cell takes the velocity interpolated
// along the segment and T = startT); the outside flood-filled from cell (0,0);
// NODE_IN / NODE_OUT cells get v = 0, T = startT.  Every cell's BC is no-slip.
//
// In the reference a later write to a cell replaces an earlier one, in segment
// order and step order.  Here every segment walks its steps in one thread twice:
// the first walk claims each cell with the largest (segment, step) sequence
// number that reaches it (atomicMax), the second writes the data where its own
// number won, which is the reference's last write.
// ---------------------------------------------------------------------------

// one segment: p1 (2), p2 (2), v1 (2), v2 (2) in grid coordinates
struct Seg2D {
    float p1x, p1y, p2x, p2y, v1x, v1y, v2x, v2y;
};

template <bool WRITE>
__global__ void raster2d_kernel(const float *__restrict__ segs, const uint8_t *__restrict__ color, int nseg, int nx,
                                int ny, unsigned long long *key, uint8_t *type, float *vel, int *status)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nseg) return;
    const Seg2D sg = reinterpret_cast<const Seg2D *>(segs)[q];
    const float ox = fsub(sg.p2x, sg.p1x), oy = fsub(sg.p2y, sg.p1y);
    const int steps = to_int(smax(fabsf(ox), fabsf(oy))) + 1;
    if (steps > MAX_WALK) {
        if (!WRITE) atomicAdd(&status[ST_BOUNDED], 1);
        return;
    }
    const float fs = __int2float_rn(steps);
    const float dpx = fdiv(ox, fs), dpy = fdiv(oy, fs);
    const float dvx = fdiv(fsub(sg.v2x, sg.v1x), fs), dvy = fdiv(fsub(sg.v2y, sg.v1y), fs);
    float px = sg.p1x, py = sg.p1y, vx = sg.v1x, vy = sg.v1y;
    for (int i = 0; i <= steps; i++) {
        const int x = to_int(px), y = to_int(py);
        if (x < 0 || x >= nx || y < 0 || y >= ny) {
            if (!WRITE) atomicAdd(&status[ST_OUTSIDE], 1);
        } else {
            const long long c = (long long)x * ny + y;
            const unsigned long long seq = ((unsigned long long)(q + 1) << 32) | (unsigned)i;
            if (!WRITE) atomicMax(&key[c], seq);
            else if (key[c] == seq) {
                type[c] = color[q];
                vel[2 * c] = vx;
                vel[2 * c + 1] = vy;
            }
        }
        px = fadd(px, dpx);
        py = fadd(py, dpy);
        vx = fadd(vx, dvx);
        vy = fadd(vy, dvy);
    }
}

// The end of Grid2D::Build (Grid2D.cpp:256-265): NODE_IN / NODE_OUT cells get v = 0;
// every cell T = startT and a no-slip BC.
__global__ void shape2d_finish_kernel(const uint8_t *__restrict__ type, float *vel, float *T, uint8_t *bc, long long n,
                                      float startT)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const uint8_t t = type[c];
        if (t == NODE_IN || t == NODE_OUT) {
            vel[2 * c] = 0.0f;
            vel[2 * c + 1] = 0.0f;
        }
        T[c] = startT;
        bc[c] = BC_NOSLIP;
    }
}

// The solver contract and the NODE_IN count of a node grid, on the device: the
// same tests as the host's check of an uploaded mask, in the same order, so the
// first failing cell in linear order (and the rule it fails) is the one the host
// check reports.  first_bad: min over failing cells of (index << 2 | rule).
__global__ void mask_census_kernel(const uint8_t *__restrict__ code, int nx, int ny, int nz,
                                   unsigned long long *first_bad, unsigned long long *num_in)
{
    const long long n = (long long)nx * ny * nz;
    const long long sx = (long long)ny * nz, sy = nz;
    const bool small = n < (1ll << 32);   // 32-bit index arithmetic suffices
    unsigned long long cnt = 0, bad = ~0ull;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (small) {
            const unsigned cu = (unsigned)c, row = cu / (unsigned)nz;
            k = (int)(cu - row * (unsigned)nz);
            i = (int)(row / (unsigned)ny);
            j = (int)(row - (unsigned)i * (unsigned)ny);
        } else {
            i = (int)(c / sx); j = (int)((c / sy) % ny); k = (int)(c % nz);
        }
        const bool frame = i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1;
        const uint8_t t = code[c] & CODE_TYPE;
        auto ty = [&](long long q) { return code[q] & CODE_TYPE; };
        int rule = 0;
        if (t == NODE_IN) {
            cnt++;
            if (frame) rule = 1;
            else if (ty(c - sx) == NODE_OUT || ty(c + sx) == NODE_OUT || ty(c - sy) == NODE_OUT ||
                     ty(c + sy) == NODE_OUT || ty(c - 1) == NODE_OUT || ty(c + 1) == NODE_OUT)
                rule = 2;
        } else if (!frame && (code[c] & (CODE_VEL_FREE | CODE_TEMP_FREE))) {
            if ((ty(c - sx) == NODE_IN && ty(c + sx) == NODE_IN) || (ty(c - sy) == NODE_IN && ty(c + sy) == NODE_IN) ||
                (ty(c - 1) == NODE_IN && ty(c + 1) == NODE_IN))
                rule = 3;
        }
        if (rule) {
            const unsigned long long key = ((unsigned long long)c << 2) | (unsigned long long)rule;
            if (key < bad) bad = key;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        const unsigned long long b = __shfl_down_sync(0xffffffffu, bad, o);
        if (b < bad) bad = b;
    }
    if ((threadIdx.x & 31) == 0) {
        if (cnt) atomicAdd(num_in, cnt);
        if (bad != ~0ull) atomicMin(first_bad, bad);
    }
}

int grid_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}

} // namespace

// Flood fill from cell (0,0,0), which becomes NODE_OUT whatever it was, through
// NODE_IN cells (6 neighbours; 4 when nz = 1): passes of X, Y and Z line scans
// until one changes nothing, at most max_passes.
static cudaError_t flood_fill(uint8_t *types, int nx, int ny, int nz, int *changed, int max_passes, int *passes_out,
                              cudaStream_t s)
{
    fill_types_kernel<<<1, 1, 0, s>>>(types, 1, NODE_OUT);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int passes = 0;
    constexpr int CHUNK = 1 << 20;   // whole lines: one forward and one backward walk per line
    auto threads = [&](long long lines, int len) { return lines * ((len + CHUNK - 1) / CHUNK) * 2; };
    const long long tz = threads((long long)nx * ny, nz), ty = threads((long long)nx * nz, ny),
                    tx = threads((long long)ny * nz, nx);
    while (passes < max_passes) {
        if ((e = cudaMemsetAsync(changed, 0, sizeof(int), s)) != cudaSuccess) return e;
        if (nz > 1)
            flood_scan_kernel<2><<<(unsigned)((tz + 127) / 128), 128, 0, s>>>(types, nx, ny, nz, CHUNK, changed);
        flood_scan_kernel<1><<<(unsigned)((ty + 127) / 128), 128, 0, s>>>(types, nx, ny, nz, CHUNK, changed);
        flood_scan_kernel<0><<<(unsigned)((tx + 127) / 128), 128, 0, s>>>(types, nx, ny, nz, CHUNK, changed);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        int h = 0;
        if ((e = cudaMemcpyAsync(&h, changed, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        passes++;
        if (!h) break;
    }
    *passes_out = passes;
    return cudaSuccess;
}

cudaError_t launch_mask_shape2d(const float *segs, const uint8_t *color, int nseg, int nx, int ny, float startT,
                                unsigned long long *key, uint8_t *type, float *vel, float *T, uint8_t *bc,
                                int *status, int *changed, int max_passes, int *passes_out, cudaStream_t s)
{
    const long long n = (long long)nx * ny;
    fill_types_kernel<<<grid_for(n, 256), 256, 0, s>>>(type, n, NODE_IN);
    cudaError_t e = cudaMemsetAsync(key, 0, sizeof(unsigned long long) * n, s);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(vel, 0, sizeof(float) * 2 * n, s)) != cudaSuccess) return e;
    if (nseg > 0) {
        const unsigned blocks = (unsigned)((nseg + 127) / 128);
        raster2d_kernel<false><<<blocks, 128, 0, s>>>(segs, color, nseg, nx, ny, key, type, vel, status);
        raster2d_kernel<true><<<blocks, 128, 0, s>>>(segs, color, nseg, nx, ny, key, type, vel, status);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // FloodFill(NODE_OUT) from (0,0) (Grid2D.cpp:156-195), 4 neighbours
    if ((e = flood_fill(type, nx, ny, 1, changed, max_passes, passes_out, s)) != cudaSuccess) return e;
    shape2d_finish_kernel<<<grid_for(n, 256), 256, 0, s>>>(type, vel, T, bc, n, startT);
    return cudaGetLastError();
}

cudaError_t launch_mask_shape3d(uint8_t *types, int nx, int ny, int nz, const float *verts, int nverts,
                                const int *tris, int ntris, int *status, int *changed, int max_passes,
                                int *passes_out, cudaStream_t s)
{
    const long long n = (long long)nx * ny * nz;
    fill_types_kernel<<<grid_for(n, 256), 256, 0, s>>>(types, n, NODE_IN);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    Grid g{types, nx, ny, nz, status};
    if (ntris > 0) {
        const long long threads = (long long)ntris * 32;
        raster_triangles_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(g, verts, tris, ntris, nverts);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // FloodFill from (0,0,0) (Grid3D.cpp:875-878)
    return flood_fill(types, nx, ny, nz, changed, max_passes, passes_out, s);
}

template <typename R>
cudaError_t launch_mask_shape3d_install(const uint8_t *types, uint8_t *code, Layer<R> nv, Layer<R> cur, long long n,
                                        R baseT, cudaStream_t s)
{
    shape_install_kernel<R><<<grid_for(n, 256), 256, 0, s>>>(types, code, nv, cur, n, baseT);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_mask_sea(uint8_t *code, uint8_t *snap, Layer<R> nv, Layer<R> cur, int nx, int ny, int nz,
                            const float *depth, int dnx, int dny, float zmin, float baseT, const float in_vel[3],
                            float in_T, int *status, cudaStream_t s)
{
    const long long cols = (long long)nx * ny, n = cols * nz;
    sea_columns_kernel<R><<<grid_for(n, 256), 256, 0, s>>>(code, nv, n, baseT);
    sea_water_kernel<<<(unsigned)((cols + 127) / 128), 128, 0, s>>>(code, nx, ny, nz, depth, dnx, dny, zmin, status);
    sea_wall_in_kernel<R><<<grid_for(n, 256), 256, 0, s>>>(code, nv, nx, ny, nz, baseT);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(snap, code, n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    sea_wall_out_kernel<R><<<grid_for(n, 256), 256, 0, s>>>(snap, code, nv, nx, ny, nz, baseT);
    sea_face_kernel<R, 1><<<(nx + 127) / 128, 128, 0, s>>>(code, nv, nx, ny, nz, in_vel[0], in_vel[1], in_vel[2], in_T);
    sea_face_kernel<R, 0><<<(ny + 127) / 128, 128, 0, s>>>(code, nv, nx, ny, nz, in_vel[0], in_vel[1], in_vel[2], in_T);
    copy_state_kernel<R><<<grid_for(n, 256), 256, 0, s>>>(nv, cur, n);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_mask_extrude2d(uint8_t *code, Layer<R> nv, Layer<R> cur, int nx, int ny, int nz,
                                  const uint8_t *t2, const float *v2, const float *T2, int active_nz, double depth_var,
                                  float baseT, int *status, cudaStream_t s)
{
    const long long cols = (long long)nx * ny;
    extrude2d_kernel<R><<<(unsigned)((cols + 127) / 128), 128, 0, s>>>(code, nv, cur, nx, ny, nz, t2, v2, T2, active_nz,
                                                                       depth_var, baseT, status);
    return cudaGetLastError();
}

cudaError_t launch_mask_census(const uint8_t *code, int nx, int ny, int nz, unsigned long long *out2,
                               cudaStream_t s)
{
    const unsigned long long init[2] = {~0ull, 0ull};
    cudaError_t e = cudaMemcpyAsync(out2, init, sizeof init, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    const long long n = (long long)nx * ny * nz;
    mask_census_kernel<<<grid_for(n, 256), 256, 0, s>>>(code, nx, ny, nz, out2, out2 + 1);
    return cudaGetLastError();
}

#define MASK_INST(R)                                                                                              \
    template cudaError_t launch_mask_shape3d_install<R>(const uint8_t *, uint8_t *, Layer<R>, Layer<R>, long long, R, \
                                                        cudaStream_t);                                            \
    template cudaError_t launch_mask_sea<R>(uint8_t *, uint8_t *, Layer<R>, Layer<R>, int, int, int, const float *, \
                                            int, int, float, float, const float *, float, int *, cudaStream_t);     \
    template cudaError_t launch_mask_extrude2d<R>(uint8_t *, Layer<R>, Layer<R>, int, int, int, const uint8_t *,   \
                                                  const float *, const float *, int, double, float, int *,        \
                                                  cudaStream_t);
MASK_INST(float)
MASK_INST(double)
#undef MASK_INST

} // namespace adi
