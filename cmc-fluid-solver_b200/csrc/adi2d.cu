// 2D ADI time step (the reference's AdiSolver2D) on the GPU.
//
// Semantics follow the reference's CPU 2D solver operation by operation (this
// file is compiled with --fmad=false and spells every expression in the
// reference's operand order, so float results equal the reference's and double
// results the FP64 restatement's, bit for bit):
//   * segments (AdiSolver2D.cpp:228-277): one per row (X sweep) and one per column
//     (Y sweep), from the node before the first IN node to the node after the last
//     one; obstacle nodes inside are ordinary matrix rows;
//   * rows (AdiSolver2D.cpp:74-178): BC rows by the node's BC type for every
//     variable (FREE: x0 - x1 = 0, x[n-2] - x[n-1] = 0), BuildMatrix rows with
//     1/dt, advection by temp_local U (X) or V (Y), pressure term v_T T', and the
//     2D dissipation function; Thomas without pivoting (Algorithms.h:21-39);
//   * SolveDirection (:203-226): temp_local = temp, then num_local times: every
//     segment into next_local, temp_local = next_local (first) or merged with it
//     (later) on IN nodes; finally temp and next take temp_local / next_local on
//     IN nodes;
//   * TimeStep (:279-323): next, half, temp = cur; global iterations X then Y
//     sweep while it < num_global or the divergence error exceeds 0.1, temp taking
//     next (first) or merging with it; OUT nodes of next cleared; cur = next;
//   * layer copies and merges stop one row and one column short, as the
//     reference's loops do (TimeLayer2D.h:98-176); the cells they never reach keep
//     what they held (zero from allocation);
//   * where the reference calls exit(1) (error above 1.0, more than 100 global
//     iterations) the step returns ADI_ERR_DIVERGENCE / ADI_ERR_NOT_CONVERGED.
// The divergence error (TimeLayer2D.h:86-100, written dy*(dU) + dU'/2) is summed in
// double by a fixed-order tree; the reference sums in FTYPE sequentially, so its
// printed value can differ in the last digits; it only decides the loop exit.
//
// Kernels are one thread per segment (the sweeps; at most a few hundred lines)
// and grid-stride elementwise passes; a step is one CUDA graph launch plus one
// read of the per-iteration errors.
#include "adi_b200.h"
#include "adi_internal.cuh"

#include <cmath>
#include <cstring>
#include <string>
#include <algorithm>
#include <vector>

struct adi2d_handle;

namespace adi {
namespace d2 {

enum : uint8_t { T_IN = 1, T_OUT = 2, T_BOUND = 4, T_VALVE = 8 };   // node-type bit masks

template <typename R>
struct L2 {
    R *f[3];   // U, V, T
};

struct Seg {
    int posx, posy, size, dir;   // dir 0: along x (rows), 1: along y (columns)
};

template <typename R>
struct Consts {
    R dt, dx, dy, v_T, v_vis, t_vis, t_phi, startT;
};

__device__ __forceinline__ long long gid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gstr() { return (long long)gridDim.x * blockDim.x; }

__device__ __forceinline__ uint8_t tbit(uint8_t t) { return (uint8_t)(1u << t); }

// dst = src on the nodes whose type is in `mask`, i < nx-1, j < ny-1.
template <typename R>
__global__ void copy_types_kernel(int nx, int ny, const uint8_t *__restrict__ type, L2<R> src, L2<R> dst, uint8_t mask)
{
    const long long n = (long long)nx * ny;
    for (long long id = gid(); id < n; id += gstr()) {
        const int i = (int)(id / ny), j = (int)(id - (long long)i * ny);
        if (i >= nx - 1 || j >= ny - 1 || !(tbit(type[id]) & mask)) continue;
#pragma unroll
        for (int v = 0; v < 3; v++) dst.f[v][id] = src.f[v][id];
    }
}

// dst = (dst + src) / 2 on IN nodes, i < nx-1, j < ny-1.
template <typename R>
__global__ void merge_in_kernel(int nx, int ny, const uint8_t *__restrict__ type, L2<R> src, L2<R> dst)
{
    const long long n = (long long)nx * ny;
    for (long long id = gid(); id < n; id += gstr()) {
        const int i = (int)(id / ny), j = (int)(id - (long long)i * ny);
        if (i >= nx - 1 || j >= ny - 1 || type[id] != NODE_IN) continue;
#pragma unroll
        for (int v = 0; v < 3; v++) dst.f[v][id] = (dst.f[v][id] + src.f[v][id]) / R(2);
    }
}

// cur[BOUND|VALVE] = node data (Solver2D.cpp:40-51); the copy into next follows
// as copy_types.
template <typename R>
__global__ void update_bnd_kernel(long long n, const uint8_t *__restrict__ type, L2<R> data, L2<R> cur)
{
    for (long long id = gid(); id < n; id += gstr()) {
        if (type[id] != NODE_BOUND && type[id] != NODE_VALVE) continue;
#pragma unroll
        for (int v = 0; v < 3; v++) cur.f[v][id] = data.f[v][id];
    }
}

// OUT nodes of next: U = V = 0, T = startT (Solver2D.cpp:68-80).
template <typename R>
__global__ void clear_out_kernel(long long n, const uint8_t *__restrict__ type, L2<R> next, R startT)
{
    for (long long id = gid(); id < n; id += gstr()) {
        if (type[id] != NODE_OUT) continue;
        next.f[0][id] = R(0);
        next.f[1][id] = R(0);
        next.f[2][id] = startT;
    }
}

// Divergence error terms of the 2x2 all-IN blocks, one fixed-order block tree per
// CTA into partial[blockIdx.x], then the last kernel folds the partials.
// Tolerance-mode residual: max |x - t| and max |x| over NODE_IN nodes and the three
// fields, folded per warp with shuffles and across warps with atomicMax on the bit
// patterns (non-negative values order like their patterns; a NaN wins).
template <typename R>
__device__ __forceinline__ R max_nan2(R a, R b)
{
    return (b > a || b != b) ? b : a;
}

template <typename R>
__global__ void residual2_kernel(long long n, const uint8_t *__restrict__ type, L2<R> x, L2<R> t,
                                 unsigned long long *out)
{
    R dm = R(0), xm = R(0);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (type[i] != NODE_IN) continue;
#pragma unroll
        for (int v = 0; v < 3; v++) {
            const R a = x.f[v][i];
            dm = max_nan2(dm, (R)fabs(a - t.f[v][i]));
            xm = max_nan2(xm, (R)fabs(a));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dm = max_nan2(dm, __shfl_xor_sync(0xffffffffu, dm, o));
        xm = max_nan2(xm, __shfl_xor_sync(0xffffffffu, xm, o));
    }
    if ((threadIdx.x & 31) == 0) {
        unsigned long long bd, bx;
        if (sizeof(R) == 8) {
            bd = (unsigned long long)__double_as_longlong((double)dm);
            bx = (unsigned long long)__double_as_longlong((double)xm);
        } else {
            bd = (unsigned long long)__float_as_uint((float)dm);
            bx = (unsigned long long)__float_as_uint((float)xm);
        }
        atomicMax(out, bd);
        atomicMax(out + 1, bx);
    }
}

template <typename R>
__global__ void div2_partial_kernel(int nx, int ny, const uint8_t *__restrict__ type, L2<R> l, R dx, R dy,
                                    double *psum, unsigned long long *pcnt)
{
    double acc = 0.0;
    unsigned long long cnt = 0;
    const long long n = (long long)nx * ny;
    const R *U = l.f[0], *V = l.f[1];
    for (long long id = gid(); id < n; id += gstr()) {
        const int i = (int)(id / ny), j = (int)(id - (long long)i * ny);
        if (i >= nx - 1 || j >= ny - 1) continue;
        if (type[id] != NODE_IN || type[id + ny] != NODE_IN || type[id + 1] != NODE_IN || type[id + ny + 1] != NODE_IN)
            continue;
        const R tx = dy * (U[id + ny] - U[id]) + (U[id + ny + 1] - U[id + 1]) / R(2);
        const R ty = dx * (V[id + 1] - V[id]) + (V[id + ny + 1] - V[id + ny]) / R(2);
        acc += (double)fabs(tx + ty);
        cnt++;
    }
    __shared__ double ss[256];
    __shared__ unsigned long long sc[256];
    ss[threadIdx.x] = acc;
    sc[threadIdx.x] = cnt;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            ss[threadIdx.x] += ss[threadIdx.x + w];
            sc[threadIdx.x] += sc[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        psum[blockIdx.x] = ss[0];
        pcnt[blockIdx.x] = sc[0];
    }
}

__global__ void div2_final_kernel(const double *psum, const unsigned long long *pcnt, int nb, double *out)
{
    double s = 0.0;
    unsigned long long c = 0;
    for (int b = threadIdx.x; b < nb; b += 32) {
        s += psum[b];
        c += pcnt[b];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (threadIdx.x == 0) *out = c ? s / (double)c : NAN;
}

// One thread per segment: rows, Thomas (forward into scratch, back substitution)
// for U, V (shared a, b, c) and T, written into next_local on the segment nodes.
template <typename R>
__global__ void sweep2_kernel(int nx, int ny, const Seg *__restrict__ segs, int nseg, const uint8_t *__restrict__ bct,
                              L2<R> data, L2<R> cur, L2<R> tl, L2<R> nl, R *__restrict__ scratch, Consts<R> k)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const Seg g = segs[s];
    const int n = g.size;
    const long long st = g.dir == 0 ? ny : 1;   // stride along the segment
    const long long id0 = (long long)g.posx * ny + g.posy;
    const long long idn = id0 + (long long)(n - 1) * st;
    // scratch [q][p][segment]: c'_uv, c'_t, d'_u, d'_v, d'_t; a list's segments all
    // run along one axis, so positions p < (dir == 0 ? nx : ny) and the five
    // quantities take 5 * nx * ny values at most
    R *sc = scratch + s;
    const long long qs = (long long)(g.dir == 0 ? nx : ny) * nseg;
    const R *TU = tl.f[0], *TV = tl.f[1], *TT = tl.f[2];
    const R two = R(2);
    const R vis_xu = k.v_vis / (k.dx * k.dx), vis_xt = k.t_vis / (k.dx * k.dx);
    const R vis_yu = k.v_vis / (k.dy * k.dy), vis_yt = k.t_vis / (k.dy * k.dy);
    R cpu = R(0), cpt = R(0), du = R(0), dv = R(0), dT = R(0);
    for (int p = 0; p < n; p++) {
        const long long id = id0 + (long long)p * st;
        R au, bu, cu, at, bt, ct, d0, d1, d2;
        if (p == 0) {   // ApplyBC0
            const bool fr = bct[id] == BC_FREE;
            au = at = R(0);
            bu = bt = R(1);
            cu = ct = fr ? R(-1) : R(0);
            d0 = fr ? R(0) : data.f[0][id];
            d1 = fr ? R(0) : data.f[1][id];
            d2 = fr ? R(0) : data.f[2][id];
        } else if (p == n - 1) {   // ApplyBC1
            const bool fr = bct[id] == BC_FREE;
            au = at = fr ? R(1) : R(0);
            bu = bt = fr ? R(-1) : R(1);
            cu = ct = R(0);   // c[n-1] = 0 (Algorithms.h:23)
            d0 = fr ? R(0) : data.f[0][id];
            d1 = fr ? R(0) : data.f[1][id];
            d2 = fr ? R(0) : data.f[2][id];
        } else if (g.dir == 0) {   // BuildMatrix, X
            const R w = TU[id];
            const R vu = vis_xu, vt = vis_xt;
            au = -w / (two * k.dx) - vu;
            bu = R(1) / k.dt + two * vu;
            cu = w / (two * k.dx) - vu;
            at = -w / (two * k.dx) - vt;
            bt = R(1) / k.dt + two * vt;
            ct = w / (two * k.dx) - vt;
            const R Tx = (TT[id + ny] - TT[id - ny]) / (two * k.dx);
            d0 = cur.f[0][id] / k.dt - k.v_T * Tx;
            d1 = cur.f[1][id] / k.dt;
            const R ux = (TU[id + ny] - TU[id - ny]) / (two * k.dx);
            const R vx = (TV[id + ny] - TV[id - ny]) / (two * k.dx);
            const R uy = (TU[id + 1] - TU[id - 1]) / (two * k.dy);
            d2 = cur.f[2][id] / k.dt + k.t_phi * (two * ux * ux + vx * vx + uy * vx);
        } else {   // BuildMatrix, Y
            const R w = TV[id];
            const R vu = vis_yu, vt = vis_yt;
            au = -w / (two * k.dy) - vu;
            bu = R(1) / k.dt + two * vu;
            cu = w / (two * k.dy) - vu;
            at = -w / (two * k.dy) - vt;
            bt = R(1) / k.dt + two * vt;
            ct = w / (two * k.dy) - vt;
            const R Ty = (TT[id + 1] - TT[id - 1]) / (two * k.dy);
            d0 = cur.f[0][id] / k.dt;
            d1 = cur.f[1][id] / k.dt - k.v_T * Ty;
            const R vx = (TV[id + ny] - TV[id - ny]) / (two * k.dx);
            const R uy = (TU[id + 1] - TU[id - 1]) / (two * k.dy);
            const R vy = (TV[id + 1] - TV[id - 1]) / (two * k.dy);
            d2 = cur.f[2][id] / k.dt + k.t_phi * (uy * uy + two * vy * vy + vx * uy);
        }
        // Thomas forward step (Algorithms.h:25-32), the reference's operand order
        R ncu, nct, n0, n1, n2;
        if (p == 0) {
            ncu = cu / bu;
            nct = ct / bt;
            n0 = d0 / bu;
            n1 = d1 / bu;
            n2 = d2 / bt;
        } else {
            ncu = cu / (bu - au * cpu);
            nct = ct / (bt - at * cpt);
            n0 = (d0 - du * au) / (bu - au * cpu);
            n1 = (d1 - dv * au) / (bu - au * cpu);
            n2 = (d2 - dT * at) / (bt - at * cpt);
        }
        cpu = ncu; cpt = nct; du = n0; dv = n1; dT = n2;
        R *q = sc + (long long)p * nseg;
        q[0] = ncu;
        q[qs] = nct;
        q[2 * qs] = n0;
        q[3 * qs] = n1;
        q[4 * qs] = n2;
    }
    R x0 = du, x1 = dv, x2 = dT;
    nl.f[0][idn] = x0;
    nl.f[1][idn] = x1;
    nl.f[2][idn] = x2;
    for (int p = n - 2; p >= 0; p--) {
        const long long id = id0 + (long long)p * st;
        const R *q = sc + (long long)p * nseg;
        x0 = q[2 * qs] - q[0] * x0;
        x1 = q[3 * qs] - q[0] * x1;
        x2 = q[4 * qs] - q[qs] * x2;
        nl.f[0][id] = x0;
        nl.f[1][id] = x1;
        nl.f[2][id] = x2;
    }
}

// Row coefficients of one segment row p (BC rows at the ends, BuildMatrix rows
// inside), the reference's operand order.  Shared by both 2D sweep kernels.
template <typename R>
__device__ __forceinline__ void row2(const Seg &g, int p, int n, long long id, int ny, const uint8_t *__restrict__ bct,
                                     const L2<R> &data, const L2<R> &cur, const L2<R> &tl, const Consts<R> &k, R &au,
                                     R &bu, R &cu, R &at, R &bt, R &ct, R &d0, R &d1, R &d2)
{
    const R *TU = tl.f[0], *TV = tl.f[1], *TT = tl.f[2];
    const R two = R(2);
    if (p == 0 || p == n - 1) {   // ApplyBC0 / ApplyBC1
        const bool fr = bct[id] == BC_FREE;
        if (p == 0) {
            au = at = R(0);
            bu = bt = R(1);
            cu = ct = fr ? R(-1) : R(0);
        } else {
            au = at = fr ? R(1) : R(0);
            bu = bt = fr ? R(-1) : R(1);
            cu = ct = R(0);   // c[n-1] = 0 (Algorithms.h:23)
        }
        d0 = fr ? R(0) : data.f[0][id];
        d1 = fr ? R(0) : data.f[1][id];
        d2 = fr ? R(0) : data.f[2][id];
    } else if (g.dir == 0) {
        const R vu = k.v_vis / (k.dx * k.dx), vt = k.t_vis / (k.dx * k.dx);
        const R w = TU[id];
        au = -w / (two * k.dx) - vu;
        bu = R(1) / k.dt + two * vu;
        cu = w / (two * k.dx) - vu;
        at = -w / (two * k.dx) - vt;
        bt = R(1) / k.dt + two * vt;
        ct = w / (two * k.dx) - vt;
        const R Tx = (TT[id + ny] - TT[id - ny]) / (two * k.dx);
        d0 = cur.f[0][id] / k.dt - k.v_T * Tx;
        d1 = cur.f[1][id] / k.dt;
        const R ux = (TU[id + ny] - TU[id - ny]) / (two * k.dx);
        const R vx = (TV[id + ny] - TV[id - ny]) / (two * k.dx);
        const R uy = (TU[id + 1] - TU[id - 1]) / (two * k.dy);
        d2 = cur.f[2][id] / k.dt + k.t_phi * (two * ux * ux + vx * vx + uy * vx);
    } else {
        const R vu = k.v_vis / (k.dy * k.dy), vt = k.t_vis / (k.dy * k.dy);
        const R w = TV[id];
        au = -w / (two * k.dy) - vu;
        bu = R(1) / k.dt + two * vu;
        cu = w / (two * k.dy) - vu;
        at = -w / (two * k.dy) - vt;
        bt = R(1) / k.dt + two * vt;
        ct = w / (two * k.dy) - vt;
        const R Ty = (TT[id + 1] - TT[id - 1]) / (two * k.dy);
        d0 = cur.f[0][id] / k.dt;
        d1 = cur.f[1][id] / k.dt - k.v_T * Ty;
        const R vx = (TV[id + ny] - TV[id - ny]) / (two * k.dx);
        const R uy = (TU[id + 1] - TU[id - 1]) / (two * k.dy);
        const R vy = (TV[id + 1] - TV[id - 1]) / (two * k.dy);
        d2 = cur.f[2][id] / k.dt + k.t_phi * (uy * uy + two * vy * vy + vx * uy);
    }
}

// One CTA per segment: all threads build the rows into shared memory, lanes 0-2
// run the Thomas recurrences of U, V and T side by side (the same instructions on
// their own arrays; U and V each recompute the shared c'), all threads write the
// solution back.  Bit-identical to sweep2_kernel; latency per row is a shared-
// memory round trip instead of a global one.
template <typename R>
__global__ void sweep2_smem_kernel(int nx, int ny, const Seg *__restrict__ segs, const uint8_t *__restrict__ bct,
                                   L2<R> data, L2<R> cur, L2<R> tl, L2<R> nl, Consts<R> k)
{
    extern __shared__ __align__(16) unsigned char sm2[];
    const Seg g = segs[blockIdx.x];
    const int n = g.size;
    const long long st = g.dir == 0 ? ny : 1;
    const long long id0 = (long long)g.posx * ny + g.posy;
    // arrays of n: a, b, c for U/V and T (6), d for U, V, T (3), c' for U, V, T (3)
    R *A = reinterpret_cast<R *>(sm2);
    R *a_uv = A, *b_uv = A + n, *c_uv = A + 2 * n, *a_t = A + 3 * n, *b_t = A + 4 * n, *c_t = A + 5 * n;
    R *dd = A + 6 * n;    // [3][n]
    R *cpr = A + 9 * n;   // [3][n]
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        R au, bu, cu, at, bt, ct, d0, d1, d2;
        row2<R>(g, p, n, id0 + (long long)p * st, ny, bct, data, cur, tl, k, au, bu, cu, at, bt, ct, d0, d1, d2);
        a_uv[p] = au; b_uv[p] = bu; c_uv[p] = cu;
        a_t[p] = at; b_t[p] = bt; c_t[p] = ct;
        dd[p] = d0; dd[n + p] = d1; dd[2 * n + p] = d2;
    }
    __syncthreads();
    const int v = threadIdx.x;
    if (v < 3) {
        const R *a = v < 2 ? a_uv : a_t, *b = v < 2 ? b_uv : b_t, *c = v < 2 ? c_uv : c_t;
        R *d = dd + v * n, *cp = cpr + v * n;
        // Thomas (Algorithms.h:21-39) in the reference's operand order
        // Each row's coefficients are read before the previous row's results are
        // stored, so the shared-memory loads stay off the dependent chain (the
        // arithmetic and its order are unchanged).
        R cprev = c[0] / b[0];
        R dprev = d[0] / b[0];
        cp[0] = cprev;
        d[0] = dprev;
        R an = a[1], bn = b[1], cn = c[1], dn = d[1];   // segments have at least three rows
        for (int p = 1; p < n; p++) {
            const R ap = an, bp = bn, cq = cn, dq = dn;
            if (p + 1 < n) {
                an = a[p + 1];
                bn = b[p + 1];
                cn = c[p + 1];
                dn = d[p + 1];
            }
            const R cc = cq / (bp - ap * cprev);
            const R dv = (dq - dprev * ap) / (bp - ap * cprev);
            cp[p] = cc;
            d[p] = dv;
            cprev = cc;
            dprev = dv;
        }
        R x = dprev;   // x[n-1] = d'[n-1]
        R dm = d[n - 2], cm = cp[n - 2];
        for (int p = n - 2; p >= 0; p--) {
            const R dq = dm, cq = cm;
            if (p > 0) {
                dm = d[p - 1];
                cm = cp[p - 1];
            }
            x = dq - cq * x;
            d[p] = x;
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        const long long id = id0 + (long long)p * st;
        nl.f[0][id] = dd[p];
        nl.f[1][id] = dd[n + p];
        nl.f[2][id] = dd[2 * n + p];
    }
    (void)nx;
}

} // namespace d2
} // namespace adi

using namespace adi;
using namespace adi::d2;

struct adi2d_handle {
    int nx = 0, ny = 0, prec = ADI_FP64;
    double dx = 0, dy = 0, startT = 0;
    adi_fluid_params params{};
    cudaStream_t stream = nullptr, cap_stream = nullptr;
    uint8_t *d_type = nullptr, *d_bct = nullptr;
    std::vector<uint8_t> h_type;
    void *d_data[3] = {}, *d_L[7][3] = {};   // cur, next, half, temp, next_local, temp_local, prev
    Seg *d_segx = nullptr, *d_segy = nullptr;
    int nsegx = 0, nsegy = 0;
    void *d_scratch = nullptr;
    double *d_psum = nullptr, *d_err = nullptr;   // d_err: one value per global iteration slot
    unsigned long long *d_pcnt = nullptr;
    double *h_err = nullptr;
    int err_slots = 0;
    bool grid_set = false;
    double last_err = 0;
    int last_iters = 0;
    std::string msg;
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_key[2] = {0, 0};
    unsigned long long *d_res = nullptr;   // tolerance mode: max |x - t|, max |x| bit patterns
    int seg_mode = 0;             // 0: row-spanning (the reference), 1: masked segments
    size_t scratch_bytes = 0;
};

namespace {

constexpr int D2_BLOCKS = 64;
enum { CUR = 0, NXT = 1, HALF = 2, TMP = 3, NLOC = 4, TLOC = 5, PREV = 6 };

adi_status f2(adi2d_handle *h, adi_status s, const std::string &m)
{
    if (h) h->msg = m;
    return s;
}

#define CK2(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return f2(h, ADI_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

size_t es2(const adi2d_handle *h) { return h->prec == ADI_FP64 ? 8 : 4; }

template <typename R>
L2<R> lay(const adi2d_handle *h, int l)
{
    L2<R> x;
    for (int v = 0; v < 3; v++) x.f[v] = (R *)h->d_L[l][v];
    return x;
}

template <typename R>
Consts<R> consts(const adi2d_handle *h, double dt)
{
    Consts<R> k;
    k.dt = (R)dt;
    k.dx = (R)h->dx;
    k.dy = (R)h->dy;
    k.v_T = (R)h->params.v_T;
    k.v_vis = (R)h->params.v_vis;
    k.t_vis = (R)h->params.t_vis;
    k.t_phi = (R)h->params.t_phi;
    k.startT = (R)h->startT;
    return k;
}

int blocks_for(long long n)
{
    long long b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

template <typename R>
adi_status copy_types(adi2d_handle *h, int src, int dst, uint8_t mask)
{
    copy_types_kernel<R><<<blocks_for((long long)h->nx * h->ny), 256, 0, h->stream>>>(h->nx, h->ny, h->d_type,
                                                                                      lay<R>(h, src), lay<R>(h, dst), mask);
    CK2(cudaGetLastError());
    return ADI_OK;
}

template <typename R>
adi_status merge_in(adi2d_handle *h, int src, int dst)
{
    merge_in_kernel<R><<<blocks_for((long long)h->nx * h->ny), 256, 0, h->stream>>>(h->nx, h->ny, h->d_type,
                                                                                    lay<R>(h, src), lay<R>(h, dst));
    CK2(cudaGetLastError());
    return ADI_OK;
}

template <typename R>
adi_status div2(adi2d_handle *h, int l, int slot)
{
    div2_partial_kernel<R><<<D2_BLOCKS, 256, 0, h->stream>>>(h->nx, h->ny, h->d_type, lay<R>(h, l), (R)h->dx,
                                                              (R)h->dy, h->d_psum, h->d_pcnt);
    CK2(cudaGetLastError());
    div2_final_kernel<<<1, 32, 0, h->stream>>>(h->d_psum, h->d_pcnt, D2_BLOCKS, h->d_err + slot);
    CK2(cudaGetLastError());
    return ADI_OK;
}

// SolveDirection (AdiSolver2D.cpp:203-226) for one segment list.
template <typename R>
adi_status solve_dir(adi2d_handle *h, double dt, int num_local, const Seg *segs, int nseg, int cur, int next)
{
    const size_t fb = (size_t)h->nx * h->ny * sizeof(R);
    for (int v = 0; v < 3; v++) CK2(cudaMemsetAsync(h->d_L[TLOC][v], 0, fb, h->stream));
    adi_status s = copy_types<R>(h, TMP, TLOC, T_IN | T_OUT | T_BOUND | T_VALVE);
    if (s != ADI_OK) return s;
    L2<R> data;
    for (int v = 0; v < 3; v++) data.f[v] = (R *)h->d_data[v];
    // longest possible segment of this list: the extent along its axis
    const int len = (nseg > 0 && segs == h->d_segy) ? h->nx : h->ny;
    const size_t smem = (size_t)12 * len * sizeof(R);
    for (int it = 0; it < num_local; it++) {
        if (nseg > 0 && smem <= 200 * 1024) {
            static SmemOptIn opt_in;
            if (smem > 48 * 1024) CK2(ensure_dynamic_smem(opt_in, sweep2_smem_kernel<R>, smem));
            sweep2_smem_kernel<R><<<nseg, 128, smem, h->stream>>>(h->nx, h->ny, segs, h->d_bct, data, lay<R>(h, cur),
                                                                  lay<R>(h, TLOC), lay<R>(h, NLOC), consts<R>(h, dt));
            CK2(cudaGetLastError());
        } else if (nseg > 0) {
            sweep2_kernel<R><<<(nseg + 127) / 128, 128, 0, h->stream>>>(h->nx, h->ny, segs, nseg, h->d_bct, data,
                                                                        lay<R>(h, cur), lay<R>(h, TLOC),
                                                                        lay<R>(h, NLOC), (R *)h->d_scratch,
                                                                        consts<R>(h, dt));
            CK2(cudaGetLastError());
        }
        s = it == 0 ? copy_types<R>(h, NLOC, TLOC, T_IN) : merge_in<R>(h, NLOC, TLOC);
        if (s != ADI_OK) return s;
    }
    if ((s = copy_types<R>(h, TLOC, TMP, T_IN)) != ADI_OK) return s;
    return copy_types<R>(h, NLOC, next, T_IN);
}

// One global iteration (AdiSolver2D.cpp:293-301), its error into err slot `slot`.
template <typename R>
adi_status global_iteration(adi2d_handle *h, double dt, int num_local, int it, int slot)
{
    adi_status s = solve_dir<R>(h, dt, num_local, h->d_segy, h->nsegy, CUR, HALF);
    if (s != ADI_OK) return s;
    if ((s = solve_dir<R>(h, dt, num_local, h->d_segx, h->nsegx, HALF, NXT)) != ADI_OK) return s;
    if ((s = div2<R>(h, NXT, slot)) != ADI_OK) return s;
    return it == 0 ? copy_types<R>(h, NXT, TMP, T_IN) : merge_in<R>(h, NXT, TMP);
}

template <typename R>
adi_status update_boundaries(adi2d_handle *h)
{
    L2<R> data;
    for (int v = 0; v < 3; v++) data.f[v] = (R *)h->d_data[v];
    const long long n = (long long)h->nx * h->ny;
    update_bnd_kernel<R><<<blocks_for(n), 256, 0, h->stream>>>(n, h->d_type, data, lay<R>(h, CUR));
    CK2(cudaGetLastError());
    return copy_types<R>(h, CUR, NXT, T_BOUND | T_VALVE);
}

// The step start and num_global iterations, errors into slots 0..num_global.
template <typename R>
adi_status enqueue_first(adi2d_handle *h, double dt, int num_global, int num_local, bool bnd)
{
    adi_status s;
    if (bnd && (s = update_boundaries<R>(h)) != ADI_OK) return s;
    const uint8_t all = T_IN | T_OUT | T_BOUND | T_VALVE;
    if ((s = copy_types<R>(h, CUR, NXT, all)) != ADI_OK) return s;
    if ((s = copy_types<R>(h, CUR, HALF, all)) != ADI_OK) return s;
    if ((s = copy_types<R>(h, CUR, TMP, all)) != ADI_OK) return s;
    if ((s = div2<R>(h, NXT, 0)) != ADI_OK) return s;
    for (int it = 0; it < num_global; it++)
        if ((s = global_iteration<R>(h, dt, num_local, it, it + 1)) != ADI_OK) return s;
    CK2(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(double) * (num_global + 1), cudaMemcpyDeviceToHost, h->stream));
    return ADI_OK;
}

template <typename R>
adi_status time_step(adi2d_handle *h, double dt, int num_global, int num_local, bool bnd, int *iters)
{
    if (num_global + 2 > h->err_slots) {
        cudaFree(h->d_err);
        cudaFreeHost(h->h_err);
        h->d_err = nullptr;
        h->h_err = nullptr;
        h->err_slots = num_global + 2 > 128 ? num_global + 2 : 128;
        CK2(cudaMalloc((void **)&h->d_err, sizeof(double) * h->err_slots));
        CK2(cudaMallocHost((void **)&h->h_err, sizeof(double) * h->err_slots));
        if (h->graph) cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    // the start and the first num_global iterations: one graph launch
    uint64_t key[2];
    memcpy(&key[0], &dt, 8);
    key[1] = (uint64_t)num_global | ((uint64_t)num_local << 20) | ((uint64_t)bnd << 40) | ((uint64_t)h->stream << 41);
    if (!h->graph || memcmp(key, h->graph_key, sizeof key)) {
        if (h->graph) cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        const cudaStream_t user = h->stream;
        h->stream = h->cap_stream;
        cudaGraph_t g = nullptr;
        CK2(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        adi_status s = enqueue_first<R>(h, dt, num_global, num_local, bnd);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        h->stream = user;
        if (s != ADI_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        CK2(e);
        e = cudaGraphInstantiate(&h->graph, g, 0);
        cudaGraphDestroy(g);
        CK2(e);
        memcpy(h->graph_key, key, sizeof key);
    }
    CK2(cudaGraphLaunch(h->graph, h->stream));
    CK2(cudaStreamSynchronize(h->stream));
    double err = h->h_err[0];
    int it = 0;
    for (; it < num_global; it++) {
        err = h->h_err[it + 1];
        if (it > 100) return f2(h, ADI_ERR_NOT_CONVERGED, "more than 100 global iterations");
        if (err > 0.1 * 10) {
            h->last_err = err;
            return f2(h, ADI_ERR_DIVERGENCE, "2D divergence error above 1.0");
        }
    }
    // further iterations while the error stays above 0.1
    while (err > 0.1) {
        adi_status s = global_iteration<R>(h, dt, num_local, it, 0);
        if (s != ADI_OK) return s;
        CK2(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK2(cudaStreamSynchronize(h->stream));
        err = h->h_err[0];
        if (it > 100) return f2(h, ADI_ERR_NOT_CONVERGED, "more than 100 global iterations");
        if (err > 0.1 * 10) {
            h->last_err = err;
            return f2(h, ADI_ERR_DIVERGENCE, "2D divergence error above 1.0");
        }
        it++;
    }
    const long long n = (long long)h->nx * h->ny;
    clear_out_kernel<R><<<blocks_for(n), 256, 0, h->stream>>>(n, h->d_type, lay<R>(h, NXT), (R)h->startT);
    CK2(cudaGetLastError());
    adi_status s = copy_types<R>(h, NXT, CUR, T_IN | T_OUT | T_BOUND | T_VALVE);
    if (s != ADI_OK) return s;
    h->last_err = err;
    h->last_iters = it;
    if (iters) *iters = it;
    return ADI_OK;
}

// Tolerance mode (no counterpart in the reference, whose 2D loop runs num_global
// iterations and then continues while the divergence error exceeds 0.1,
// AdiSolver2D.cpp:290-314): global iterations run until the change of the iterate
//   r = max |x_k - x_(k-1)| / max |x_k|   over NODE_IN nodes and the three fields
// (x_k the layer after iteration k, x_0 the state the step starts from) is <= tol,
// at most max_global of them.  (The nonlinear layer itself is no measure here:
// SolveDirection hands its temp_local back to temp, AdiSolver2D.cpp:220-225, so
// after the X direction it equals the result.)  The reference's guard stays: an
// error above 1.0 is ADI_ERR_DIVERGENCE.  The host reads error and residual after
// every iteration, so this path runs eagerly.
template <typename R>
adi_status time_step_tol(adi2d_handle *h, double dt, int max_global, int num_local, double tol, bool bnd,
                         int *iters, double *residual)
{
    if (h->err_slots < 4) {
        cudaFree(h->d_err);
        cudaFreeHost(h->h_err);
        h->d_err = nullptr;
        h->h_err = nullptr;
        h->err_slots = 128;
        CK2(cudaMalloc((void **)&h->d_err, sizeof(double) * h->err_slots));
        CK2(cudaMallocHost((void **)&h->h_err, sizeof(double) * h->err_slots));
        if (h->graph) cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    adi_status s;
    if (bnd && (s = update_boundaries<R>(h)) != ADI_OK) return s;
    const uint8_t all = T_IN | T_OUT | T_BOUND | T_VALVE;
    if ((s = copy_types<R>(h, CUR, NXT, all)) != ADI_OK) return s;
    if ((s = copy_types<R>(h, CUR, HALF, all)) != ADI_OK) return s;
    if ((s = copy_types<R>(h, CUR, TMP, all)) != ADI_OK) return s;
    const long long n = (long long)h->nx * h->ny;
    double err = 0, r = NAN;
    int it = 0;
    while (it < max_global) {
        if ((s = copy_types<R>(h, NXT, PREV, T_IN)) != ADI_OK) return s;
        if ((s = solve_dir<R>(h, dt, num_local, h->d_segy, h->nsegy, CUR, HALF)) != ADI_OK) return s;
        if ((s = solve_dir<R>(h, dt, num_local, h->d_segx, h->nsegx, HALF, NXT)) != ADI_OK) return s;
        if ((s = div2<R>(h, NXT, 0)) != ADI_OK) return s;
        CK2(cudaMemsetAsync(h->d_res, 0, 2 * sizeof(unsigned long long), h->stream));
        residual2_kernel<R><<<blocks_for(n), 256, 0, h->stream>>>(n, h->d_type, lay<R>(h, NXT), lay<R>(h, PREV),
                                                                  h->d_res);
        CK2(cudaGetLastError());
        if ((s = it == 0 ? copy_types<R>(h, NXT, TMP, T_IN) : merge_in<R>(h, NXT, TMP)) != ADI_OK) return s;
        CK2(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK2(cudaMemcpyAsync(h->h_err + 1, h->d_res, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            h->stream));
        CK2(cudaStreamSynchronize(h->stream));
        it++;
        err = h->h_err[0];
        unsigned long long bits[2];
        memcpy(bits, h->h_err + 1, sizeof bits);
        double dm, xm;
        if (sizeof(R) == 8) {
            memcpy(&dm, &bits[0], 8);
            memcpy(&xm, &bits[1], 8);
        } else {
            float a, b;
            const uint32_t ua = (uint32_t)bits[0], ub = (uint32_t)bits[1];
            memcpy(&a, &ua, 4);
            memcpy(&b, &ub, 4);
            dm = a;
            xm = b;
        }
        r = xm > 0 ? dm / xm : dm;
        if (err > 0.1 * 10) {
            h->last_err = err;
            return f2(h, ADI_ERR_DIVERGENCE, "2D divergence error above 1.0");
        }
        if (r <= tol) break;
    }
    clear_out_kernel<R><<<blocks_for(n), 256, 0, h->stream>>>(n, h->d_type, lay<R>(h, NXT), (R)h->startT);
    CK2(cudaGetLastError());
    if ((s = copy_types<R>(h, NXT, CUR, all)) != ADI_OK) return s;
    CK2(cudaStreamSynchronize(h->stream));
    h->last_err = err;
    h->last_iters = it;
    if (iters) *iters = it;
    if (residual) *residual = r;
    return ADI_OK;
}

// Masked segments: the 3D solver's segmentation (Grid3D::GenerateListSegments,
// Grid3D.cpp:47-127) on the 2D grid's columns and rows -- every maximal run of IN
// nodes, with the non-IN node on each side as its boundary rows; a run reaching the
// last node of a line has no closing node and is dropped, as there.
void build_segments_masked(const adi2d_handle *h, std::vector<Seg> &cols, std::vector<Seg> &rows)
{
    const int nx = h->nx, ny = h->ny;
    for (int dir = 1; dir >= 0; dir--) {
        const int nlines = dir == 1 ? nx : ny, len = dir == 1 ? ny : nx;
        for (int l = 0; l < nlines; l++) {
            int open = -1;
            for (int p = 0; p + 1 < len; p++) {
                const size_t nxt = dir == 1 ? (size_t)l * ny + (p + 1) : (size_t)(p + 1) * ny + l;
                const bool in_next = h->h_type[nxt] == NODE_IN;
                if (open < 0 && in_next) {
                    open = p;
                } else if (open >= 0 && !in_next) {
                    if (dir == 1) cols.push_back(Seg{l, open, p + 2 - open, 1});
                    else rows.push_back(Seg{open, l, p + 2 - open, 0});
                    open = -1;
                }
            }
        }
    }
}

// AdiSolver2D::CreateSegments (AdiSolver2D.cpp:228-277), or the masked segments.
void build_segments(const adi2d_handle *h, std::vector<Seg> &cols, std::vector<Seg> &rows)
{
    if (h->seg_mode == 1) {
        build_segments_masked(h, cols, rows);
        return;
    }
    const int nx = h->nx, ny = h->ny;
    auto T = [&](int i, int j) { return h->h_type[(size_t)i * ny + j]; };
    for (int i = 0; i < nx; i++) {
        int j = 0;
        while (j < ny && T(i, j) == NODE_OUT) j++;
        while (j + 1 < ny && T(i, j + 1) != NODE_IN) j++;
        if (j + 1 >= ny) continue;
        const int start = j;
        j = ny - 1;
        while (j >= 0 && T(i, j) == NODE_OUT) j--;
        while (j - 1 >= 0 && T(i, j - 1) != NODE_IN) j--;
        cols.push_back(Seg{i, start, j - start + 1, 1});
    }
    for (int j = 0; j < ny; j++) {
        int i = 0;
        while (i < nx && T(i, j) == NODE_OUT) i++;
        while (i + 1 < nx && T(i + 1, j) != NODE_IN) i++;
        if (i + 1 >= nx) continue;
        const int start = i;
        i = nx - 1;
        while (i >= 0 && T(i, j) == NODE_OUT) i--;
        while (i - 1 >= 0 && T(i - 1, j) != NODE_IN) i--;
        rows.push_back(Seg{start, j, i - start + 1, 0});
    }
}

void free2(adi2d_handle *h)
{
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    cudaFree(h->d_type);
    cudaFree(h->d_bct);
    for (int v = 0; v < 3; v++) cudaFree(h->d_data[v]);
    for (int l = 0; l < 7; l++)
        for (int v = 0; v < 3; v++) cudaFree(h->d_L[l][v]);
    cudaFree(h->d_segx);
    cudaFree(h->d_segy);
    cudaFree(h->d_scratch);
    cudaFree(h->d_psum);
    cudaFree(h->d_pcnt);
    cudaFree(h->d_res);
    cudaFree(h->d_err);
    cudaFreeHost(h->h_err);
}

} // namespace

extern "C" {

adi_status adi2d_create(int nx, int ny, double dx, double dy, int precision, const adi_fluid_params *p,
                        adi2d_handle **out)
{
    if (!out || !p || nx < 3 || ny < 3 || !(dx > 0) || !(dy > 0)) return ADI_ERR_BAD_ARG;
    if (precision != ADI_FP32 && precision != ADI_FP64) return ADI_ERR_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ADI_ERR_NO_DEVICE;
    adi2d_handle *h = new (std::nothrow) adi2d_handle();
    if (!h) return ADI_ERR_CAPACITY;
    h->nx = nx;
    h->ny = ny;
    h->dx = dx;
    h->dy = dy;
    h->prec = precision;
    h->params = *p;
    const size_t n = (size_t)nx * ny, fb = n * es2(h);
    cudaError_t e = cudaMalloc((void **)&h->d_type, n);
    if (e == cudaSuccess) e = cudaMalloc((void **)&h->d_bct, n);
    for (int v = 0; v < 3 && e == cudaSuccess; v++) e = cudaMalloc(&h->d_data[v], fb);
    for (int l = 0; l < 7 && e == cudaSuccess; l++)
        for (int v = 0; v < 3 && e == cudaSuccess; v++) {
            e = cudaMalloc(&h->d_L[l][v], fb);
            if (e == cudaSuccess) e = cudaMemset(h->d_L[l][v], 0, fb);
        }
    if (e == cudaSuccess) e = cudaMalloc(&h->d_scratch, 5 * fb);
    if (e == cudaSuccess) h->scratch_bytes = 5 * fb;
    if (e == cudaSuccess) e = cudaMalloc((void **)&h->d_psum, sizeof(double) * D2_BLOCKS);
    if (e == cudaSuccess) e = cudaMalloc((void **)&h->d_res, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc((void **)&h->d_pcnt, sizeof(unsigned long long) * D2_BLOCKS);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        free2(h);
        delete h;
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? ADI_ERR_CAPACITY : ADI_ERR_CUDA;
    }
    *out = h;
    return ADI_OK;
}

adi_status adi2d_destroy(adi2d_handle *h)
{
    if (!h) return ADI_OK;
    cudaStreamSynchronize(h->stream);
    free2(h);
    delete h;
    return ADI_OK;
}

adi_status adi2d_set_stream(adi2d_handle *h, void *stream)
{
    if (!h) return ADI_ERR_BAD_ARG;
    h->stream = (cudaStream_t)stream;
    return ADI_OK;
}

// Builds the segment lists of the handle's mode from its node types and uploads
// them; the per-segment scratch of sweep2_kernel (5 values per row of every
// segment, laid out by the list's longest line) grows to fit.  Drops the graph.
static adi_status upload_segments(adi2d_handle *h)
{
    std::vector<Seg> cols, rows;
    build_segments(h, cols, rows);
    const size_t es = es2(h);
    const size_t need = 5 * es * std::max((size_t)h->ny * cols.size(), (size_t)h->nx * rows.size());
    if (need > h->scratch_bytes) {
        cudaFree(h->d_scratch);
        h->d_scratch = nullptr;
        h->scratch_bytes = 0;
        CK2(cudaMalloc(&h->d_scratch, need));
        h->scratch_bytes = need;
    }
    cudaFree(h->d_segx);
    cudaFree(h->d_segy);
    h->d_segx = h->d_segy = nullptr;
    h->nsegx = (int)cols.size();
    h->nsegy = (int)rows.size();
    if (!cols.empty()) {
        CK2(cudaMalloc((void **)&h->d_segx, sizeof(Seg) * cols.size()));
        CK2(cudaMemcpy(h->d_segx, cols.data(), sizeof(Seg) * cols.size(), cudaMemcpyHostToDevice));
    }
    if (!rows.empty()) {
        CK2(cudaMalloc((void **)&h->d_segy, sizeof(Seg) * rows.size()));
        CK2(cudaMemcpy(h->d_segy, rows.data(), sizeof(Seg) * rows.size(), cudaMemcpyHostToDevice));
    }
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    return ADI_OK;
}

adi_status adi2d_set_grid(adi2d_handle *h, const uint8_t *type, const uint8_t *bc_type, const double *vx,
                          const double *vy, const double *T, double startT)
{
    if (!h || !type || !bc_type || !vx || !vy || !T) return ADI_ERR_BAD_ARG;
    const size_t n = (size_t)h->nx * h->ny, fb = n * es2(h);
    for (size_t q = 0; q < n; q++)
        if (type[q] > NODE_VALVE || bc_type[q] > BC_FREE)
            return f2(h, ADI_ERR_BAD_ARG, "node type or BC type out of range at index " + std::to_string(q));
    h->h_type.assign(type, type + n);
    h->startT = startT;
    CK2(cudaMemcpy(h->d_type, type, n, cudaMemcpyHostToDevice));
    CK2(cudaMemcpy(h->d_bct, bc_type, n, cudaMemcpyHostToDevice));
    const double *src[3] = {vx, vy, T};
    std::vector<float> tmp(n);
    for (int v = 0; v < 3; v++) {
        const void *p = src[v];
        if (h->prec == ADI_FP32) {
            for (size_t q = 0; q < n; q++) tmp[q] = (float)src[v][q];
            p = tmp.data();
        }
        CK2(cudaMemcpy(h->d_data[v], p, fb, cudaMemcpyHostToDevice));
        // AdiSolver2D::Init: cur = node data everywhere (AdiSolver2D.cpp:35-47)
        CK2(cudaMemcpy(h->d_L[CUR][v], p, fb, cudaMemcpyHostToDevice));
    }
    adi_status st = upload_segments(h);
    if (st != ADI_OK) return st;
    h->grid_set = true;
    return ADI_OK;
}

adi_status adi2d_set_segments(adi2d_handle *h, int mode)
{
    if (!h || (mode != 0 && mode != 1)) return ADI_ERR_BAD_ARG;
    if (!h->grid_set) return f2(h, ADI_ERR_STATE, "adi2d_set_grid has not been called");
    CK2(cudaStreamSynchronize(h->stream));
    const int old = h->seg_mode;
    h->seg_mode = mode;
    const adi_status st = upload_segments(h);
    if (st != ADI_OK) h->seg_mode = old;
    return st;
}

adi_status adi2d_update_boundaries(adi2d_handle *h)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (!h->grid_set) return f2(h, ADI_ERR_STATE, "adi2d_set_grid has not been called");
    adi_status s = h->prec == ADI_FP64 ? update_boundaries<double>(h) : update_boundaries<float>(h);
    if (s != ADI_OK) return s;
    CK2(cudaStreamSynchronize(h->stream));
    return ADI_OK;
}

static adi_status step2(adi2d_handle *h, double dt, int num_global, int num_local, bool bnd, int *iters)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (!h->grid_set) return f2(h, ADI_ERR_STATE, "adi2d_set_grid has not been called");
    if (num_global < 0 || num_local < 1) return f2(h, ADI_ERR_BAD_ARG, "num_global >= 0 and num_local >= 1");
    if (!(dt > 0) || !std::isfinite(dt)) return f2(h, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    if (h->prec == ADI_FP64) return time_step<double>(h, dt, num_global, num_local, bnd, iters);
    return time_step<float>(h, dt, num_global, num_local, bnd, iters);
}

adi_status adi2d_time_step(adi2d_handle *h, double dt, int num_global, int num_local, int *iters_used)
{
    return step2(h, dt, num_global, num_local, false, iters_used);
}

adi_status adi2d_step(adi2d_handle *h, double dt, int num_global, int num_local, int *iters_used)
{
    return step2(h, dt, num_global, num_local, true, iters_used);
}

adi_status adi2d_step_tol(adi2d_handle *h, double dt, int max_global, int num_local, double tol, int *iters_used,
                          double *residual)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (!h->grid_set) return f2(h, ADI_ERR_STATE, "adi2d_set_grid has not been called");
    if (max_global < 1 || num_local < 1) return f2(h, ADI_ERR_BAD_ARG, "max_global >= 1 and num_local >= 1");
    if (!(dt > 0) || !std::isfinite(dt)) return f2(h, ADI_ERR_BAD_ARG, "dt must be positive and finite");
    if (!(tol >= 0)) return f2(h, ADI_ERR_BAD_ARG, "tol must be >= 0");
    if (h->prec == ADI_FP64) return time_step_tol<double>(h, dt, max_global, num_local, tol, true, iters_used, residual);
    return time_step_tol<float>(h, dt, max_global, num_local, tol, true, iters_used, residual);
}

adi_status adi2d_get_state(adi2d_handle *h, int which, void *u, void *v, void *T)
{
    if (!h || !u || !v || !T || (which != 0 && which != 1)) return ADI_ERR_BAD_ARG;
    const size_t fb = (size_t)h->nx * h->ny * es2(h);
    void *dst[3] = {u, v, T};
    for (int f = 0; f < 3; f++)
        CK2(cudaMemcpyAsync(dst[f], h->d_L[which ? NXT : CUR][f], fb, cudaMemcpyDeviceToHost, h->stream));
    CK2(cudaStreamSynchronize(h->stream));
    return ADI_OK;
}

adi_status adi2d_set_state(adi2d_handle *h, const void *u, const void *v, const void *T)
{
    if (!h || !u || !v || !T) return ADI_ERR_BAD_ARG;
    const size_t fb = (size_t)h->nx * h->ny * es2(h);
    const void *src[3] = {u, v, T};
    for (int f = 0; f < 3; f++)
        CK2(cudaMemcpyAsync(h->d_L[CUR][f], src[f], fb, cudaMemcpyHostToDevice, h->stream));
    CK2(cudaStreamSynchronize(h->stream));
    return ADI_OK;
}

adi_status adi2d_get_layer(adi2d_handle *h, int outdimx, int outdimy, double *vel2, double *T)
{
    if (!h || !vel2 || !T || outdimx < 0 || outdimy < 0) return ADI_ERR_BAD_ARG;
    if (outdimx == 0) outdimx = h->nx;
    if (outdimy == 0) outdimy = h->ny;
    const size_t n = (size_t)h->nx * h->ny, es = es2(h);
    std::vector<unsigned char> buf(3 * n * es);
    for (int f = 0; f < 3; f++)
        CK2(cudaMemcpyAsync(buf.data() + f * n * es, h->d_L[NXT][f], n * es, cudaMemcpyDeviceToHost, h->stream));
    CK2(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < outdimx; i++)
        for (int j = 0; j < outdimy; j++) {
            const size_t src = (size_t)(i * h->nx / outdimx) * h->ny + (j * h->ny / outdimy);
            const size_t o = (size_t)i * outdimy + j;
            double a[3];
            for (int f = 0; f < 3; f++)
                a[f] = es == 8 ? ((const double *)buf.data())[f * n + src] : ((const float *)buf.data())[f * n + src];
            vel2[2 * o] = a[0];
            vel2[2 * o + 1] = a[1];
            T[o] = a[2];
        }
    return ADI_OK;
}

adi_status adi2d_last_error(adi2d_handle *h, double *err, int *iters)
{
    if (!h) return ADI_ERR_BAD_ARG;
    if (err) *err = h->last_err;
    if (iters) *iters = h->last_iters;
    return ADI_OK;
}

const char *adi2d_last_error_string(const adi2d_handle *h)
{
    if (!h) return "null handle";
    return h->msg.c_str();
}

} // extern "C"
