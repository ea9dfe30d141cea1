// Exact segmented tridiagonal sweep: one thread per grid line, four variables.
//
// Replaces the reference's per-direction sweep (CPU: AdiSolver3D::SolveDirection,
// AdiSolver3D.cpp:587-603 -> SolveSegment/BuildMatrix/ApplyBC0/ApplyBC1/
// SolveTridiagonal/UpdateSegment, :687-852 and Common/Algorithms.h:21-39;
// GPU twin: solve_segments / solve_tridiagonal, AdiSolver3D.cu:75-495).
//
// Every line of the sweep direction is one tridiagonal system that is block
// diagonal: each segment of the line is a block, nodes outside segments have no
// row.  A thread walks its line twice in lock step with the 31 other lines of
// its warp (lanes = neighbouring lines, so each access of a warp is one
// contiguous row of the grid for X and Y sweeps):
//   forward:  builds each row (BC row at a segment end node, BuildMatrix row at
//             an IN node) and runs the Thomas elimination, writing the modified
//             coefficients c' (one per matrix: velocity, temperature) and d' (one
//             per variable) to a line-interleaved scratch area;
//   backward: back-substitutes, writes x to `next` for every segment node and the
//             nonlinear merge temp_out = (temp_in + x)/2 at IN nodes (twice when
//             the time step's extra per-iteration merge falls on this sweep,
//             AdiSolver3D.cpp:347-357).
// Velocities share one matrix (a, b, c depend only on the advecting component and
// v_vis), so their c' is computed once; this is the same arithmetic the reference
// repeats per variable.
//
// Exactness: this file is compiled with --fmad=false and spells out every
// operation in the reference's order (e.g. cur*3/dt, (-w)/(2h) - vis), divisions
// are IEEE divisions, so the float results equal the reference CPU solver's bit
// for bit.  A segment's first row never looks at the previous segment
// (c'0 = c0/b0, d'0 = d0/b0, as Algorithms.h:25-26), and a segment's last row
// starts the back-substitution (x = d'), so segments stay independent; a node
// that ends one segment and starts the next carries the later segment's start row,
// which is the value the reference writes last.  Nodes outside segments are never
// written.
//
// Scratch: 6 values per line position, layout [q][position][line]; a warp's 32
// lines are adjacent, so scratch traffic is coalesced.
#include "adi_b200.h"
#include "adi_internal.cuh"

#include <climits>

namespace adi {

template <typename R>
struct RowKind {
    enum : int { NONE = 0, START = 1, INTERIOR = 2, END = 3, SHARED = 4 };
};

// DissFunc along the sweep direction on temp (TimeLayer3D.h:554-588), operand
// order of the reference for each direction.
template <typename R, int DIR>
__device__ __forceinline__ R diss(const CLayer<R> &t, long long off, long long sl, long long so1, long long so2,
                                  const SweepConst<R> &k)
{
    const R *U = t.f[0], *V = t.f[1], *W = t.f[2];
    if (DIR == 0) {
        R u_x = (U[off + sl] - U[off - sl]) / k.two_dx;
        R v_x = (V[off + sl] - V[off - sl]) / k.two_dx;
        R w_x = (W[off + sl] - W[off - sl]) / k.two_dx;
        R u_y = (U[off + so1] - U[off - so1]) / k.two_dy;
        R u_z = (U[off + so2] - U[off - so2]) / k.two_dz;
        return R(2) * u_x * u_x + v_x * v_x + w_x * w_x + v_x * u_y + w_x * u_z;
    } else if (DIR == 1) {
        R u_y = (U[off + sl] - U[off - sl]) / k.two_dy;
        R v_y = (V[off + sl] - V[off - sl]) / k.two_dy;
        R w_y = (W[off + sl] - W[off - sl]) / k.two_dy;
        R v_x = (V[off + so1] - V[off - so1]) / k.two_dx;
        R v_z = (V[off + so2] - V[off - so2]) / k.two_dz;
        return u_y * u_y + R(2) * v_y * v_y + w_y * w_y + u_y * v_x + w_y * v_z;
    } else {
        R u_z = (U[off + sl] - U[off - sl]) / k.two_dz;
        R v_z = (V[off + sl] - V[off - sl]) / k.two_dz;
        R w_z = (W[off + sl] - W[off - sl]) / k.two_dz;
        R w_x = (W[off + so1] - W[off - so1]) / k.two_dx;
        R w_y = (W[off + so2] - W[off - so2]) / k.two_dy;
        return u_z * u_z + v_z * v_z + R(2) * w_z * w_z + u_z * w_x + v_z * w_y;
    }
}

__device__ __forceinline__ int row_kind(uint8_t cm, uint8_t c0, uint8_t cp, bool has_m, bool has_p)
{
    if (code_is_in(c0)) return 2;
    bool inm = has_m && code_is_in(cm);
    bool inp = has_p && code_is_in(cp);
    if (inm && inp) return 4;
    if (inp) return 1;
    if (inm) return 3;
    return 0;
}

template <typename R, int DIR>
__global__ void __launch_bounds__(128) sweep_exact_kernel(DomainView<R> d, LineGeom g, const int *__restrict__ line_lo,
                                                          const int *__restrict__ line_hi, CLayer<R> cur, CLayer<R> tin,
                                                          Layer<R> next, Layer<R> tout, R *__restrict__ scratch,
                                                          SweepConst<R> k, int merges)
{
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = line < g.nlines;
    int lo = INT_MAX, hi = -1;
    if (valid) {
        int a = line_lo[line], b = line_hi[line];
        if (a >= 0) { lo = a; hi = b; }
    }
    const unsigned full = 0xffffffffu;
    const int wlo = __reduce_min_sync(full, lo);
    const int whi = __reduce_max_sync(full, hi);
    if (!valid || hi < 0) return;  // after the warp-wide reductions

    const long long sl = g.stride;
    // off-line strides for DissFunc: X -> (y, z), Y -> (x, z), Z -> (x, y)
    const long long sx = (long long)g.ny * g.nz, sy = g.nz;
    const long long so1 = DIR == 0 ? sy : sx;
    const long long so2 = DIR == 2 ? sy : 1;
    const long long base = line_base(DIR, g, line);
    const long long qstride = (long long)g.len * g.nlines;  // between scratch quantities
    R *scr = scratch + line;

    const R *Fd = tin.f[DIR];  // advecting velocity component along the line
    const R *Tt = tin.f[3];
    const R three = k.three, dt = k.dt;

    // ---------------- forward elimination ----------------
    R cpv = R(0), cpt = R(0), dp0 = R(0), dp1 = R(0), dp2 = R(0), dp3 = R(0);
    for (int p = wlo; p <= whi; p++) {
        if (p < lo || p > hi) continue;
        const long long off = base + (long long)p * sl;
        const uint8_t c0 = d.code[off];
        const uint8_t cm = p > 0 ? d.code[off - sl] : uint8_t(NODE_OUT);
        const uint8_t cp = p + 1 < g.len ? d.code[off + sl] : uint8_t(NODE_OUT);
        const int kind = row_kind(cm, c0, cp, p > 0, p + 1 < g.len);
        if (kind == 0) continue;
        R ncv, nct, n0, n1, n2, n3;
        if (kind == 2) {
            // BuildMatrix row (AdiSolver3D.cpp:759-797)
            const R w = Fd[off];
            const R av = -w / k.two_h - k.vis_v;
            const R at = -w / k.two_h - k.vis_t;
            const R cv = w / k.two_h - k.vis_v;
            const R ct = w / k.two_h - k.vis_t;
            R dd[4];
#pragma unroll
            for (int v = 0; v < 4; v++) dd[v] = cur.f[v][off] * three / dt;
            dd[DIR] = dd[DIR] - k.v_T * ((Tt[off + sl] - Tt[off - sl]) / k.two_h);
            dd[3] = dd[3] + k.t_phi * diss<R, DIR>(tin, off, sl, so1, so2, k);
            // Thomas step (Algorithms.h:30-31)
            ncv = cv / (k.b_v - av * cpv);
            nct = ct / (k.b_t - at * cpt);
            n0 = (dd[0] - dp0 * av) / (k.b_v - av * cpv);
            n1 = (dd[1] - dp1 * av) / (k.b_v - av * cpv);
            n2 = (dd[2] - dp2 * av) / (k.b_v - av * cpv);
            n3 = (dd[3] - dp3 * at) / (k.b_t - at * cpt);
        } else if (kind == 1 || kind == 4) {
            // first row of a segment: ApplyBC0 (AdiSolver3D.cpp:804-827), then
            // c'0 = c0/b0, d'0 = d0/b0 (Algorithms.h:25-26)
            const bool vf = (c0 & CODE_VEL_FREE) != 0, tf = (c0 & CODE_TEMP_FREE) != 0;
            const R bv = vf ? R(2) : R(1), cvv = vf ? R(-1) : R(0);
            const R bt = tf ? R(2) : R(1), ctt = tf ? R(-1) : R(0);
            const R d0 = vf ? R(0) : d.nv[0][off];
            const R d1 = vf ? R(0) : d.nv[1][off];
            const R d2 = vf ? R(0) : d.nv[2][off];
            const R d3 = tf ? R(0) : d.nv[3][off];
            ncv = cvv / bv;
            nct = ctt / bt;
            n0 = d0 / bv;
            n1 = d1 / bv;
            n2 = d2 / bv;
            n3 = d3 / bt;
        } else {
            // last row of a segment: ApplyBC1 (AdiSolver3D.cpp:829-852), c = 0
            const bool vf = (c0 & CODE_VEL_FREE) != 0, tf = (c0 & CODE_TEMP_FREE) != 0;
            const R av = vf ? R(-1) : R(0), bv = vf ? R(2) : R(1);
            const R at = tf ? R(-1) : R(0), bt = tf ? R(2) : R(1);
            const R d0 = vf ? R(0) : d.nv[0][off];
            const R d1 = vf ? R(0) : d.nv[1][off];
            const R d2 = vf ? R(0) : d.nv[2][off];
            const R d3 = tf ? R(0) : d.nv[3][off];
            ncv = R(0);
            nct = R(0);
            n0 = (d0 - dp0 * av) / (bv - av * cpv);
            n1 = (d1 - dp1 * av) / (bv - av * cpv);
            n2 = (d2 - dp2 * av) / (bv - av * cpv);
            n3 = (d3 - dp3 * at) / (bt - at * cpt);
        }
        cpv = ncv; cpt = nct; dp0 = n0; dp1 = n1; dp2 = n2; dp3 = n3;
        R *s = scr + (long long)p * g.nlines;
        s[0 * qstride] = ncv;
        s[1 * qstride] = nct;
        s[2 * qstride] = n0;
        s[3 * qstride] = n1;
        s[4 * qstride] = n2;
        s[5 * qstride] = n3;
    }

    // ---------------- back substitution + write-back + merge ----------------
    R x0 = R(0), x1 = R(0), x2 = R(0), x3 = R(0);
    for (int p = whi; p >= wlo; p--) {
        if (p < lo || p > hi) continue;
        const long long off = base + (long long)p * sl;
        const uint8_t c0 = d.code[off];
        const uint8_t cm = p > 0 ? d.code[off - sl] : uint8_t(NODE_OUT);
        const uint8_t cp = p + 1 < g.len ? d.code[off + sl] : uint8_t(NODE_OUT);
        const int kind = row_kind(cm, c0, cp, p > 0, p + 1 < g.len);
        if (kind == 0) continue;
        const R *s = scr + (long long)p * g.nlines;
        const R ncv = s[0 * qstride], nct = s[1 * qstride];
        const R n0 = s[2 * qstride], n1 = s[3 * qstride], n2 = s[4 * qstride], n3 = s[5 * qstride];
        if (kind == 3) {
            x0 = n0; x1 = n1; x2 = n2; x3 = n3;          // x[n-1] = d[n-1]
        } else {
            x0 = n0 - ncv * x0;                           // x[i] = d[i] - c[i]*x[i+1]
            x1 = n1 - ncv * x1;
            x2 = n2 - ncv * x2;
            x3 = n3 - nct * x3;
        }
        next.f[0][off] = x0;
        next.f[1][off] = x1;
        next.f[2][off] = x2;
        next.f[3][off] = x3;
        if (kind == 2) {
            // MergeFieldTo: temp = (temp + next) / 2 (TimeLayer3D.h:430), once or twice
            R m0 = (tin.f[0][off] + x0) / R(2);
            R m1 = (tin.f[1][off] + x1) / R(2);
            R m2 = (tin.f[2][off] + x2) / R(2);
            R m3 = (tin.f[3][off] + x3) / R(2);
            if (merges == 2) {
                m0 = (m0 + x0) / R(2);
                m1 = (m1 + x1) / R(2);
                m2 = (m2 + x2) / R(2);
                m3 = (m3 + x3) / R(2);
            }
            tout.f[0][off] = m0;
            tout.f[1][off] = m1;
            tout.f[2][off] = m2;
            tout.f[3][off] = m3;
        }
    }
}

template <typename R>
cudaError_t launch_sweep_exact(int dir, const DomainView<R> &d, const int *line_lo, const int *line_hi,
                               CLayer<R> cur, CLayer<R> temp_in, Layer<R> next, Layer<R> temp_out,
                               R *scratch, const SweepConst<R> &k, int merges, cudaStream_t s)
{
    LineGeom g = line_geom(dir, d.nx, d.ny, d.nz);
    const int threads = 128;
    const int blocks = (g.nlines + threads - 1) / threads;
    if (dir == 0)
        sweep_exact_kernel<R, 0><<<blocks, threads, 0, s>>>(d, g, line_lo, line_hi, cur, temp_in, next, temp_out,
                                                             scratch, k, merges);
    else if (dir == 1)
        sweep_exact_kernel<R, 1><<<blocks, threads, 0, s>>>(d, g, line_lo, line_hi, cur, temp_in, next, temp_out,
                                                             scratch, k, merges);
    else
        sweep_exact_kernel<R, 2><<<blocks, threads, 0, s>>>(d, g, line_lo, line_hi, cur, temp_in, next, temp_out,
                                                             scratch, k, merges);
    return cudaGetLastError();
}

template cudaError_t launch_sweep_exact<float>(int, const DomainView<float> &, const int *, const int *,
                                               CLayer<float>, CLayer<float>, Layer<float>, Layer<float>, float *,
                                               const SweepConst<float> &, int, cudaStream_t);
template cudaError_t launch_sweep_exact<double>(int, const DomainView<double> &, const int *, const int *,
                                                CLayer<double>, CLayer<double>, Layer<double>, Layer<double>,
                                                double *, const SweepConst<double> &, int, cudaStream_t);

} // namespace adi

// ===========================================================================
// Allocation-free entry point: adi_sweep_exact_static.
//
// Some callers cannot allocate device memory at run time: hosts whose device
// memory is entirely owned by their own pool allocator, solver loops that must
// not hit cudaMalloc's implicit synchronisation and latency in their time step,
// and code running where allocation is forbidden.  For them this entry point runs
// one exact sweep (the same arithmetic as sweep_exact_kernel) on device arrays the
// caller owns: node types and BC codes as in Grid3D's Node (uint8, three arrays),
// the node values, and the four fields of cur, temp_in, next and temp_out.  It
// needs no segment lists (each line finds its own segment range) and no
// allocation: its elimination scratch is the fixed array below, shared by every
// call.  Lines are processed in batches that fit the array, one launch per batch,
// in stream order.
// ===========================================================================
namespace adi {

constexpr size_t STATIC_SCRATCH_BYTES = (size_t)16 << 20;   // 16 MiB per device
static __device__ __align__(256) unsigned char g_static_scratch[STATIC_SCRATCH_BYTES];

template <typename R, int DIR>
__global__ void __launch_bounds__(128)
    sweep_exact_static_kernel(LineGeom g, int line0, int nbatch, const uint8_t *__restrict__ ntype,
                              const uint8_t *__restrict__ nbcv, const uint8_t *__restrict__ nbct, CLayer<R> nv,
                              CLayer<R> cur, CLayer<R> tin, Layer<R> next, Layer<R> tout, R *__restrict__ scratch,
                              SweepConst<R> k, int merges)
{
    const int lb = blockIdx.x * blockDim.x + threadIdx.x;   // line within the batch
    const int line = line0 + lb;
    const bool valid = lb < nbatch && line < g.nlines;
    const long long sl = g.stride;
    const long long base = valid ? line_base(DIR, g, line) : 0;
    auto code_at = [&](long long off) -> uint8_t {
        return (uint8_t)(ntype[off] | (nbcv[off] == BC_FREE ? CODE_VEL_FREE : 0) |
                         (nbct[off] == BC_FREE ? CODE_TEMP_FREE : 0));
    };
    // Caller-owned masks are not checked on the host the way adi_set_mask checks
    // them, so a line that breaks the solver contract where it would make a read
    // leave the arrays -- a NODE_IN cell at either end of the line, or any NODE_IN
    // cell in a line on the outer frame (its off-line stencil crosses the face) --
    // is skipped whole: its nodes are neither read as rows nor written.
    bool usable = valid;
    if (valid) {
        int c1, c2, n1, n2;   // the line's two fixed coordinates and their extents
        if (DIR == 0) { c1 = line / g.nz; c2 = line % g.nz; n1 = g.ny; n2 = g.nz; }
        else if (DIR == 1) { c1 = line / g.nz; c2 = line % g.nz; n1 = g.nx; n2 = g.nz; }
        else { c1 = line / g.ny; c2 = line % g.ny; n1 = g.nx; n2 = g.ny; }
        const bool on_frame = c1 == 0 || c1 == n1 - 1 || c2 == 0 || c2 == n2 - 1;
        const bool end_in = ntype[base] == NODE_IN || ntype[base + (long long)(g.len - 1) * sl] == NODE_IN;
        if (end_in) usable = false;
        if (on_frame) {
            for (int q = 1; q + 1 < g.len && usable; q++)
                if (ntype[base + (long long)q * sl] == NODE_IN) usable = false;
        }
    }
    // segment range of the line, by the rule of Grid3D::GenerateListSegments
    int lo = INT_MAX, hi = -1;
    if (usable) {
        int state = 0, start = 0;
        for (int q = 0; q + 1 < g.len; q++) {
            const bool in = ntype[base + (long long)(q + 1) * sl] == NODE_IN;
            if (in) {
                if (!state) start = q;
                state = 1;
            } else if (state) {
                if (lo == INT_MAX) lo = start;
                hi = q + 1;
                state = 0;
            }
        }
        if (hi < 0) lo = INT_MAX;
    }
    const unsigned full = 0xffffffffu;
    const int wlo = __reduce_min_sync(full, lo);
    const int whi = __reduce_max_sync(full, hi);
    if (!usable || hi < 0) return;

    const long long sx = (long long)g.ny * g.nz, sy = g.nz;
    const long long so1 = DIR == 0 ? sy : sx;
    const long long so2 = DIR == 2 ? sy : 1;
    const long long qstride = (long long)g.len * nbatch;
    R *scr = scratch + lb;
    const R *Fd = tin.f[DIR];
    const R *Tt = tin.f[3];
    const R three = k.three, dt = k.dt;

    R cpv = R(0), cpt = R(0), dp0 = R(0), dp1 = R(0), dp2 = R(0), dp3 = R(0);
    for (int p = wlo; p <= whi; p++) {
        if (p < lo || p > hi) continue;
        const long long off = base + (long long)p * sl;
        const uint8_t c0 = code_at(off);
        const uint8_t cm = p > 0 ? code_at(off - sl) : uint8_t(NODE_OUT);
        const uint8_t cp = p + 1 < g.len ? code_at(off + sl) : uint8_t(NODE_OUT);
        const int kind = row_kind(cm, c0, cp, p > 0, p + 1 < g.len);
        if (kind == 0) continue;
        R ncv, nct, n0, n1, n2, n3;
        if (kind == 2) {
            const R w = Fd[off];
            const R av = -w / k.two_h - k.vis_v;
            const R at = -w / k.two_h - k.vis_t;
            const R cv = w / k.two_h - k.vis_v;
            const R ct = w / k.two_h - k.vis_t;
            R dd[4];
#pragma unroll
            for (int v = 0; v < 4; v++) dd[v] = cur.f[v][off] * three / dt;
            dd[DIR] = dd[DIR] - k.v_T * ((Tt[off + sl] - Tt[off - sl]) / k.two_h);
            dd[3] = dd[3] + k.t_phi * diss<R, DIR>(tin, off, sl, so1, so2, k);
            ncv = cv / (k.b_v - av * cpv);
            nct = ct / (k.b_t - at * cpt);
            n0 = (dd[0] - dp0 * av) / (k.b_v - av * cpv);
            n1 = (dd[1] - dp1 * av) / (k.b_v - av * cpv);
            n2 = (dd[2] - dp2 * av) / (k.b_v - av * cpv);
            n3 = (dd[3] - dp3 * at) / (k.b_t - at * cpt);
        } else if (kind == 1 || kind == 4) {
            const bool vf = (c0 & CODE_VEL_FREE) != 0, tf = (c0 & CODE_TEMP_FREE) != 0;
            const R bv = vf ? R(2) : R(1), cvv = vf ? R(-1) : R(0);
            const R bt = tf ? R(2) : R(1), ctt = tf ? R(-1) : R(0);
            ncv = cvv / bv;
            nct = ctt / bt;
            n0 = (vf ? R(0) : nv.f[0][off]) / bv;
            n1 = (vf ? R(0) : nv.f[1][off]) / bv;
            n2 = (vf ? R(0) : nv.f[2][off]) / bv;
            n3 = (tf ? R(0) : nv.f[3][off]) / bt;
        } else {
            const bool vf = (c0 & CODE_VEL_FREE) != 0, tf = (c0 & CODE_TEMP_FREE) != 0;
            const R av = vf ? R(-1) : R(0), bv = vf ? R(2) : R(1);
            const R at = tf ? R(-1) : R(0), bt = tf ? R(2) : R(1);
            ncv = R(0);
            nct = R(0);
            n0 = ((vf ? R(0) : nv.f[0][off]) - dp0 * av) / (bv - av * cpv);
            n1 = ((vf ? R(0) : nv.f[1][off]) - dp1 * av) / (bv - av * cpv);
            n2 = ((vf ? R(0) : nv.f[2][off]) - dp2 * av) / (bv - av * cpv);
            n3 = ((tf ? R(0) : nv.f[3][off]) - dp3 * at) / (bt - at * cpt);
        }
        cpv = ncv; cpt = nct; dp0 = n0; dp1 = n1; dp2 = n2; dp3 = n3;
        R *s = scr + (long long)p * nbatch;
        s[0 * qstride] = ncv;
        s[1 * qstride] = nct;
        s[2 * qstride] = n0;
        s[3 * qstride] = n1;
        s[4 * qstride] = n2;
        s[5 * qstride] = n3;
    }

    R x0 = R(0), x1 = R(0), x2 = R(0), x3 = R(0);
    for (int p = whi; p >= wlo; p--) {
        if (p < lo || p > hi) continue;
        const long long off = base + (long long)p * sl;
        const uint8_t c0 = code_at(off);
        const uint8_t cm = p > 0 ? code_at(off - sl) : uint8_t(NODE_OUT);
        const uint8_t cp = p + 1 < g.len ? code_at(off + sl) : uint8_t(NODE_OUT);
        const int kind = row_kind(cm, c0, cp, p > 0, p + 1 < g.len);
        if (kind == 0) continue;
        const R *s = scr + (long long)p * nbatch;
        const R ncv = s[0 * qstride], nct = s[1 * qstride];
        const R n0 = s[2 * qstride], n1 = s[3 * qstride], n2 = s[4 * qstride], n3 = s[5 * qstride];
        if (kind == 3) {
            x0 = n0; x1 = n1; x2 = n2; x3 = n3;
        } else {
            x0 = n0 - ncv * x0;
            x1 = n1 - ncv * x1;
            x2 = n2 - ncv * x2;
            x3 = n3 - nct * x3;
        }
        next.f[0][off] = x0;
        next.f[1][off] = x1;
        next.f[2][off] = x2;
        next.f[3][off] = x3;
        if (kind == 2) {
            R m0 = (tin.f[0][off] + x0) / R(2);
            R m1 = (tin.f[1][off] + x1) / R(2);
            R m2 = (tin.f[2][off] + x2) / R(2);
            R m3 = (tin.f[3][off] + x3) / R(2);
            if (merges == 2) {
                m0 = (m0 + x0) / R(2);
                m1 = (m1 + x1) / R(2);
                m2 = (m2 + x2) / R(2);
                m3 = (m3 + x3) / R(2);
            }
            tout.f[0][off] = m0;
            tout.f[1][off] = m1;
            tout.f[2][off] = m2;
            tout.f[3][off] = m3;
        }
    }
}

namespace {

// Device address of g_static_scratch in the current device's context.  Host code
// cannot pass the symbol itself (its host-side name is a stand-in, not a device
// address), so every call looks the address up with the device current; the
// lookup is a host-side table read once the module is loaded, and looking it up
// each time keeps it right after a device reset or in another driver context.
// The first lookup on a device loads the module.
cudaError_t static_scratch(void **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    *out = p;
    return cudaSuccess;
}

template <typename R>
adi_status static_sweep(const adi_static_sweep_args *a, void *scratch)
{
    const LineGeom g = line_geom(a->dir, a->dimx, a->dimy, a->dimz);
    const long long per_line = 6LL * g.len * (long long)sizeof(R);
    const long long max_batch = (long long)STATIC_SCRATCH_BYTES / per_line;
    if (max_batch < 128) return ADI_ERR_CAPACITY;   // line too long for the fixed scratch
    const int batch = (int)(max_batch < g.nlines ? (max_batch / 128) * 128 : g.nlines);
    // constants with BuildMatrix's operations (AdiSolver3D.cpp:744-752,760-797)
    SweepConst<R> k;
    const R dx = (R)a->dx, dy = (R)a->dy, dz = (R)a->dz, dt = (R)a->dt;
    const R hh = a->dir == 0 ? dx : (a->dir == 1 ? dy : dz);
    k.three = R(3);
    k.dt = dt;
    k.two_h = R(2) * hh;
    k.vis_v = (R)a->params.v_vis / (hh * hh);
    k.vis_t = (R)a->params.t_vis / (hh * hh);
    k.b_v = R(3) / dt + R(2) * k.vis_v;
    k.b_t = R(3) / dt + R(2) * k.vis_t;
    k.v_T = (R)a->params.v_T;
    k.t_phi = (R)a->params.t_phi;
    k.two_dx = R(2) * dx;
    k.two_dy = R(2) * dy;
    k.two_dz = R(2) * dz;
    CLayer<R> nv, cur, tin;
    Layer<R> next, tout;
    for (int v = 0; v < 4; v++) {
        nv.f[v] = (const R *)a->node_value[v];
        cur.f[v] = (const R *)a->cur[v];
        tin.f[v] = (const R *)a->temp_in[v];
        next.f[v] = (R *)a->next[v];
        tout.f[v] = (R *)a->temp_out[v];
    }
    cudaStream_t s = (cudaStream_t)a->stream;
    for (int line0 = 0; line0 < g.nlines; line0 += batch) {
        const int nb = g.nlines - line0 < batch ? g.nlines - line0 : batch;
        const int threads = 128, blocks = (nb + threads - 1) / threads;
#define SL(D)                                                                                                   \
    sweep_exact_static_kernel<R, D><<<blocks, threads, 0, s>>>(g, line0, nb, a->node_type, a->bc_vel, a->bc_temp, \
                                                               nv, cur, tin, next, tout, (R *)scratch, k, a->merges)
        if (a->dir == 0) SL(0);
        else if (a->dir == 1) SL(1);
        else SL(2);
#undef SL
        // peek, not get: a launch error stays pending for the caller's own
        // cudaGetLastError (this entry point has no handle to carry a message)
        if (cudaPeekAtLastError() != cudaSuccess) return ADI_ERR_CUDA;
    }
    return ADI_OK;
}

} // namespace
} // namespace adi

extern "C" adi_status adi_sweep_exact_static(const adi_static_sweep_args *a)
{
    using namespace adi;
    if (!a || a->dir < 0 || a->dir > 2 || a->dimx < 3 || a->dimy < 3 || a->dimz < 3) return ADI_ERR_BAD_ARG;
    if (a->precision != ADI_FP32 && a->precision != ADI_FP64) return ADI_ERR_BAD_ARG;
    if (a->merges != 1 && a->merges != 2) return ADI_ERR_BAD_ARG;
    if (!(a->dt > 0) || !(a->dx > 0) || !(a->dy > 0) || !(a->dz > 0)) return ADI_ERR_BAD_ARG;
    if (!a->node_type || !a->bc_vel || !a->bc_temp) return ADI_ERR_BAD_ARG;
    for (int v = 0; v < 4; v++)
        if (!a->node_value[v] || !a->cur[v] || !a->temp_in[v] || !a->next[v] || !a->temp_out[v])
            return ADI_ERR_BAD_ARG;
    // an error left pending by earlier work is the caller's: report it, keep it
    if (cudaPeekAtLastError() != cudaSuccess) return ADI_ERR_CUDA;
    void *scratch = nullptr;
    if (static_scratch(&scratch) != cudaSuccess) return ADI_ERR_CUDA;
    if (a->precision == ADI_FP64) return static_sweep<double>(a, scratch);
    return static_sweep<float>(a, scratch);
}

extern "C" size_t adi_static_scratch_bytes(void) { return adi::STATIC_SCRATCH_BYTES; }
