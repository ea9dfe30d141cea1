// Discrete adjoint of the time step (no counterpart in the reference).
//
// The forward sweep of direction dir solves, on every line, A(t) x = d(s, t, nv)
// (rows: BuildMatrix at IN nodes, ApplyBC0/ApplyBC1 at segment ends, as in
// sweep_exact.cu), writes x to the destination layer on the segment nodes and
// merges temp_out = temp_in/2 + x/2 on NODE_IN (temp_in/4 + 3x/4 when the
// iteration's extra merge falls on the sweep).  Its adjoint, given xbar (the
// destination's adjoint on the segment nodes plus the merge's share of the temp
// adjoint), is one transposed tridiagonal solve per line, lambda = A^-T xbar, and
//   sbar  += 3/dt lambda                         IN rows (d = 3/dt s + ...)
//   nvbar += lambda                              Dirichlet rows (d = node value)
//   tbar[dir] += lambda (x[p-1] - x[p+1])/(2h)   IN rows (a, c carry w = t[dir])
//   tbar[T][p-+1] +-= v_T lambda/(2h)            velocity along dir (pressure term)
//   tbar += t_phi lambda dDiss/dt                temperature rows
// A^T keeps the line's block structure: its row p has sub-diagonal A[p-1][p]
// (row p-1's c), diagonal A[p][p] and super-diagonal A[p+1][p] (row p+1's a).
//
// adjoint_sweep_kernel: one thread per line, two passes like the exact sweep
// (forward elimination of A^T into a line-interleaved scratch, then back
// substitution with the accumulations).  The dissipation terms that reach other
// lines (the advecting component's off-line derivatives) go to two planes that
// adjoint_gather_kernel folds into tbar afterwards, so every cell is written by
// one thread only and the result does not depend on scheduling.
#include "adi_internal.cuh"

#include <climits>

namespace adi {

namespace {

enum : int { A_NONE = 0, A_START = 1, A_IN = 2, A_END = 3, A_SHARED = 4 };

__device__ __forceinline__ int akind(bool inm, bool in0, bool inp)
{
    if (in0) return A_IN;
    if (inm && inp) return A_SHARED;
    if (inp) return A_START;
    if (inm) return A_END;
    return A_NONE;
}

// Entries of row p of the forward matrix of one variable class (velocity: vf =
// bc_vel FREE, vis_v, b_v; temperature: bc_temp, vis_t, b_t).
template <typename R>
struct RowABC {
    R a, b, c;
};

template <typename R>
__device__ __forceinline__ RowABC<R> row_entries(int kind, bool free_bc, R r, R vis, R b_in)
{
    RowABC<R> e;
    if (kind == A_IN) {
        e.a = -r - vis;
        e.b = b_in;
        e.c = r - vis;
    } else if (kind == A_START || kind == A_SHARED) {
        const bool fr = free_bc && kind == A_START;
        e.a = R(0);
        e.b = fr ? R(2) : R(1);
        e.c = fr ? R(-1) : R(0);
    } else if (kind == A_END) {
        e.a = free_bc ? R(-1) : R(0);
        e.b = free_bc ? R(2) : R(1);
        e.c = R(0);
    } else {
        e.a = R(0);
        e.b = R(1);
        e.c = R(0);
    }
    return e;
}

} // namespace

template <typename R, int DIR>
__global__ void __launch_bounds__(128)
    adjoint_sweep_kernel(DomainView<R> d, LineGeom g, const int *__restrict__ line_lo, const int *__restrict__ line_hi,
                         CLayer<R> ti, CLayer<R> xs, Layer<R> sbar, Layer<R> dbar, Layer<R> tbar, Layer<R> nvbar,
                         R *__restrict__ ga, R *__restrict__ gb, R *__restrict__ scratch, SweepConst<R> k, int merges)
{
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    if (line >= g.nlines) return;
    const int lo = line_lo[line];
    if (lo < 0) return;   // no segment on this line
    const int hi = line_hi[line];
    const long long sl = g.stride;
    const long long sx = (long long)g.ny * g.nz, sy = g.nz;
    const long long so1 = DIR == 0 ? sy : sx;   // off-line axes: X -> (y, z), Y -> (x, z), Z -> (x, y)
    const long long so2 = DIR == 2 ? sy : 1;
    const R h1 = DIR == 0 ? k.inv_two_dy : k.inv_two_dx;
    const R h2 = DIR == 2 ? k.inv_two_dy : k.inv_two_dz;
    const long long base = line_base(DIR, g, line);
    const long long qstride = (long long)g.len * g.nlines;
    R *scr = scratch + line;
    const R mx = merges == 2 ? R(0.75) : R(0.5);
    const R mt = merges == 2 ? R(0.25) : R(0.5);
    const R *W = ti.f[DIR];

    auto code_at = [&](int p) -> uint8_t { return (p >= 0 && p < g.len) ? d.code[base + (long long)p * sl] : uint8_t(NODE_OUT); };
    auto kind_at = [&](int p) -> int {
        if (p < 0 || p >= g.len) return A_NONE;
        return akind(code_is_in(code_at(p - 1)), code_is_in(code_at(p)), code_is_in(code_at(p + 1)));
    };
    auto entries = [&](int p, int kind, int m) -> RowABC<R> {
        const uint8_t c = code_at(p);
        const bool fr = m == 0 ? (c & CODE_VEL_FREE) != 0 : (c & CODE_TEMP_FREE) != 0;
        const R r = kind == A_IN ? W[base + (long long)p * sl] * k.inv_two_h : R(0);
        return row_entries<R>(kind, fr, r, m == 0 ? k.vis_v : k.vis_t, m == 0 ? k.b_v : k.b_t);
    };

    // ---------------- pass 1: xbar, the merge, forward elimination of A^T ----------------
    int km = kind_at(lo - 1), k0 = kind_at(lo);
    R cpv = R(0), cpt = R(0), dp[4] = {R(0), R(0), R(0), R(0)};
    for (int p = lo; p <= hi; p++) {
        const int kp = kind_at(p + 1);
        const long long off = base + (long long)p * sl;
        R xb[4] = {R(0), R(0), R(0), R(0)};
        if (k0 != A_NONE) {
#pragma unroll
            for (int v = 0; v < 4; v++) {
                xb[v] = dbar.f[v][off];
                dbar.f[v][off] = R(0);   // the sweep overwrote the destination here
            }
        }
        if (k0 == A_IN) {
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const R t = tbar.f[v][off];
                xb[v] += mx * t;
                tbar.f[v][off] = mt * t;
            }
        }
        R ncv, nct;
        {
            // matrix m: sub = A[p-1][p] (row p-1's c), diag, super = A[p+1][p] (row p+1's a)
            const RowABC<R> ev = entries(p, k0, 0), et = entries(p, k0, 1);
            const R subv = km == A_NONE ? R(0) : entries(p - 1, km, 0).c;
            const R subt = km == A_NONE ? R(0) : entries(p - 1, km, 1).c;
            const R supv = kp == A_NONE ? R(0) : entries(p + 1, kp, 0).a;
            const R supt = kp == A_NONE ? R(0) : entries(p + 1, kp, 1).a;
            const R denv = ev.b - subv * cpv, dent = et.b - subt * cpt;
            ncv = supv / denv;
            nct = supt / dent;
#pragma unroll
            for (int v = 0; v < 3; v++) dp[v] = (xb[v] - subv * dp[v]) / denv;
            dp[3] = (xb[3] - subt * dp[3]) / dent;
        }
        cpv = ncv;
        cpt = nct;
        R *s = scr + (long long)p * g.nlines;
        s[0 * qstride] = ncv;
        s[1 * qstride] = nct;
#pragma unroll
        for (int v = 0; v < 4; v++) s[(2 + v) * qstride] = dp[v];
        km = k0;
        k0 = kp;
    }

    // ---------------- pass 2: back substitution and accumulation ----------------
    R lam[4] = {R(0), R(0), R(0), R(0)};
    for (int p = hi; p >= lo; p--) {
        const long long off = base + (long long)p * sl;
        const R *s = scr + (long long)p * g.nlines;
        const R cv = s[0], ct = s[qstride];
#pragma unroll
        for (int v = 0; v < 3; v++) lam[v] = s[(2 + v) * qstride] - cv * lam[v];
        lam[3] = s[5 * qstride] - ct * lam[3];
        const int kd = kind_at(p);
        if (kd == A_NONE) continue;
        if (kd != A_IN) {
            const uint8_t c = d.code[off];
            const bool shared = kd == A_SHARED;
            const bool vf = !shared && (c & CODE_VEL_FREE) != 0, tf = !shared && (c & CODE_TEMP_FREE) != 0;
            if (!vf) {
#pragma unroll
                for (int v = 0; v < 3; v++) nvbar.f[v][off] += lam[v];
            }
            if (!tf) nvbar.f[3][off] += lam[3];
            continue;
        }
        // IN row
#pragma unroll
        for (int v = 0; v < 4; v++) sbar.f[v][off] += k.three_dt * lam[v];
        R wb = R(0);
#pragma unroll
        for (int v = 0; v < 4; v++) wb += lam[v] * (xs.f[v][off - sl] - xs.f[v][off + sl]);
        tbar.f[DIR][off] += wb * k.inv_two_h;
        const R pt = k.v_T * lam[DIR] * k.inv_two_h;
        tbar.f[3][off + sl] -= pt;
        tbar.f[3][off - sl] += pt;
        // DissFunc of the direction at this row, scaled by t_phi * lambda_T
        const R gl = k.t_phi * lam[3];
        const R *U = ti.f[0], *V = ti.f[1], *Wt = ti.f[2];
        const R ua = (U[off + sl] - U[off - sl]) * k.inv_two_h;
        const R va = (V[off + sl] - V[off - sl]) * k.inv_two_h;
        const R wa = (Wt[off + sl] - Wt[off - sl]) * k.inv_two_h;
        const R *Fd = ti.f[DIR];
        const R f1 = (Fd[off + so1] - Fd[off - so1]) * h1;   // advecting component along off-line axis 1
        const R f2 = (Fd[off + so2] - Fd[off - so2]) * h2;   // ... and axis 2
        R gu, gv, gw, g1, g2;
        if (DIR == 0) {        // 2 u_x^2 + v_x^2 + w_x^2 + v_x u_y + w_x u_z
            gu = R(4) * ua; gv = R(2) * va + f1; gw = R(2) * wa + f2; g1 = va; g2 = wa;
        } else if (DIR == 1) { // u_y^2 + 2 v_y^2 + w_y^2 + u_y v_x + w_y v_z
            gu = R(2) * ua + f1; gv = R(4) * va; gw = R(2) * wa + f2; g1 = ua; g2 = wa;
        } else {               // u_z^2 + v_z^2 + 2 w_z^2 + u_z w_x + v_z w_y
            gu = R(2) * ua + f1; gv = R(2) * va + f2; gw = R(4) * wa; g1 = ua; g2 = va;
        }
        const R s_h = gl * k.inv_two_h;
        tbar.f[0][off + sl] += gu * s_h;
        tbar.f[0][off - sl] -= gu * s_h;
        tbar.f[1][off + sl] += gv * s_h;
        tbar.f[1][off - sl] -= gv * s_h;
        tbar.f[2][off + sl] += gw * s_h;
        tbar.f[2][off - sl] -= gw * s_h;
        ga[off] = gl * g1;   // coefficient of d(advecting)/d(axis 1) at this cell
        gb[off] = gl * g2;
    }
}

// tbar[dir] += the off-line derivative terms: a cell's value f enters d_a f at
// its neighbours c - e_a (+1/(2h_a)) and c + e_a (-1/(2h_a)).
template <typename R, int DIR>
__global__ void adjoint_gather_kernel(DomainView<R> d, R *__restrict__ tb, const R *__restrict__ ga,
                                      const R *__restrict__ gb, SweepConst<R> k)
{
    const long long sx = (long long)d.ny * d.nz, sy = d.nz;
    const long long s1 = DIR == 0 ? sy : sx, s2 = DIR == 2 ? sy : 1;
    const R h1 = DIR == 0 ? k.inv_two_dy : k.inv_two_dx;
    const R h2 = DIR == 2 ? k.inv_two_dy : k.inv_two_dz;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < d.n;
         id += (long long)gridDim.x * blockDim.x) {
        const int kk = (int)(id % d.nz);
        const long long r = id / d.nz;
        const int j = (int)(r % d.ny), i = (int)(r / d.ny);
        // coordinates along off-line axes 1 and 2 and their extents
        const int c1 = DIR == 0 ? j : i, n1 = DIR == 0 ? d.ny : d.nx;
        const int c2 = DIR == 2 ? j : kk, n2 = DIR == 2 ? d.ny : d.nz;
        R acc = R(0);
        if (c1 > 0) acc += ga[id - s1] * h1;
        if (c1 + 1 < n1) acc -= ga[id + s1] * h1;
        if (c2 > 0) acc += gb[id - s2] * h2;
        if (c2 + 1 < n2) acc -= gb[id + s2] * h2;
        if (acc != R(0)) tb[id] += acc;
    }
}

// Adjoint of the step start and of UpdateBoundaries: temp = cur everywhere,
// next[B|V] = cur[B|V], cur[B|V] = node values.
template <typename R>
__global__ void adjoint_step_start_kernel(DomainView<R> d, Layer<R> cbar, Layer<R> nbar, Layer<R> tbar, Layer<R> nvbar)
{
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < d.n;
         id += (long long)gridDim.x * blockDim.x) {
        const bool bv = code_is_bv(d.code[id]);
        // every load of the cell first: the four layers are distinct arrays, but the
        // compiler cannot know that and would order each load after the last store
        R c[4], t[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            c[v] = cbar.f[v][id];
            t[v] = tbar.f[v][id];
        }
        if (bv) {
            R nb[4], nv[4];
#pragma unroll
            for (int v = 0; v < 4; v++) {
                nb[v] = nbar.f[v][id];
                nv[v] = nvbar.f[v][id];
            }
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const R x = c[v] + t[v] + nb[v];
                nbar.f[v][id] = R(0);
                nvbar.f[v][id] = nv[v] + x;
                cbar.f[v][id] = R(0);
            }
        } else {
#pragma unroll
            for (int v = 0; v < 4; v++) cbar.f[v][id] = c[v] + t[v];
        }
    }
}

// J = 1/2 sum over NODE_IN cells of the box of u^2 + v^2 + w^2 (per-block partial
// sums in double) and its gradient cbar = (u, v, w, 0) there, 0 elsewhere.
template <typename R>
__global__ void objective_kernel(DomainView<R> d, CLayer<R> x, int3 lo, int3 hi, Layer<R> cbar, double *psum)
{
    double acc = 0.0;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < d.n;
         id += (long long)gridDim.x * blockDim.x) {
        const int kk = (int)(id % d.nz);
        const long long r = id / d.nz;
        const int j = (int)(r % d.ny), i = (int)(r / d.ny);
        const bool in_box = i >= lo.x && i < hi.x && j >= lo.y && j < hi.y && kk >= lo.z && kk < hi.z &&
                            code_is_in(d.code[id]);
#pragma unroll
        for (int v = 0; v < 3; v++) {
            const R a = in_box ? x.f[v][id] : R(0);
            cbar.f[v][id] = a;
            acc += (double)a * (double)a;
        }
        cbar.f[3][id] = R(0);
    }
    __shared__ double sm[256];
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) psum[blockIdx.x] = sm[0];
}

__global__ void objective_final_kernel(const double *psum, int nblocks, double *out)
{
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 32) s += psum[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = 0.5 * s;
}

template <typename R>
cudaError_t launch_adjoint_sweep(int dir, const DomainView<R> &d, const int *lo, const int *hi, CLayer<R> ti,
                                 CLayer<R> xs, Layer<R> sbar, Layer<R> dbar, Layer<R> tbar, Layer<R> nvbar, R *ga, R *gb,
                                 R *scratch, const SweepConst<R> &k, int merges, int chunk_K, Layer<R> lam,
                                 cudaStream_t s)
{
    const LineGeom g = line_geom(dir, d.nx, d.ny, d.nz);
    {
        int NL = 0, P = 0;
        if (chunk_K < 0 && adjoint_chunk_supported(g.len, -chunk_K, (int)sizeof(R), NL, P))
            return launch_adjoint_chunk<R>(dir, -chunk_K, d, lo, hi, ti, xs, sbar, dbar, tbar, nvbar, ga, gb, k,
                                           merges, true, lam, s);
    }
    cudaError_t e = cudaMemsetAsync(ga, 0, sizeof(R) * d.n, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(gb, 0, sizeof(R) * d.n, s);
    if (e != cudaSuccess) return e;
    int NL = 0, P = 0;
    const bool chunked = chunk_K > 0 && adjoint_chunk_supported(g.len, chunk_K, (int)sizeof(R), NL, P);
    const int blocks = (g.nlines + 127) / 128;
    long long gb_ = (d.n + 255) / 256;
    const int gblocks = (int)(gb_ > 148 * 16 ? 148 * 16 : gb_);
#define AS(DD)                                                                                                   \
    if (dir == DD) {                                                                                             \
        if (chunked)                                                                                             \
            e = launch_adjoint_chunk<R>(DD, chunk_K, d, lo, hi, ti, xs, sbar, dbar, tbar, nvbar, ga, gb, k,       \
                                        merges, false, lam, s);                                                  \
        else {                                                                                                   \
            adjoint_sweep_kernel<R, DD><<<blocks, 128, 0, s>>>(d, g, lo, hi, ti, xs, sbar, dbar, tbar, nvbar, ga, \
                                                               gb, scratch, k, merges);                          \
            e = cudaGetLastError();                                                                              \
        }                                                                                                        \
        if (e != cudaSuccess) return e;                                                                          \
        adjoint_gather_kernel<R, DD><<<gblocks, 256, 0, s>>>(d, tbar.f[DD], ga, gb, k);                          \
        return cudaGetLastError();                                                                               \
    }
    AS(0) AS(1) AS(2)
#undef AS
    return cudaErrorInvalidValue;
}

template <typename R>
cudaError_t launch_adjoint_step_start(const DomainView<R> &d, Layer<R> cbar, Layer<R> nbar, Layer<R> tbar,
                                      Layer<R> nvbar, cudaStream_t s)
{
    long long b = (d.n + 255) / 256;
    const int blocks = (int)(b > 148 * 16 ? 148 * 16 : b);
    adjoint_step_start_kernel<R><<<blocks, 256, 0, s>>>(d, cbar, nbar, tbar, nvbar);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_objective(const DomainView<R> &d, CLayer<R> x, const int lo[3], const int hi[3], Layer<R> cbar,
                             double *psum, int nblocks, double *out, cudaStream_t s)
{
    objective_kernel<R><<<nblocks, 256, 0, s>>>(d, x, make_int3(lo[0], lo[1], lo[2]), make_int3(hi[0], hi[1], hi[2]),
                                                cbar, psum);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    objective_final_kernel<<<1, 32, 0, s>>>(psum, nblocks, out);
    return cudaGetLastError();
}

#define INST(R)                                                                                                     \
    template cudaError_t launch_adjoint_sweep<R>(int, const DomainView<R> &, const int *, const int *, CLayer<R>,   \
                                                 CLayer<R>, Layer<R>, Layer<R>, Layer<R>, Layer<R>, R *, R *, R *,  \
                                                 const SweepConst<R> &, int, int, Layer<R>, cudaStream_t);          \
    template cudaError_t launch_adjoint_step_start<R>(const DomainView<R> &, Layer<R>, Layer<R>, Layer<R>, Layer<R>, \
                                                      cudaStream_t);                                                \
    template cudaError_t launch_objective<R>(const DomainView<R> &, CLayer<R>, const int *, const int *, Layer<R>,  \
                                             double *, int, double *, cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace adi
