// Fast segmented tridiagonal sweep: lines cut into chunks, coefficients in registers.
//
// Same equations as the exact sweep (BuildMatrix / ApplyBC0 / ApplyBC1 rows of
// AdiSolver3D.cpp:732-852 on the block-diagonal line system, merge of
// TimeLayer3D.h:415-436), solved with a two-level partition method instead of one
// sequential Thomas pass per line:
//
//   1. Each thread owns K consecutive rows of one line (a chunk).  It loads the
//      rows' inputs in one burst and builds them.  A row is kept as its advection
//      term r = w/(2h) (IN rows) plus the four right-hand sides; the matrix
//      entries of both matrices (velocity, temperature) are derived from r and
//      the row kind when needed.  IN rows are solved in increment form,
//      x = cur + delta: substituting into a x[i-1] + b x[i] + c x[i+1] = cur*3/dt + S
//      with b = 3/dt + 2 vis, a = -r - vis, c = r - vis gives
//          a delta[i-1] + b delta[i] + c delta[i+1]
//              = S + vis (cm - 2 cur + cp) - r (cp - cm)
//      (cm, cp: cur at the IN neighbours, 0 at boundary rows, whose unknown is
//      x itself).  The 3/dt terms cancel exactly, so the float solve carries the
//      small increment instead of O(3/dt) right-hand sides.
//   2. The chunk's interior rows are eliminated so that each interior unknown is
//      expressed through the chunk's first and last unknowns:
//          x_i = d''_i - a''_i x_first - c''_i x_last.
//   3. The first/last rows of the P chunks of a line form a tridiagonal system of
//      2P unknowns.  One cyclic-reduction step (each thread removes the chunk-last
//      unknowns from its chunk-first row) leaves P rows, one per thread, which
//      parallel cyclic reduction solves in ceil(log2 P) steps; the chunk-last
//      unknowns follow from their own rows.  Rows are exchanged through shared
//      memory, one barrier per step, so every thread of the CTA works in every
//      phase.
//   4. Each thread recovers its interior unknowns, writes `next` for every
//      segment row and the merged nonlinear layer at IN rows.
//
// Rows outside segments are identity rows (a = c = 0, b = 1) and are never
// written; a segment's first row has a = 0 and its last row c = 0, so segments
// stay independent inside one line system.  The velocities share one matrix.
//
// Thread mapping (coalescing): for X and Y sweeps the NL lines of a CTA are the
// fastest thread index (neighbouring lines are neighbouring addresses); for Z
// sweeps, whose lines are contiguous, the chunks of one line are the fastest index
// and each thread reads its K rows with 16-byte vector loads.
//
// Rounding differs from the reference (increment form, reciprocal-multiply, fused
// multiply-add, partitioned elimination); the exact sweep is the bit-faithful one.
//
// Reciprocals: float uses the hardware approximation (rcp.approx) refined by one
// Newton-Raphson step r' = r + r (1 - x r); double uses IEEE division.  The chunk
// elimination, the cyclic-reduction step and the PCR updates are the shared ones
// of sweep_common.cuh (packed FP32 in float); the float write-back here is packed too.
#include "adi_internal.cuh"
#include "sweep_common.cuh"

#include <climits>

namespace adi {

namespace {

enum : int { K_NONE = 0, K_START = 1, K_IN = 2, K_END = 3, K_SHARED = 4 };

__device__ __forceinline__ int kind_of(uint8_t cm, uint8_t c0, uint8_t cp)
{
    if (code_is_in(c0)) return K_IN;
    bool inm = code_is_in(cm), inp = code_is_in(cp);
    if (inm && inp) return K_SHARED;
    if (inp) return K_START;
    if (inm) return K_END;
    return K_NONE;
}

template <typename R>
struct Vec4;
template <>
struct Vec4<float> {
    using T = float4;
};
template <>
struct Vec4<double> {
    using T = double2;  // 16 bytes
};

// Shared-memory slot of value q (0..7) of chunk c of CTA line li in one buffer;
// conflict-free for the thread mapping of each direction.
template <int DIR>
__device__ __forceinline__ int slot(int li, int c, int q, int NL, int P)
{
    if (DIR == 2) return (li * 8 + q) * P + c;
    return (c * 8 + q) * NL + li;
}

} // namespace

// One CTA's work: NL lines starting at line0, P chunks of K rows each, threads
// t < NL*P live.  Threads beyond NL*P (a batch item narrower than the block) keep
// every barrier but load and write nothing global and share one spare slot; each
// buffer holds buf_elems >= NL*P*8 (+ 8 when such threads exist) values.
template <typename R, int DIR, int K>
__device__ __forceinline__ void sweep_fast_block(unsigned char *smem_raw, int buf_elems, const DomainView<R> &d,
                                                 const LineGeom &g, int NL, int P, int line0,
                                                 const int *__restrict__ line_lo, const int *__restrict__ line_hi,
                                                 CLayer<R> cur, CLayer<R> tin, Layer<R> next, Layer<R> tout,
                                                 const SweepConst<R> &kc, int merges, int vec_ok)
{
    R *buf0 = reinterpret_cast<R *>(smem_raw);
    R *buf1 = buf0 + buf_elems;

    const int t = threadIdx.x;
    int li, ch;
    if (DIR == 2) { li = t / P; ch = t - li * P; }
    else { ch = t / NL; li = t - ch * NL; }
    const bool live = t < NL * P;
    // Shared-memory slot of value q of chunk c of line li.  A thread beyond NL*P
    // (batch items narrower than the block) uses one spare slot past the live ones:
    // it keeps the barriers but its values are never read by a live thread.
    auto slot_of = [&](int li_, int c_, int q_) { return live ? slot<DIR>(li_, c_, q_, NL, P) : NL * P * 8 + q_; };
    const int line = line0 + li;
    int lo = INT_MAX, hi = -1;
    long long base = 0;
    if (live && line < g.nlines) {
        const int a = line_lo[line];
        if (a >= 0) { lo = a; hi = line_hi[line]; }
        base = line_base(DIR, g, line);
    }
    const long long sl = g.stride;
    const long long sx = (long long)g.ny * g.nz, sy = g.nz;
    const long long so1 = DIR == 0 ? sy : sx;
    const long long so2 = DIR == 2 ? sy : 1;
    const int p0 = ch * K;
    const bool active = p0 <= hi && p0 + K - 1 >= lo;

    // ---------------- 1. load and build the chunk's rows ----------------
    // Every input of the rows -1..K that lie inside the line's segment range is
    // requested in one burst (no load waits on another), then the rows are built.
    int kind[K];
    unsigned freebits = 0;  // bit 2i: velocity BC FREE at row i, bit 2i+1: temperature
    R rr[K];                // advection term w/(2h) of IN rows
    R dv[4][K];             // right-hand sides (increment form at IN rows), later d''
    R tv[4][K + 2];         // temp at rows -1..K (stencils; own rows also for the merge)
    R cu[4][K + 2];         // cur at rows -1..K
    {
        uint8_t cc[K + 2];
        R g1v[K], g2v[K];
        const bool vec = DIR == 2 && vec_ok && (K % (16 / sizeof(R))) == 0 && active && p0 + K <= g.len;
#pragma unroll
        for (int q = 0; q < K + 2; q++) {
            const int p = p0 - 1 + q;
            const bool in_range = active && p >= lo && p <= hi;
            const long long off = base + (long long)p * sl;
            cc[q] = in_range ? __ldg(d.code + off) : uint8_t(NODE_OUT);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                tv[v][q] = R(0);
                cu[v][q] = R(0);
            }
            if (in_range && (!vec || q == 0 || q == K + 1)) {
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    tv[v][q] = __ldg(tin.f[v] + off);
                    cu[v][q] = __ldg(cur.f[v] + off);
                }
            }
            if (q >= 1 && q <= K) {
                // off-line neighbours of the advecting component; in bounds for every
                // row of a line that has segments (such lines are not on the frame)
                g1v[q - 1] = g2v[q - 1] = R(0);
                if (in_range) {
                    const R *Fd = tin.f[DIR];
                    g1v[q - 1] = __ldg(Fd + off + so1) - __ldg(Fd + off - so1);
                    g2v[q - 1] = __ldg(Fd + off + so2) - __ldg(Fd + off - so2);
                }
            }
        }
        if (vec) {
            using V = typename Vec4<R>::T;
            constexpr int W = 16 / sizeof(R);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const V *st = reinterpret_cast<const V *>(tin.f[v] + base + p0);
                const V *sc = reinterpret_cast<const V *>(cur.f[v] + base + p0);
#pragma unroll
                for (int q = 0; q < K / W; q++) {
                    V x = __ldg(st + q), y = __ldg(sc + q);
                    const R *xr = reinterpret_cast<const R *>(&x);
                    const R *yr = reinterpret_cast<const R *>(&y);
#pragma unroll
                    for (int e = 0; e < W; e++) {
                        tv[v][1 + q * W + e] = xr[e];
                        cu[v][1 + q * W + e] = yr[e];
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < K; i++) {
            kind[i] = kind_of(cc[i], cc[i + 1], cc[i + 2]);
            if (cc[i + 1] & CODE_VEL_FREE) freebits |= 1u << (2 * i);
            if (cc[i + 1] & CODE_TEMP_FREE) freebits |= 2u << (2 * i);
        }
        // reference vector of the increment form: cur at IN rows, 0 elsewhere
        bool inr[K + 2];
#pragma unroll
        for (int q = 0; q < K + 2; q++) inr[q] = code_is_in(cc[q]);
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int kd = kind[i];
            rr[i] = R(0);
            if (kd == K_IN) {
                const R r = tv[DIR][i + 1] * kc.inv_two_h;
                rr[i] = r;
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const R vis = v < 3 ? kc.vis_v : kc.vis_t;
                    const R cm = inr[i] ? cu[v][i] : R(0);
                    const R cp = inr[i + 2] ? cu[v][i + 2] : R(0);
                    dv[v][i] = vis * (cm - R(2) * cu[v][i + 1] + cp) - r * (cp - cm);
                }
                dv[DIR][i] -= kc.v_T * ((tv[3][i + 2] - tv[3][i]) * kc.inv_two_h);
                // DissFunc along the line (TimeLayer3D.h:554-588)
                const R fa = (tv[0][i + 2] - tv[0][i]) * kc.inv_two_h;
                const R fb = (tv[1][i + 2] - tv[1][i]) * kc.inv_two_h;
                const R fc = (tv[2][i + 2] - tv[2][i]) * kc.inv_two_h;
                const R g1 = g1v[i] * (DIR == 0 ? kc.inv_two_dy : kc.inv_two_dx);
                const R g2 = g2v[i] * (DIR == 2 ? kc.inv_two_dy : kc.inv_two_dz);
                R diss;
                if (DIR == 0) diss = R(2) * fa * fa + fb * fb + fc * fc + fb * g1 + fc * g2;
                else if (DIR == 1) diss = fa * fa + R(2) * fb * fb + fc * fc + fa * g1 + fc * g2;
                else diss = fa * fa + fb * fb + R(2) * fc * fc + fa * g1 + fb * g2;
                dv[3][i] += kc.t_phi * diss;
            } else if (kd == K_NONE) {
#pragma unroll
                for (int v = 0; v < 4; v++) dv[v][i] = R(0);
            } else {
                // boundary row, unknown x itself.  Dirichlet: x = node value.  BC_FREE
                // couples to the IN neighbour, whose unknown is cur + delta, so that
                // neighbour's cur moves to the right-hand side: start row 2x0 - x1 = 0
                // becomes 2x0 - delta1 = cur1, end row -x[n-2] + 2x[n-1] = 0 becomes
                // -delta[n-2] + 2x[n-1] = cur[n-2].
                const long long off = base + (long long)(p0 + i) * sl;
                const bool vf = (freebits >> (2 * i)) & 1u, tf = (freebits >> (2 * i + 1)) & 1u;
                const bool from_left = kd == K_END;   // IN neighbour at row i-1, else at i+1
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const bool fr = v < 3 ? vf : tf;
                    const R cn = from_left ? cu[v][i] : cu[v][i + 2];
                    dv[v][i] = fr ? cn : (kc.nv_in_temp ? tv[v][i + 1] : __ldg(d.nv[v] + off));
                }
            }
        }
    }

    // ---------------- 2. chunk elimination (shared with the X/Y/Z sweeps) ----------------
    // ea[m][i], ec[m][i] (interior rows 1..K-2) end as a'', c''; dv as d''.
    R ea[2][K], ec[2][K];
    sweep::Reduced<R> red;
    sweep::eliminate<R, K>(kind, rr, freebits, kc, dv, ea, ec, red);
    const R(&Al)[2] = red.Al;
    const R(&Cl)[2] = red.Cl;
    const R(&Dl)[4] = red.Dl;

    // ---------------- 3. reduced system of the line ----------------
    // (a) one cyclic-reduction step: remove x_last of chunks ch-1 and ch from the
    //     chunk-first row of chunk ch.
    buf0[slot_of(li, ch, 0)] = Al[0];
    buf0[slot_of(li, ch, 1)] = Cl[0];
    buf0[slot_of(li, ch, 2)] = Al[1];
    buf0[slot_of(li, ch, 3)] = Cl[1];
#pragma unroll
    for (int v = 0; v < 4; v++) buf0[slot_of(li, ch, 4 + v)] = Dl[v];
    __syncthreads();
    R ea_[2], ec_[2], ed[4];  // the chunk-first row after the reduction, normalised
    {
        R pv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (ch > 0) {
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = buf0[slot_of(li, ch - 1, q)];
        }
        sweep::cr_step<R>(red, pv, ea_, ec_, ed);
    }
    // (b) parallel cyclic reduction over the P chunk-first unknowns.  Step n
    //     writes buffer (n odd ? buf1 : buf0); the barrier of step n+1 (or of
    //     stage (c)) orders step n's reads before the buffer is written again.
    //     A partner outside the line contributes zeros.
    int nstep = 0;
    for (int s = 1; s < P; s <<= 1, nstep++) {
        R *bw = (nstep & 1) ? buf0 : buf1;
        bw[slot_of(li, ch, 0)] = ea_[0];
        bw[slot_of(li, ch, 1)] = ec_[0];
        bw[slot_of(li, ch, 2)] = ea_[1];
        bw[slot_of(li, ch, 3)] = ec_[1];
#pragma unroll
        for (int v = 0; v < 4; v++) bw[slot_of(li, ch, 4 + v)] = ed[v];
        __syncthreads();
        R mv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        R pv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (ch - s >= 0) {
#pragma unroll
            for (int q = 0; q < 8; q++) mv[q] = bw[slot_of(li, ch - s, q)];
        }
        if (ch + s < P) {
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = bw[slot_of(li, ch + s, q)];
        }
        sweep::pcr_update<R>(mv, pv, ea_, ec_, ed);
    }
    // (c) x_first of this chunk is ed; x_last from its own row and x_first(ch+1)
    R *bx = (nstep & 1) ? buf0 : buf1;
#pragma unroll
    for (int v = 0; v < 4; v++) bx[slot_of(li, ch, v)] = ed[v];
    __syncthreads();
    R xf[4], xl[4];
    {
        R nf[4] = {R(0), R(0), R(0), R(0)};
        if (ch + 1 < P) {
#pragma unroll
            for (int v = 0; v < 4; v++) nf[v] = bx[slot_of(li, ch + 1, v)];
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            xf[v] = ed[v];
            const int m = v < 3 ? 0 : 1;
            xl[v] = Dl[v] - Al[m] * xf[v] - Cl[m] * nf[v];
        }
    }
    if (!active) return;

    // ---------------- 4. interior unknowns, write-back, merge ----------------
    // merged nonlinear value: (temp + x) / 2, or with the extra merge (temp + 3 x) / 4
    const R gw_new = merges == 2 ? R(0.75) : R(0.5), gw_old = R(1) - gw_new;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int kd = kind[i];
        if (kd == K_NONE) continue;
        R x[4];
        if (i == 0) {
#pragma unroll
            for (int v = 0; v < 4; v++) x[v] = xf[v];
        } else if (i == K - 1) {
#pragma unroll
            for (int v = 0; v < 4; v++) x[v] = xl[v];
        } else if constexpr (sizeof(R) == 4) {
            // packed FP32: (U, T) and (V, W) two at a time
            using namespace sweep;
            const float2 nea = p2(-ea[0][i], -ea[1][i]), nec = p2(-ec[0][i], -ec[1][i]);
            const float2 x03 = fma2(nec, p2(xl[0], xl[3]), fma2(nea, p2(xf[0], xf[3]), p2(dv[0][i], dv[3][i])));
            const float2 x12 =
                fma2(bc2(nec.x), p2(xl[1], xl[2]), fma2(bc2(nea.x), p2(xf[1], xf[2]), p2(dv[1][i], dv[2][i])));
            x[0] = x03.x; x[3] = x03.y; x[1] = x12.x; x[2] = x12.y;
        } else {
#pragma unroll
            for (int v = 0; v < 3; v++) x[v] = dv[v][i] - ea[0][i] * xf[v] - ec[0][i] * xl[v];
            x[3] = dv[3][i] - ea[1][i] * xf[3] - ec[1][i] * xl[3];
        }
        const long long off = base + (long long)(p0 + i) * sl;
        if (kd == K_IN) {
            if constexpr (sizeof(R) == 4) {
                using namespace sweep;
                const float2 x03 = add2(p2(cu[0][i + 1], cu[3][i + 1]), p2(x[0], x[3]));
                const float2 x12 = add2(p2(cu[1][i + 1], cu[2][i + 1]), p2(x[1], x[2]));
                const float2 m03 = fma2(x03, bc2(gw_new), mul2(p2(tv[0][i + 1], tv[3][i + 1]), bc2(gw_old)));
                const float2 m12 = fma2(x12, bc2(gw_new), mul2(p2(tv[1][i + 1], tv[2][i + 1]), bc2(gw_old)));
                next.f[0][off] = x03.x; next.f[3][off] = x03.y; next.f[1][off] = x12.x; next.f[2][off] = x12.y;
                tout.f[0][off] = m03.x; tout.f[3][off] = m03.y; tout.f[1][off] = m12.x; tout.f[2][off] = m12.y;
            } else {
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const R xv = cu[v][i + 1] + x[v];
                    next.f[v][off] = xv;
                    tout.f[v][off] = fma(xv, gw_new, tv[v][i + 1] * gw_old);
                }
            }
        } else {
#pragma unroll
            for (int v = 0; v < 4; v++) next.f[v][off] = x[v];
        }
    }
}

template <typename R, int DIR, int K>
__global__ void __launch_bounds__(256)
    sweep_fast_kernel(DomainView<R> d, LineGeom g, int NL, int P, const int *__restrict__ line_lo,
                      const int *__restrict__ line_hi, CLayer<R> cur, CLayer<R> tin, Layer<R> next, Layer<R> tout,
                      SweepConst<R> kc, int merges, int vec_ok)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    sweep_fast_block<R, DIR, K>(smem_raw, NL * P * 8, d, g, NL, P, blockIdx.x * NL, line_lo, line_hi, cur, tin,
                                next, tout, kc, merges, vec_ok);
}

// Many domains in one persistent launch: CTA b takes items b, b + gridDim.x, ...
// of the direction's work list (domain, first line); every item runs with the
// domain's own geometry, constants and lines-per-CTA.  Layer roles are indices
// into each domain's five layers, the same for every domain of the batch.
template <typename R, int DIR, int K>
__global__ void __launch_bounds__(256, K == 4 ? 2 : 1)
    sweep_fast_batch_kernel(const BatchDomain<R> *__restrict__ doms, const int2 *__restrict__ items, int nitems,
                            int src, int tin, int dst, int tout, int merges)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const BatchDomain<R> &bd = doms[w.x];
        const DomainView<R> d = bd.d;
        const LineGeom g = line_geom(DIR, d.nx, d.ny, d.nz);
        CLayer<R> c, ti;
        Layer<R> nx, to;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            c.f[v] = bd.L[src][v];
            ti.f[v] = bd.L[tin][v];
            nx.f[v] = bd.L[dst][v];
            to.f[v] = bd.L[tout][v];
        }
        sweep_fast_block<R, DIR, K>(smem_raw, blockDim.x * 8, d, g, bd.NL[DIR], bd.P[DIR], w.y, bd.lo[DIR], bd.hi[DIR],
                                    c, ti, nx, to, bd.kc[DIR], merges, bd.vec_ok);
        __syncthreads();   // the shared buffers are reused by the next item
    }
}

template <typename R>
cudaError_t launch_sweep_fast_batch(int dir, int K, const BatchDomain<R> *doms, const int2 *items, int nitems,
                                    int grid, int src, int tin, int dst, int tout, int merges, cudaStream_t s)
{
    if (nitems == 0) return cudaSuccess;
    const size_t smem = (size_t)2 * 256 * 8 * sizeof(R);
#define FB(DD, KK)                                                                                                 \
    if (dir == DD && K == KK) {                                                                                    \
        sweep_fast_batch_kernel<R, DD, KK><<<grid, 256, smem, s>>>(doms, items, nitems, src, tin, dst, tout, merges); \
        return cudaGetLastError();                                                                                 \
    }
    FB(0, 4) FB(0, 8) FB(1, 4) FB(1, 8) FB(2, 4) FB(2, 8)
#undef FB
    return cudaErrorInvalidConfiguration;
}

template cudaError_t launch_sweep_fast_batch<float>(int, int, const BatchDomain<float> *, const int2 *, int, int, int,
                                                    int, int, int, int, cudaStream_t);
template cudaError_t launch_sweep_fast_batch<double>(int, int, const BatchDomain<double> *, const int2 *, int, int,
                                                     int, int, int, int, int, cudaStream_t);

bool fast_shape_supported(int dir, FastShape s, int len, int elem_bytes)
{
    if (s.mode != 0) return false;
    if (s.K != 4 && s.K != 8 && s.K != 12 && s.K != 16) return false;
    if (s.NL < 1 || s.P < 1 || (long long)s.P * s.K < len) return false;
    const int threads = s.NL * s.P;
    if (threads > 256 || threads < 32) return false;
    const size_t smem = (size_t)2 * s.NL * s.P * 8 * elem_bytes;
    if (smem > 48 * 1024) return false;
    (void)dir;
    return true;
}

template <typename R, int DIR, int K>
static cudaError_t launch_k(const DomainView<R> &d, const LineGeom &g, const int *lo, const int *hi, CLayer<R> cur,
                            CLayer<R> tin, Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges,
                            FastShape s, cudaStream_t st)
{
    const int threads = s.NL * s.P;
    const int blocks = (g.nlines + s.NL - 1) / s.NL;
    const size_t smem = (size_t)2 * s.NL * s.P * 8 * sizeof(R);
    int vec_ok = 0;
    if (DIR == 2) {
        const size_t W = 16 / sizeof(R);
        bool al = (g.nz % W) == 0;
        for (int v = 0; v < 4 && al; v++)
            al = ((uintptr_t)cur.f[v] % 16) == 0 && ((uintptr_t)tin.f[v] % 16) == 0;
        vec_ok = al ? 1 : 0;
    }
    sweep_fast_kernel<R, DIR, K><<<blocks, threads, smem, st>>>(d, g, s.NL, s.P, lo, hi, cur, tin, next, tout, k,
                                                               merges, vec_ok);
    return cudaGetLastError();
}

template <typename R, int DIR>
static cudaError_t launch_dir(const DomainView<R> &d, const int *lo, const int *hi, CLayer<R> cur, CLayer<R> tin,
                              Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges, FastShape s,
                              cudaStream_t st)
{
    const LineGeom g = line_geom(DIR, d.nx, d.ny, d.nz);
    switch (s.K) {
    case 4: return launch_k<R, DIR, 4>(d, g, lo, hi, cur, tin, next, tout, k, merges, s, st);
    case 8: return launch_k<R, DIR, 8>(d, g, lo, hi, cur, tin, next, tout, k, merges, s, st);
    case 12: return launch_k<R, DIR, 12>(d, g, lo, hi, cur, tin, next, tout, k, merges, s, st);
    case 16: return launch_k<R, DIR, 16>(d, g, lo, hi, cur, tin, next, tout, k, merges, s, st);
    default: return cudaErrorInvalidValue;
    }
}

template <typename R>
cudaError_t launch_sweep_fast(int dir, const DomainView<R> &d, const int *line_lo, const int *line_hi,
                              CLayer<R> cur, CLayer<R> temp_in, Layer<R> next, Layer<R> temp_out,
                              const SweepConst<R> &k, int merges, FastShape shape, cudaStream_t s)
{
    const LineGeom g = line_geom(dir, d.nx, d.ny, d.nz);
    if (!fast_shape_supported(dir, shape, g.len, (int)sizeof(R))) return cudaErrorInvalidConfiguration;
    if (dir == 0) return launch_dir<R, 0>(d, line_lo, line_hi, cur, temp_in, next, temp_out, k, merges, shape, s);
    if (dir == 1) return launch_dir<R, 1>(d, line_lo, line_hi, cur, temp_in, next, temp_out, k, merges, shape, s);
    return launch_dir<R, 2>(d, line_lo, line_hi, cur, temp_in, next, temp_out, k, merges, shape, s);
}

template cudaError_t launch_sweep_fast<float>(int, const DomainView<float> &, const int *, const int *,
                                              CLayer<float>, CLayer<float>, Layer<float>, Layer<float>,
                                              const SweepConst<float> &, int, FastShape, cudaStream_t);
template cudaError_t launch_sweep_fast<double>(int, const DomainView<double> &, const int *, const int *,
                                               CLayer<double>, CLayer<double>, Layer<double>, Layer<double>,
                                               const SweepConst<double> &, int, FastShape, cudaStream_t);

} // namespace adi
