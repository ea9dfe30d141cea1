// Chunked adjoint sweep: the transposed tridiagonal solve of adjoint.cu with the
// parallel structure of the fast forward sweep (sweep_fast.cu).
//
// Each thread owns K consecutive rows of one line.  It builds its rows of A^T
// (sub-diagonal: row p-1's c, diagonal: row p's b, super-diagonal: row p+1's a,
// for the velocity and the temperature matrix) and the right-hand sides xbar (the
// destination's adjoint on segment rows plus the merge's share of the temp
// adjoint), eliminates its interior rows (eliminate_abc), and the chunk-first /
// chunk-last unknowns of the line's P chunks are solved by one cyclic-reduction
// step and parallel cyclic reduction through shared memory, as in the forward.
// The accumulations then happen per owned row; the contributions a row makes to
// its neighbours p-1 and p+1 (pressure term, along-line dissipation terms) stay
// in the thread or cross one chunk boundary through shared memory, so every
// cell of tbar has one writer.  Off-line dissipation terms go through the two
// planes that adjoint_gather_kernel (adjoint.cu) folds in afterwards.
#include "adi_internal.cuh"
#include "sweep_common.cuh"

#include <climits>

namespace adi {

namespace {

enum : int { Q_NONE = 0, Q_START = 1, Q_IN = 2, Q_END = 3, Q_SHARED = 4 };

__device__ __forceinline__ int qkind(bool inm, bool in0, bool inp)
{
    if (in0) return Q_IN;
    if (inm && inp) return Q_SHARED;
    if (inp) return Q_START;
    if (inm) return Q_END;
    return Q_NONE;
}

// Entries (a, b, c) of forward row p for matrix m from its kind, BC code and
// advection term r.
template <typename R>
__device__ __forceinline__ void fwd_entries(int kind, uint8_t code, int m, R r, const SweepConst<R> &k, R &a, R &b,
                                            R &c)
{
    const R vis = m == 0 ? k.vis_v : k.vis_t;
    const bool fr = m == 0 ? (code & CODE_VEL_FREE) != 0 : (code & CODE_TEMP_FREE) != 0;
    if (kind == Q_IN) {
        a = -r - vis;
        b = m == 0 ? k.b_v : k.b_t;
        c = r - vis;
    } else if (kind == Q_START) {
        a = R(0);
        b = fr ? R(2) : R(1);
        c = fr ? R(-1) : R(0);
    } else if (kind == Q_END) {
        a = fr ? R(-1) : R(0);
        b = fr ? R(2) : R(1);
        c = R(0);
    } else {   // SHARED (Dirichlet by the solver contract) and NONE
        a = R(0);
        b = R(1);
        c = R(0);
    }
}

template <typename R>
CLayer<R> clayer_view(const Layer<R> &x)
{
    CLayer<R> c;
    for (int v = 0; v < 4; v++) c.f[v] = x.f[v];
    return c;
}

template <int DIR>
__device__ __forceinline__ int aslot(int li, int c, int q, int NL, int P)
{
    if (DIR == 2) return (li * 8 + q) * P + c;
    return (c * 8 + q) * NL + li;
}

} // namespace

// SPLIT: the solve only.  The kernel stores the line's adjoint solution lambda
// (lamo, four fields, at every row that is not NONE), consumes dbar and
// accumulates nvbar on the boundary rows, and leaves the IN rows' accumulations
// to adjoint_accum_kernel, which runs over the cells with full occupancy.
template <typename R, int DIR, int K, bool SPLIT>
__global__ void __launch_bounds__(256, SPLIT ? 4 : 2)
    adjoint_chunk_kernel(DomainView<R> d, LineGeom g, int NL, int P, const int *__restrict__ line_lo,
                         const int *__restrict__ line_hi, CLayer<R> ti, CLayer<R> xs, Layer<R> sbar, Layer<R> dbar,
                         Layer<R> tbar, Layer<R> nvbar, R *__restrict__ ga, R *__restrict__ gb, SweepConst<R> kc,
                         int merges, Layer<R> lamo)
{
    using namespace sweep;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *buf0 = reinterpret_cast<R *>(smem_raw);
    R *buf1 = buf0 + (size_t)NL * P * 8;
    const int t = threadIdx.x;
    int li, ch;
    if (DIR == 2) { li = t / P; ch = t - li * P; }
    else { ch = t / NL; li = t - ch * NL; }
    const int line = blockIdx.x * NL + li;
    int lo = INT_MAX, hi = -1;
    long long base = 0;
    if (line < g.nlines) {
        const int a = line_lo[line];
        if (a >= 0) { lo = a; hi = line_hi[line]; }
        base = line_base(DIR, g, line);
    }
    const long long sl = g.stride;
    const long long sx = (long long)g.ny * g.nz, sy = g.nz;
    const long long so1 = DIR == 0 ? sy : sx;
    const long long so2 = DIR == 2 ? sy : 1;
    const R h1 = DIR == 0 ? kc.inv_two_dy : kc.inv_two_dx;
    const R h2 = DIR == 2 ? kc.inv_two_dy : kc.inv_two_dz;
    const int p0 = ch * K;
    const bool active = p0 <= hi && p0 + K - 1 >= lo;
    const R mx = merges == 2 ? R(0.75) : R(0.5);
    const R mt = merges == 2 ? R(0.25) : R(0.5);

    // ---------------- rows: kinds, window values, A^T and xbar ----------------
    // All first-phase loads go out together: codes, the advecting field and the
    // destination / temp adjoints of every row inside the line's segment range
    // (addresses valid there); the row kinds then mask what a row does not use.
    uint8_t cc[K + 4];   // codes of rows p0-2 .. p0+K+1 (OUT outside the segment range)
#pragma unroll
    for (int q = 0; q < K + 4; q++) {
        const int p = p0 - 2 + q;
        cc[q] = (active && p >= lo && p <= hi) ? d.code[base + (long long)p * sl] : uint8_t(NODE_OUT);
    }
    R wv[K + 2];     // advecting temp at window rows
#pragma unroll
    for (int q = 0; q < K + 2; q++) {
        const int p = p0 - 1 + q;
        wv[q] = (active && p >= lo && p <= hi) ? ti.f[DIR][base + (long long)p * sl] : R(0);
    }
    R dbr[4][K], tbr[4][K];   // destination and temp adjoints at the owned rows
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int p = p0 + i;
        const bool ok = active && p >= lo && p <= hi;
        const long long off = base + (long long)p * sl;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            dbr[v][i] = ok ? dbar.f[v][off] : R(0);
            tbr[v][i] = ok ? tbar.f[v][off] : R(0);
        }
    }
    int kd[K + 2];   // kinds of rows p0-1 .. p0+K
#pragma unroll
    for (int q = 0; q < K + 2; q++) kd[q] = qkind(code_is_in(cc[q]), code_is_in(cc[q + 1]), code_is_in(cc[q + 2]));
#pragma unroll
    for (int q = 0; q < K + 2; q++) wv[q] = kd[q] == Q_IN ? wv[q] : R(0);
    R A[2][K], B[2][K], C[2][K], xb[4][K];
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int q = i + 1;
        const long long off = base + (long long)(p0 + i) * sl;
#pragma unroll
        for (int m = 0; m < 2; m++) {
            R a0, b0, c0, am, bm, cm, ap, bp, cp;
            fwd_entries<R>(kd[q], cc[q + 1], m, wv[q] * kc.inv_two_h, kc, a0, b0, c0);
            fwd_entries<R>(kd[q - 1], cc[q], m, wv[q - 1] * kc.inv_two_h, kc, am, bm, cm);
            fwd_entries<R>(kd[q + 1], cc[q + 2], m, wv[q + 1] * kc.inv_two_h, kc, ap, bp, cp);
            A[m][i] = cm;   // A^T[p][p-1] = A[p-1][p]
            B[m][i] = b0;
            C[m][i] = ap;   // A^T[p][p+1] = A[p+1][p]
            (void)a0; (void)c0; (void)bm; (void)am; (void)bp; (void)cp;
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const R db = kd[q] != Q_NONE ? dbr[v][i] : R(0);
            const R to = kd[q] == Q_IN ? tbr[v][i] : R(0);
            xb[v][i] = db + mx * to;
        }
        (void)off;
    }

    // ---------------- chunk elimination of A^T ----------------
    R ea[2][K], ec[2][K];
    Reduced<R> red;
    eliminate_abc<R, K>(A, B, C, xb, ea, ec, red);

    // ---------------- reduced system: one CR step + PCR ----------------
    R lf[4], ll[4];
    int nstep = 0;
    // Split kernel, P a power of two up to 32: each line's chunks as one P-lane
    // segment of a warp, CR and PCR in shuffles (couplings to rows outside the line
    // are exactly zero, so a lane whose partner lies outside takes its own row:
    // finite values times 0).  Z lines already sit that way (lane = chunk); X and Y
    // lines, one chunk per line across the lanes, go through shared memory once.
    const bool warp_pcr = SPLIT && P <= 32 && (P & (P - 1)) == 0;
    if (warp_pcr) {
        auto shuffled = [&](const Reduced<R> &wr, int wc, R (&xo)[8]) {
            auto up = [&](R x, int dd) { return __shfl_up_sync(0xffffffffu, x, dd, P); };
            auto dn = [&](R x, int dd) { return __shfl_down_sync(0xffffffffu, x, dd, P); };
            R ea_[2], ec_[2], ed[4];
            {
                R pv[8] = {up(wr.Al[0], 1), up(wr.Cl[0], 1), up(wr.Al[1], 1), up(wr.Cl[1], 1),
                           up(wr.Dl[0], 1), up(wr.Dl[1], 1), up(wr.Dl[2], 1), up(wr.Dl[3], 1)};
                if (wc == 0) {
#pragma unroll
                    for (int q = 0; q < 8; q++) pv[q] = R(0);
                }
                cr_step<R>(wr, pv, ea_, ec_, ed);
            }
            for (int st = 1; st < P; st <<= 1) {
                const R mv[8] = {up(ea_[0], st), up(ec_[0], st), up(ea_[1], st), up(ec_[1], st),
                                 up(ed[0], st),  up(ed[1], st),  up(ed[2], st),  up(ed[3], st)};
                const R pv[8] = {dn(ea_[0], st), dn(ec_[0], st), dn(ea_[1], st), dn(ec_[1], st),
                                 dn(ed[0], st),  dn(ed[1], st),  dn(ed[2], st),  dn(ed[3], st)};
                pcr_update<R>(mv, pv, ea_, ec_, ed);
            }
#pragma unroll
            for (int v = 0; v < 4; v++) {
                R nf = dn(ed[v], 1);
                if (wc == P - 1) nf = R(0);
                const int m = v < 3 ? 0 : 1;
                xo[v] = ed[v];
                xo[4 + v] = wr.Dl[v] - wr.Al[m] * ed[v] - wr.Cl[m] * nf;   // Cl = 0 on the last chunk
            }
        };
        R xo[8];
        if (DIR == 2) {
            shuffled(red, ch, xo);
        } else {
            // 16 planes of NL (P + 1) values: a thread's reduced rows at (li, ch), read
            // back by the warp lane (t / P, t % P) that owns that line's chunk
            const int NQ = NL * (P + 1);
            const int slot = li * (P + 1) + ch;
            const R rv[16] = {red.Af[0], red.Af[1], red.Cf[0], red.Cf[1], red.Al[0], red.Al[1], red.Cl[0], red.Cl[1],
                              red.Df[0], red.Df[1], red.Df[2], red.Df[3], red.Dl[0], red.Dl[1], red.Dl[2], red.Dl[3]};
#pragma unroll
            for (int q = 0; q < 16; q++) buf0[q * NQ + slot] = rv[q];
            __syncthreads();
            const int wl = t / P, wc = t - (t / P) * P;
            const int wslot = wl * (P + 1) + wc;
            Reduced<R> wr;
#pragma unroll
            for (int m = 0; m < 2; m++) {
                wr.Af[m] = buf0[m * NQ + wslot];
                wr.Cf[m] = buf0[(2 + m) * NQ + wslot];
                wr.Al[m] = buf0[(4 + m) * NQ + wslot];
                wr.Cl[m] = buf0[(6 + m) * NQ + wslot];
            }
#pragma unroll
            for (int v = 0; v < 4; v++) {
                wr.Df[v] = buf0[(8 + v) * NQ + wslot];
                wr.Dl[v] = buf0[(12 + v) * NQ + wslot];
            }
            R wx[8];
            shuffled(wr, wc, wx);
            __syncthreads();   // every plane read is done
#pragma unroll
            for (int q = 0; q < 8; q++) buf0[q * NQ + wslot] = wx[q];
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 8; q++) xo[q] = buf0[q * NQ + slot];
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            lf[v] = xo[v];
            ll[v] = xo[4 + v];
        }
    } else {
    buf0[aslot<DIR>(li, ch, 0, NL, P)] = red.Al[0];
    buf0[aslot<DIR>(li, ch, 1, NL, P)] = red.Cl[0];
    buf0[aslot<DIR>(li, ch, 2, NL, P)] = red.Al[1];
    buf0[aslot<DIR>(li, ch, 3, NL, P)] = red.Cl[1];
#pragma unroll
    for (int v = 0; v < 4; v++) buf0[aslot<DIR>(li, ch, 4 + v, NL, P)] = red.Dl[v];
    __syncthreads();
    R ea_[2], ec_[2], ed[4];
    {
        R pv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (ch > 0) {
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = buf0[aslot<DIR>(li, ch - 1, q, NL, P)];
        }
        cr_step<R>(red, pv, ea_, ec_, ed);
    }
    for (int s = 1; s < P; s <<= 1, nstep++) {
        R *bw = (nstep & 1) ? buf0 : buf1;
        bw[aslot<DIR>(li, ch, 0, NL, P)] = ea_[0];
        bw[aslot<DIR>(li, ch, 1, NL, P)] = ec_[0];
        bw[aslot<DIR>(li, ch, 2, NL, P)] = ea_[1];
        bw[aslot<DIR>(li, ch, 3, NL, P)] = ec_[1];
#pragma unroll
        for (int v = 0; v < 4; v++) bw[aslot<DIR>(li, ch, 4 + v, NL, P)] = ed[v];
        __syncthreads();
        R mv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        R pv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (ch - s >= 0) {
#pragma unroll
            for (int q = 0; q < 8; q++) mv[q] = bw[aslot<DIR>(li, ch - s, q, NL, P)];
        }
        if (ch + s < P) {
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = bw[aslot<DIR>(li, ch + s, q, NL, P)];
        }
        pcr_update<R>(mv, pv, ea_, ec_, ed);
    }
    R *bx = (nstep & 1) ? buf0 : buf1;
#pragma unroll
    for (int v = 0; v < 4; v++) bx[aslot<DIR>(li, ch, v, NL, P)] = ed[v];
    __syncthreads();
    {
        R nf[4] = {R(0), R(0), R(0), R(0)};
        if (ch + 1 < P) {
#pragma unroll
            for (int v = 0; v < 4; v++) nf[v] = bx[aslot<DIR>(li, ch + 1, v, NL, P)];
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int m = v < 3 ? 0 : 1;
            lf[v] = ed[v];
            ll[v] = red.Dl[v] - red.Al[m] * lf[v] - red.Cl[m] * nf[v];
        }
    }
    }   // shared-memory PCR

    // ---------------- accumulations per owned row ----------------
    R up[4][K], dn[4][K];   // contributions of row i to rows p+1 (up) and p-1 (dn): u, v, w, T
    R wb[K];
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int q = i + 1;
        const long long off = base + (long long)(p0 + i) * sl;
        R lam[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int m = v < 3 ? 0 : 1;
            lam[v] = i == 0 ? lf[v] : (i == K - 1 ? ll[v] : xb[v][i] - ea[m][i] * lf[v] - ec[m][i] * ll[v]);
        }
#pragma unroll
        for (int v = 0; v < 4; v++) { up[v][i] = R(0); dn[v][i] = R(0); }
        wb[i] = R(0);
        if (!active || kd[q] == Q_NONE) continue;
#pragma unroll
        for (int v = 0; v < 4; v++) dbar.f[v][off] = R(0);   // the sweep overwrote the destination here
        if constexpr (SPLIT) {
#pragma unroll
            for (int v = 0; v < 4; v++) lamo.f[v][off] = lam[v];
        }
        if (kd[q] != Q_IN) {
            const uint8_t c = cc[q + 1];
            const bool shared = kd[q] == Q_SHARED;
            const bool vf = !shared && (c & CODE_VEL_FREE) != 0, tf = !shared && (c & CODE_TEMP_FREE) != 0;
            if (!vf) {
#pragma unroll
                for (int v = 0; v < 3; v++) nvbar.f[v][off] += lam[v];
            }
            if (!tf) nvbar.f[3][off] += lam[3];
            continue;
        }
        if constexpr (!SPLIT) {
#pragma unroll
        for (int v = 0; v < 4; v++) sbar.f[v][off] += kc.three_dt * lam[v];
        R w = R(0);
#pragma unroll
        for (int v = 0; v < 4; v++) w += lam[v] * (xs.f[v][off - sl] - xs.f[v][off + sl]);
        wb[i] = w * kc.inv_two_h;
        const R pt = kc.v_T * lam[DIR] * kc.inv_two_h;
        up[3][i] = -pt;
        dn[3][i] = pt;
        const R gl = kc.t_phi * lam[3];
        const R *U = ti.f[0], *V = ti.f[1], *Wt = ti.f[2];
        const R ua = (U[off + sl] - U[off - sl]) * kc.inv_two_h;
        const R va = (V[off + sl] - V[off - sl]) * kc.inv_two_h;
        const R wa = (Wt[off + sl] - Wt[off - sl]) * kc.inv_two_h;
        const R *Fd = ti.f[DIR];
        const R f1 = (Fd[off + so1] - Fd[off - so1]) * h1;
        const R f2 = (Fd[off + so2] - Fd[off - so2]) * h2;
        R gu, gv, gw, g1, g2;
        if (DIR == 0) {
            gu = R(4) * ua; gv = R(2) * va + f1; gw = R(2) * wa + f2; g1 = va; g2 = wa;
        } else if (DIR == 1) {
            gu = R(2) * ua + f1; gv = R(4) * va; gw = R(2) * wa + f2; g1 = ua; g2 = wa;
        } else {
            gu = R(2) * ua + f1; gv = R(2) * va + f2; gw = R(4) * wa; g1 = ua; g2 = va;
        }
        const R s_h = gl * kc.inv_two_h;
        up[0][i] = gu * s_h; dn[0][i] = -gu * s_h;
        up[1][i] = gv * s_h; dn[1][i] = -gv * s_h;
        up[2][i] = gw * s_h; dn[2][i] = -gw * s_h;
        ga[off] = gl * g1;
        gb[off] = gl * g2;
        }   // !SPLIT
    }
    if constexpr (!SPLIT) {
    // chunk-boundary neighbours: the previous chunk's last row sends up, the next
    // chunk's first row sends down
    R *bz = (nstep & 1) ? buf1 : buf0;   // not bx: stage (c) may still be reading it
#pragma unroll
    for (int v = 0; v < 4; v++) {
        bz[aslot<DIR>(li, ch, v, NL, P)] = up[v][K - 1];
        bz[aslot<DIR>(li, ch, 4 + v, NL, P)] = dn[v][0];
    }
    __syncthreads();
    if (!active) return;
    R upp[4] = {R(0), R(0), R(0), R(0)}, dnn[4] = {R(0), R(0), R(0), R(0)};
    if (ch > 0) {
#pragma unroll
        for (int v = 0; v < 4; v++) upp[v] = bz[aslot<DIR>(li, ch - 1, v, NL, P)];
    }
    if (ch + 1 < P) {
#pragma unroll
        for (int v = 0; v < 4; v++) dnn[v] = bz[aslot<DIR>(li, ch + 1, 4 + v, NL, P)];
    }
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int q = i + 1;
        if (kd[q] == Q_NONE) continue;
        const long long off = base + (long long)(p0 + i) * sl;
        const bool in = kd[q] == Q_IN;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            R x = (in ? mt : R(1)) * tbr[v][i];   // loaded at the start: this thread owns the row
            if (v == DIR) x += wb[i];
            x += i > 0 ? up[v][i - 1] : upp[v];
            x += i < K - 1 ? dn[v][i + 1] : dnn[v];
            tbar.f[v][off] = x;
        }
    }
    }   // !SPLIT
}

// Dynamic shared memory of adjoint_chunk_kernel: the two PCR buffers of 8 values
// per chunk, or the split kernel's 16 planes of NL (P + 1) reduced-row values.
size_t adjoint_chunk_smem(int NL, int P, int elem_bytes)
{
    const size_t pcr = (size_t)2 * NL * P * 8 * elem_bytes, planes = (size_t)16 * NL * (P + 1) * elem_bytes;
    return pcr > planes ? pcr : planes;
}

bool adjoint_chunk_supported(int len, int K, int elem_bytes, int &NL, int &P)
{
    if (K != 4 && K != 8) return false;
    P = (len + K - 1) / K;
    if (P < 1 || P > 256) return false;
    NL = 256 / P;
    if (NL < 1) return false;
    return adjoint_chunk_smem(NL, P, elem_bytes) <= 48 * 1024;
}

// Accumulations of the split adjoint sweep, one thread per cell: with lambda of
// the rows (adjoint_chunk_kernel<..., SPLIT>) it adds, at a cell p of a line,
//   NONE rows:  nothing but the off-line dissipation terms below;
//   other rows: tbar = (IN ? mt : 1) tbar + [v == DIR] wb(p) + up(p-1) + dn(p+1),
//   IN rows:    sbar += 3/dt lambda(p),
// where wb, up and dn are the terms of the fused kernel (advection, pressure and
// along-line dissipation of IN rows p-1, p, p+1, recomputed here from lambda and
// the tape), and tbar[DIR] += the off-line dissipation terms of the four
// off-line neighbours n that are IN (ga(n) = t_phi lambda_T(n) g1(n) and gb(n)
// likewise), which the fused path writes into two planes and gathers in a
// second kernel.  Every cell has one writer, so no order of blocks matters.
template <typename R, int DIR>
__global__ void __launch_bounds__(256, 4)
    adjoint_accum_kernel(DomainView<R> d, CLayer<R> lam, CLayer<R> ti, CLayer<R> xs, Layer<R> sbar, Layer<R> tbar,
                         SweepConst<R> kc, int merges)
{
    // threadIdx.x: z; threadIdx.y: the along-line coordinate for X lines, y for Y and Z
    // lines, so a block's along-line neighbours mostly sit in the same block
    const int kk = blockIdx.x * 32 + threadIdx.x;
    const int ya = blockIdx.y * 8 + threadIdx.y;
    const int i = DIR == 0 ? ya : (int)blockIdx.z;
    const int j = DIR == 0 ? (int)blockIdx.z : ya;
    if (kk >= d.nz || i >= d.nx || j >= d.ny) return;
    const long long sx = (long long)d.ny * d.nz, sy = d.nz;
    const long long c = (long long)i * sx + (long long)j * sy + kk;
    const int p = DIR == 0 ? i : (DIR == 1 ? j : kk);
    const int len = DIR == 0 ? d.nx : (DIR == 1 ? d.ny : d.nz);
    const long long sl = DIR == 0 ? sx : (DIR == 1 ? sy : 1);
    const long long s1 = DIR == 0 ? sy : sx, s2 = DIR == 2 ? sy : 1;
    const int c1 = DIR == 0 ? j : i, n1 = DIR == 0 ? d.ny : d.nx;
    const int c2 = DIR == 2 ? j : kk, n2 = DIR == 2 ? d.ny : d.nz;
    const R h1 = DIR == 0 ? kc.inv_two_dy : kc.inv_two_dx;
    const R h2 = DIR == 2 ? kc.inv_two_dy : kc.inv_two_dz;
    // lambda, the tape and the codes are read-only here (non-coherent loads, free to
    // move ahead of the stores); sbar and tbar are read, then written, by this thread
    const R *U = ti.f[0], *V = ti.f[1], *W = ti.f[2], *Fd = ti.f[DIR];
    const uint8_t *code = d.code;

    // Every load is issued at once, without waiting for the codes: offsets that
    // would leave the line or the box are clamped to the cell itself (the values
    // loaded there are then discarded), so one memory round trip serves the cell.
    const long long om1 = p >= 1 ? -sl : 0, om2 = p >= 2 ? -2 * sl : 0;
    const long long op1 = p + 1 < len ? sl : 0, op2 = p + 2 < len ? 2 * sl : 0;
    const bool nok[4] = {c1 > 0, c1 + 1 < n1, c2 > 0, c2 + 1 < n2};
    const long long nb[4] = {c - (nok[0] ? s1 : 0), c + (nok[1] ? s1 : 0), c - (nok[2] ? s2 : 0),
                             c + (nok[3] ? s2 : 0)};
    const long long cm = c + om1, cp = c + op1;
    // off-line offsets of the rows p-1 and p+1 (their cells are IN when used, so
    // their off-line neighbours exist; clamped here only for the unused loads)
    const long long f1m = nok[0] ? s1 : 0, f1p = nok[1] ? s1 : 0, f2m = nok[2] ? s2 : 0, f2p = nok[3] ? s2 : 0;

    uint8_t cw[5], cn[4];
    cw[0] = __ldg(code + c + om2);
    cw[1] = __ldg(code + cm);
    cw[2] = __ldg(code + c);
    cw[3] = __ldg(code + cp);
    cw[4] = __ldg(code + c + op2);
#pragma unroll
    for (int q = 0; q < 4; q++) cn[q] = __ldg(code + nb[q]);
    R gl_n[4], gd_n[4];   // off-line neighbours: lambda_T and the in-line difference of g1 / g2
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const R *G = q >= 2 ? (DIR == 2 ? V : W) : (DIR == 0 ? V : U);
        gl_n[q] = __ldg(lam.f[3] + nb[q]);
        gd_n[q] = __ldg(G + nb[q] + op1) - __ldg(G + nb[q] + om1);
    }
    // rows p-1 and p+1: lambda, the in-line differences of U, V, W and the off-line
    // differences of Fd
    R lr[2][4], du[2][3], df[2][2];
#pragma unroll
    for (int v = 0; v < 4; v++) {
        lr[0][v] = __ldg(lam.f[v] + cm);
        lr[1][v] = __ldg(lam.f[v] + cp);
    }
    {
        const R u0 = __ldg(U + c), v0 = __ldg(V + c), w0 = __ldg(W + c);
        du[0][0] = u0 - __ldg(U + c + om2);
        du[0][1] = v0 - __ldg(V + c + om2);
        du[0][2] = w0 - __ldg(W + c + om2);
        du[1][0] = __ldg(U + c + op2) - u0;
        du[1][1] = __ldg(V + c + op2) - v0;
        du[1][2] = __ldg(W + c + op2) - w0;
    }
    df[0][0] = __ldg(Fd + cm + f1p) - __ldg(Fd + cm - f1m);
    df[0][1] = __ldg(Fd + cm + f2p) - __ldg(Fd + cm - f2m);
    df[1][0] = __ldg(Fd + cp + f1p) - __ldg(Fd + cp - f1m);
    df[1][1] = __ldg(Fd + cp + f2p) - __ldg(Fd + cp - f2m);
    R l0[4], dx[4], sb[4], tb[4];
#pragma unroll
    for (int v = 0; v < 4; v++) {
        l0[v] = __ldg(lam.f[v] + c);
        dx[v] = __ldg(xs.f[v] + cm) - __ldg(xs.f[v] + cp);
        sb[v] = sbar.f[v][c];
        tb[v] = tbar.f[v][c];
    }

    bool in[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int pp = p - 2 + q;
        in[q] = pp >= 0 && pp < len && code_is_in(cw[q]);
    }
    bool nin[4];
#pragma unroll
    for (int q = 0; q < 4; q++) nin[q] = nok[q] && code_is_in(cn[q]);
    const int k0 = qkind(in[1], in[2], in[3]);
    const bool in0 = k0 == Q_IN, km = in[1], kp = in[3];   // p-1, p+1 are IN rows exactly when IN cells

    // ---- off-line dissipation terms (ga / gb of the neighbours) ----
    R acc = R(0);
    {
        R g[4];
#pragma unroll
        for (int q = 0; q < 4; q++) g[q] = nin[q] ? (kc.t_phi * gl_n[q]) * (gd_n[q] * kc.inv_two_h) : R(0);
        if (nok[0]) acc += g[0] * h1;
        if (nok[1]) acc -= g[1] * h1;
        if (nok[2]) acc += g[2] * h2;
        if (nok[3]) acc -= g[3] * h2;
    }
    if (k0 == Q_NONE) {
        if (acc != R(0)) tbar.f[DIR][c] = tb[DIR] + acc;
        return;
    }

    // ---- the along-line terms rows p-1 and p+1 send here (up from p-1, dn = -up from p+1) ----
    R up[2][4];
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const R pt = kc.v_T * lr[r][DIR] * kc.inv_two_h;
        const R gl = kc.t_phi * lr[r][3];
        const R ua = du[r][0] * kc.inv_two_h, va = du[r][1] * kc.inv_two_h, wa = du[r][2] * kc.inv_two_h;
        const R f1 = df[r][0] * h1, f2 = df[r][1] * h2;
        R gu, gv, gw;
        if (DIR == 0) {
            gu = R(4) * ua; gv = R(2) * va + f1; gw = R(2) * wa + f2;
        } else if (DIR == 1) {
            gu = R(2) * ua + f1; gv = R(4) * va; gw = R(2) * wa + f2;
        } else {
            gu = R(2) * ua + f1; gv = R(2) * va + f2; gw = R(4) * wa;
        }
        const R s_h = gl * kc.inv_two_h;
        up[r][0] = gu * s_h;
        up[r][1] = gv * s_h;
        up[r][2] = gw * s_h;
        up[r][3] = -pt;
    }
    R wb = R(0);
    if (in0) {
        R w = R(0);
#pragma unroll
        for (int v = 0; v < 4; v++) w += l0[v] * dx[v];
        wb = w * kc.inv_two_h;
#pragma unroll
        for (int v = 0; v < 4; v++) sbar.f[v][c] = sb[v] + kc.three_dt * l0[v];
    }
    const R mt = merges == 2 ? R(0.25) : R(0.5);
#pragma unroll
    for (int v = 0; v < 4; v++) {
        R x = (in0 ? mt : R(1)) * tb[v];
        if (v == DIR) x += wb;
        x += km ? up[0][v] : R(0);
        x += kp ? -up[1][v] : R(0);
        if (v == DIR && acc != R(0)) x += acc;
        tbar.f[v][c] = x;
    }
}

template <typename R>
cudaError_t launch_adjoint_chunk(int dir, int K, const DomainView<R> &d, const int *lo, const int *hi, CLayer<R> ti,
                                 CLayer<R> xs, Layer<R> sbar, Layer<R> dbar, Layer<R> tbar, Layer<R> nvbar, R *ga, R *gb,
                                 const SweepConst<R> &k, int merges, bool split, Layer<R> lamo, cudaStream_t s)
{
    const LineGeom g = line_geom(dir, d.nx, d.ny, d.nz);
    int NL = 0, P = 0;
    if (!adjoint_chunk_supported(g.len, K, (int)sizeof(R), NL, P)) return cudaErrorInvalidConfiguration;
    const int threads = NL * P;
    const int blocks = (g.nlines + NL - 1) / NL;
    const size_t smem = adjoint_chunk_smem(NL, P, (int)sizeof(R));
#define AC(DD, KK)                                                                                                 \
    if (dir == DD && K == KK) {                                                                                    \
        if (split)                                                                                                 \
            adjoint_chunk_kernel<R, DD, KK, true><<<blocks, threads, smem, s>>>(                                  \
                d, g, NL, P, lo, hi, ti, xs, sbar, dbar, tbar, nvbar, ga, gb, k, merges, lamo);                   \
        else                                                                                                       \
            adjoint_chunk_kernel<R, DD, KK, false><<<blocks, threads, smem, s>>>(                                 \
                d, g, NL, P, lo, hi, ti, xs, sbar, dbar, tbar, nvbar, ga, gb, k, merges, lamo);                   \
        cudaError_t e = cudaGetLastError();                                                                        \
        if (e != cudaSuccess || !split) return e;                                                                  \
        const dim3 ab(32, 8);                                                                                      \
        const dim3 agrid((d.nz + 31) / 32, ((DD == 0 ? d.nx : d.ny) + 7) / 8, DD == 0 ? d.ny : d.nx);             \
        adjoint_accum_kernel<R, DD><<<agrid, ab, 0, s>>>(d, clayer_view(lamo), ti, xs, sbar, tbar, k, merges);    \
        return cudaGetLastError();                                                                                 \
    }
    AC(0, 4) AC(0, 8) AC(1, 4) AC(1, 8) AC(2, 4) AC(2, 8)
#undef AC
    return cudaErrorInvalidConfiguration;
}

#define INST(R)                                                                                                     \
    template cudaError_t launch_adjoint_chunk<R>(int, int, const DomainView<R> &, const int *, const int *,         \
                                                 CLayer<R>, CLayer<R>, Layer<R>, Layer<R>, Layer<R>, Layer<R>, R *, \
                                                 R *, const SweepConst<R> &, int, bool, Layer<R>, cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace adi
