// X and Y sweeps fed by the Tensor Memory Accelerator, on persistent CTAs.
//
// X and Y lines are strided in memory (X: ny*nz elements between the rows of a
// line, Y: nz), so a CTA works on a tile: NLT = 8 or 16 neighbouring lines
// (consecutive k at one j for X, at one i for Y) over their whole length L = P K.
// One thread issues the tile's loads (cp.async.bulk.tensor, no multicast) into
// shared memory:
//   cur   U V W T           NLT x L each
//   temp  three fields      NLT x L each
//   temp  advecting field   WIDE x L (the lines plus a k halo of at least one
//                                     line, x start kept 16-byte aligned)
//   temp  advecting field   NLT x L at j+-1 (X) / i+-1 (Y), the other off-line axis
//   codes                   16 x L bytes (16-byte aligned k start)
// Out-of-range boxes (first/last lines of the grid) are zero-filled by the hardware.
//
// The grid is persistent: as many CTAs as fit on the GPU, CTA b taking tiles b,
// b + gridDim.x, ...  Each tile's buffer is given back as early as possible.  Every
// thread builds its rows from the tile and eliminates its chunk (as the generic
// fast sweep, sweep_fast.cu: increment form, chunk elimination), then keeps in
// registers all that its write-back needs:
//   D  the row's new value when the chunk-end unknowns are zero (cur folded in at
//      increment-form rows),
//   G  the merged nonlinear value likewise ((temp + D) / 2, or its second merge),
// so that after one barrier the next tile's loads go into the same buffer and land
// while this tile's reduced system is solved and its results are written.  The
// reduced rows of the chunks go through shared memory to warps that own whole
// lines (lane = chunk), which run the cyclic-reduction step and the PCR over the
// chunk-first unknowns in warp shuffles, as the Z sweep does (sweep_zwarp.cu): two
// CTA barriers per tile instead of one per PCR step.  With c = a'' x_first +
// c'' x_last the write-back is next = D - c and, at IN rows, temp_out = G - c/2
// (3c/4 when the sweep carries the extra merge), straight from registers to global
// memory; nodes without a row are not touched.
//
// Thread t owns chunk c = t / NLT (rows c K .. c K + K - 1) of line t % NLT, so the
// lanes of a warp read the same row-in-chunk of 32 / NLT neighbouring chunks.  The
// tensor maps split the line coordinate into (row-in-chunk, chunk) so that tiles
// land as [i][c][lines]: those lanes then read 32 consecutive words, where the
// row-major [row][lines] layout put rows K apart into the same banks.
//
// The wait for a tile is bounded: if it has not landed after about a second the
// CTA raises the handle's error flag and leaves without writing that tile.
#include "adi_internal.cuh"
#include "sweep_common.cuh"

#include "tma.cuh"
#include "sweep_xyload.cuh"

#include <mutex>
#include <unordered_map>
#include <type_traits>
#include <vector>

namespace adi {

using tma::smem_u32;
using tma::load_4d;

namespace {

// Tile geometry of an X/Y launch with NLT lines of element type R.
template <typename R, int NLT>
struct XYTile {
    static constexpr int WIDE = NLT == 8 ? 16 : 24;   // advecting-field tile width
    static constexpr int WOFF = 4;                    // column of line 0 in that tile (k0 - 4 is 16-byte aligned)
};

__host__ __device__ constexpr size_t round128(size_t b) { return (b + 127) / 128 * 128; }

// CTAs per SM a launch shape is compiled for (FP32; FP64 tiles fit fewer): the
// register cap follows from it and the shared-memory budget per CTA must allow it
// (K = 8 with 8 lines: a 47 KB tile plus 11 KB of reduced-system slots, three;
// lines longer than 32 chunks: one CTA of NLT * P threads).
__host__ __device__ constexpr int xy_ctas_per_sm(int es, int K, int NLT, int P)
{
    return es != 4 || P > 32 ? 1
                             : (K == 4 ? (NLT == 8 ? 3 : 1) : (K == 8 ? (NLT == 8 ? 3 : 2) : (K == 5 ? 2 : 1)));
}


template <typename R, int NLT>
__host__ __device__ constexpr size_t xy_tile_bytes(int L)
{
    return 9 * round128((size_t)L * NLT * sizeof(R)) + round128((size_t)L * XYTile<R, NLT>::WIDE * sizeof(R)) +
           round128((size_t)L * 16);
}

} // namespace

// P (chunks per line) is a template parameter so that every tile offset is an
// immediate.  The register cap lets as many CTAs be resident as their shared
// memory allows (xy_ctas_per_sm): FP32 K = 8 four of 8 lines or two of 16, K = 4
// three of 8 lines.
template <typename R, int DIR, int K, int NLT, int P, typename Loader>
__global__ void __launch_bounds__(NLT * P, xy_ctas_per_sm((int)sizeof(R), K, NLT, P))
    sweep_xy_kernel(const __grid_constant__ Loader ld, int merges, int ntiles, int *err_flag)
{
    using T = XYTile<R, NLT>;
    constexpr int WIDE = T::WIDE, WOFF = T::WOFF;
    constexpr int L = P * K;
    extern __shared__ __align__(128) unsigned char smem[];
    const int t = threadIdx.x;
    const int ch = t / NLT, li = t - ch * NLT;

    // tile layout ([K][P][width] each; every tile starts on a 128-byte boundary)
    constexpr size_t plane = round128((size_t)L * NLT * sizeof(R));
    constexpr size_t wide_bytes = round128((size_t)L * WIDE * sizeof(R));
    constexpr size_t code_bytes = round128((size_t)L * 16);
    constexpr int fs = (int)(plane / sizeof(R));                      // elements between two fields of a tile
    R *const tcur = reinterpret_cast<R *>(smem);                      // [4] cur fields
    R *const ttin = reinterpret_cast<R *>(smem + 4 * plane);          // [3] temp fields other than DIR
    R *const twide = reinterpret_cast<R *>(smem + 7 * plane);         // temp DIR field, WIDE columns
    R *const thm = reinterpret_cast<R *>(smem + 7 * plane + wide_bytes);   // temp DIR field at outer-1
    R *const thp = reinterpret_cast<R *>(smem + 8 * plane + wide_bytes);   // temp DIR field at outer+1
    uint8_t *const tcode = smem + 9 * plane + wide_bytes;             // codes, 16 columns
    // Reduced rows of the chunks go through shared memory to the warps that solve
    // them: slot q = line * (P + 1) + chunk (line-major, padded so that the writing
    // lanes -- NLT lines of 32 / NLT chunks -- and the reading lanes -- the chunks of
    // 32 / P lines -- both spread over all banks), stored as 16-byte units, unit u of
    // slot q at u * NQ + q.  RED holds the 16 values of a chunk's reduced rows, XS the
    // 8 results (x_first, x_last of the four fields) read back by the chunk's owner.
    constexpr int NQ = NLT * (P + 1);
    constexpr int UW = 16 / (int)sizeof(R);   // values per 16-byte unit
    using U16 = typename std::conditional<sizeof(R) == 4, float4, double2>::type;
    U16 *const RED = reinterpret_cast<U16 *>(smem + 9 * plane + wide_bytes + code_bytes);
    U16 *const XS = RED + 16 / UW * NQ;
    const XYSmem<R> sm{tcur, ttin, twide, thm, thp, tcode, reinterpret_cast<uint64_t *>(XS + 8 / UW * NQ)};
    auto ustore = [&](U16 *buf, int q, const R *v, int n) {
#pragma unroll
        for (int u = 0; u < n / UW; u++) {
            if constexpr (sizeof(R) == 4) buf[u * NQ + q] = make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
            else buf[u * NQ + q] = make_double2(v[2 * u], v[2 * u + 1]);
        }
    };
    auto uload = [&](const U16 *buf, int q, R *v, int n) {
#pragma unroll
        for (int u = 0; u < n / UW; u++) {
            const U16 a = buf[u * NQ + q];
            if constexpr (sizeof(R) == 4) { v[4 * u] = a.x; v[4 * u + 1] = a.y; v[4 * u + 2] = a.z; v[4 * u + 3] = a.w; }
            else { v[2 * u] = a.x; v[2 * u + 1] = a.y; }
        }
    };
    // The warp-phase role of this thread: chunk wc of line wl.  A line of P <= 32
    // chunks sits in P lanes of one warp (32 / P lines per warp); a longer line
    // (P = 32 W) in W consecutive warps, which meet on a named barrier of their own.
    const int lane = t & 31;
    constexpr int WPL = P > 32 ? P / 32 : 1;   // warps per line
    static_assert(P <= 32 || P % 32 == 0, "lines longer than a warp span whole warps");
    const int wl = P <= 32 ? (t >> 5) * (32 / P) + lane / P : (t >> 5) / WPL;
    const int wc = P <= 32 ? lane % P : 32 * ((t >> 5) % WPL) + lane;
    auto line_sync = [&]() {
        if constexpr (P <= 32) __syncwarp();
        else asm volatile("bar.sync %0, %1;" ::"r"(1 + wl), "r"(32 * WPL) : "memory");
    };


    ld.init(sm, t);
    __syncthreads();
    uint64_t codes = (int)blockIdx.x < ntiles ? ld.issue(blockIdx.x, sm, fs, t) : 0;

    using namespace sweep;
    const int p0 = ch * K;
    const R gm = merges == 2 ? R(0.75) : R(0.5);   // share of the correction c in temp_out
    // the merged nonlinear value (temp + x) / 2, or with the extra merge (temp + 3 x) / 4
    const R gw_new = gm, gw_old = R(1) - gm;
    // Tile row (i P + c) of row p0 + i, i in [-1, K]: rows -1 and K belong to the
    // neighbouring chunks; outside the line, this chunk's own row stands in.
    auto trow = [&](int i) -> int {
        if (i < 0) return ch > 0 ? (K - 1) * P + ch - 1 : ch;
        if (i >= K) return ch + 1 < P ? ch + 1 : (K - 1) * P + ch;
        return i * P + ch;
    };
    const R *__restrict__ cT = tcur + li;         // cur tile column of this line
    const R *__restrict__ wT = twide + li + WOFF; // advecting field column (k halo at -1/+1)
    auto tin_of = [&](int v) -> const R * { return ttin + (v < DIR ? v : v - 1) * fs + li; };
    auto temp_at = [&](int v, int tr) -> R { return v == DIR ? wT[tr * WIDE] : tin_of(v)[tr * NLT]; };

    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const XYTileGeo geo = ld.geo(tile);
        const SweepConst<R> &kc = ld.consts(geo);
        // The tile's copies have landed (TMA: a bounded wait; a thread whose wait
        // gave up computes on whatever the tile holds, and the CTA checks every
        // thread's wait at the release barrier and leaves before writing anything
        // of this tile).
        const bool tiles_ok = ld.wait(it, sm, t, codes);

        // ---------------- rows from the tile: one pass, 3-row window ----------------
        const int code_col = li + geo.code_off;       // this line's byte in a code row
        // window slots: 0 = row i-1, 1 = row i, 2 = row i+1.  cur is kept only for IN
        // rows (the reference vector of the increment form is 0 elsewhere).
        R cw[3][4], tw[3][4];
        uint8_t kw[3];
#define XY_LOAD_ROW(SLOT_, I_)                                                                       \
    {                                                                                                \
        const int ii = (I_);                                                                         \
        const bool ok = (ii >= 0 || ch > 0) && (ii < K || ch + 1 < P);                               \
        const int tr = trow(ii);                                                                     \
        const uint8_t c = ok ? tcode[tr * 16 + code_col] : uint8_t(NODE_OUT);                       \
        kw[SLOT_] = c;                                                                               \
        const bool in = code_is_in(c);                                                               \
        _Pragma("unroll") for (int v = 0; v < 4; v++)                                                \
        {                                                                                            \
            tw[SLOT_][v] = ok ? temp_at(v, tr) : R(0);                                               \
            cw[SLOT_][v] = in ? cT[v * fs + tr * NLT] : R(0);                                        \
        }                                                                                            \
    }
        int kind[K];
        unsigned freebits = 0;
        R rr[K], dv[4][K];
        XY_LOAD_ROW(0, -1)
        XY_LOAD_ROW(1, 0)
        // global offset of this line's node 0: X (0, j, k) = j*nz + k; Y (i, 0, k) = i*ny*nz + k
        const long long lb = geo.lb0 + li;
#pragma unroll
        for (int i = 0; i < K; i++) {
            XY_LOAD_ROW(2, i + 1)
            const int kd = row_kind(code_is_in(kw[0]), code_is_in(kw[1]), code_is_in(kw[2]));
            kind[i] = kd;
            if (kw[1] & CODE_VEL_FREE) freebits |= 1u << (2 * i);
            if (kw[1] & CODE_TEMP_FREE) freebits |= 2u << (2 * i);
            rr[i] = R(0);
            if (kd == R_IN) {
                // IN rows are never the first or last node of a line
                const R r = tw[1][DIR] * kc.inv_two_h;
                rr[i] = r;
                R fa, fb;
                if constexpr (sizeof(R) == 4) {
                    // packed FP32: (U, T) and (V, W) two at a time
                    const float2 lap03 = fma2(bc2(-2.0f), p2(cw[1][0], cw[1][3]), add2(p2(cw[0][0], cw[0][3]),
                                                                                     p2(cw[2][0], cw[2][3])));
                    const float2 lap12 = fma2(bc2(-2.0f), p2(cw[1][1], cw[1][2]), add2(p2(cw[0][1], cw[0][2]),
                                                                                     p2(cw[2][1], cw[2][2])));
                    const float2 dif03 = fma2(bc2(-1.0f), p2(cw[0][0], cw[0][3]), p2(cw[2][0], cw[2][3]));
                    const float2 dif12 = fma2(bc2(-1.0f), p2(cw[0][1], cw[0][2]), p2(cw[2][1], cw[2][2]));
                    const float2 d03 = fma2(p2(kc.vis_v, kc.vis_t), lap03, mul2(bc2(-r), dif03));
                    const float2 d12 = fma2(bc2(kc.vis_v), lap12, mul2(bc2(-r), dif12));
                    dv[0][i] = d03.x; dv[3][i] = d03.y; dv[1][i] = d12.x; dv[2][i] = d12.y;
                    const float2 fab = mul2(fma2(bc2(-1.0f), p2(tw[0][0], tw[0][1]), p2(tw[2][0], tw[2][1])),
                                            bc2(kc.inv_two_h));
                    fa = fab.x;
                    fb = fab.y;
                } else {
#pragma unroll
                    for (int v = 0; v < 4; v++) {
                        const R vis = v < 3 ? kc.vis_v : kc.vis_t;
                        dv[v][i] = vis * (cw[0][v] - R(2) * cw[1][v] + cw[2][v]) - r * (cw[2][v] - cw[0][v]);
                    }
                    fa = (tw[2][0] - tw[0][0]) * kc.inv_two_h;
                    fb = (tw[2][1] - tw[0][1]) * kc.inv_two_h;
                }
                dv[DIR][i] -= kc.v_T * ((tw[2][3] - tw[0][3]) * kc.inv_two_h);
                const R fc = (tw[2][2] - tw[0][2]) * kc.inv_two_h;
                const int tr = i * P + ch;
                const R g1 = (thp[tr * NLT + li] - thm[tr * NLT + li]) * (DIR == 0 ? kc.inv_two_dy : kc.inv_two_dx);
                const R g2 = (wT[tr * WIDE + 1] - wT[tr * WIDE - 1]) * kc.inv_two_dz;
                R diss;
                if (DIR == 0) diss = R(2) * fa * fa + fb * fb + fc * fc + fb * g1 + fc * g2;
                else diss = fa * fa + R(2) * fb * fb + fc * fc + fa * g1 + fc * g2;
                dv[3][i] += kc.t_phi * diss;
            } else if (kd == R_NONE) {
#pragma unroll
                for (int v = 0; v < 4; v++) dv[v][i] = R(0);
            } else {
                // boundary row; BC_FREE moves the IN neighbour's cur to the right side
                const bool vf = (kw[1] & CODE_VEL_FREE) != 0, tf = (kw[1] & CODE_TEMP_FREE) != 0;
                const bool from_left = kd == R_END;   // IN neighbour at p-1, else at p+1
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const bool fr = v < 3 ? vf : tf;
                    const R cn = from_left ? cw[0][v] : cw[2][v];
                    dv[v][i] = fr ? cn
                                  : (kc.nv_in_temp ? tw[1][v]
                                                   : __ldg(ld.nv(geo, v) + lb + (long long)(p0 + i) * geo.stride));
                }
            }
#pragma unroll
            for (int v = 0; v < 4; v++) {
                cw[0][v] = cw[1][v]; cw[1][v] = cw[2][v];
                tw[0][v] = tw[1][v]; tw[1][v] = tw[2][v];
            }
            kw[0] = kw[1];
            kw[1] = kw[2];
        }
#undef XY_LOAD_ROW

        // ---------------- chunk elimination ----------------
        R ea[2][K], ec[2][K];
        Reduced<R> red;
        eliminate<R, K>(kind, rr, freebits, kc, dv, ea, ec, red);

        // ---------------- D and G from the tile, kinds packed ----------------
        // dv becomes D: d'' plus cur at IN rows for the interior rows, and for the
        // chunk-end rows (whose d' went into the reduced rows) cur at IN rows, else 0.
        R gv[4][K];
        using KindBits = typename std::conditional<(3 * K > 32), unsigned long long, unsigned>::type;
        KindBits kinds = 0;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int kd = kind[i];
            kinds |= (KindBits)kd << (3 * i);
            const bool edge = i == 0 || i == K - 1;
            const int tr = i * P + ch;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                R dd = edge ? R(0) : dv[v][i], m = R(0);
                if (kd == R_IN) {
                    dd += cT[v * fs + tr * NLT];
                    m = fma(dd, gw_new, temp_at(v, tr) * gw_old);
                }
                dv[v][i] = dd;
                gv[v][i] = m;
            }
        }

        // ---------------- reduced system: CR step + PCR in warp shuffles ----------------
        {
            const R rv[16] = {red.Af[0], red.Af[1], red.Cf[0], red.Cf[1], red.Al[0], red.Al[1], red.Cl[0], red.Cl[1],
                              red.Df[0], red.Df[1], red.Df[2], red.Df[3], red.Dl[0], red.Dl[1], red.Dl[2], red.Dl[3]};
            ustore(RED, li * (P + 1) + ch, rv, 16);
        }
        // Release barrier: every read of this tile is done, so the next tile's loads
        // may overwrite it; a thread whose wait gave up makes the whole CTA leave.
        if (__syncthreads_or(!tiles_ok)) {
            if (t == 0) atomicExch(err_flag, 1);
            ld.abandon(it, sm, t);
            break;
        }
        if (tile + (int)gridDim.x < ntiles) codes = ld.issue(tile + gridDim.x, sm, fs, t);
        {
            // Lane wc of a P-lane segment holds chunk wc of line wl.  Couplings to rows
            // outside the line are exactly zero (the first row of a line has a = 0, the
            // last c = 0, and PCR keeps them zero), so a lane whose partner lies outside
            // the segment takes its own row from the shuffle: finite values times 0.
            R rv[16];
            uload(RED, wl * (P + 1) + wc, rv, 16);
            Reduced<R> wr;
#pragma unroll
            for (int m = 0; m < 2; m++) {
                wr.Af[m] = rv[m]; wr.Cf[m] = rv[2 + m]; wr.Al[m] = rv[4 + m]; wr.Cl[m] = rv[6 + m];
            }
#pragma unroll
            for (int v = 0; v < 4; v++) { wr.Df[v] = rv[8 + v]; wr.Dl[v] = rv[12 + v]; }
            R ea_[2], ec_[2], ed[4];
            R xo[8];
            (void)line_sync;
            if constexpr (P <= 32) {
                auto up = [&](R x, int dd) { return __shfl_up_sync(0xffffffffu, x, dd, P); };
                auto dn = [&](R x, int dd) { return __shfl_down_sync(0xffffffffu, x, dd, P); };
                {
                    // cyclic-reduction step with the previous chunk's last row
                    R pv[8] = {up(wr.Al[0], 1), up(wr.Cl[0], 1), up(wr.Al[1], 1), up(wr.Cl[1], 1),
                               up(wr.Dl[0], 1), up(wr.Dl[1], 1), up(wr.Dl[2], 1), up(wr.Dl[3], 1)};
                    if (wc == 0) {
#pragma unroll
                        for (int q = 0; q < 8; q++) pv[q] = R(0);
                    }
                    cr_step<R>(wr, pv, ea_, ec_, ed);
                }
#pragma unroll
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
            } else {
                // The line's rows are exchanged through shared memory, the line's
                // warps meeting on their named barrier: the cyclic-reduction step
                // reads the previous chunk's RED slot, then RED's two halves serve as
                // the ping-pong buffers of the PCR steps (each 8 values per slot).
                const int q = wl * (P + 1) + wc;
                {
                    R pv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
                    if (wc > 0) {
                        R pr[16];
                        uload(RED, q - 1, pr, 16);
                        pv[0] = pr[4]; pv[1] = pr[6]; pv[2] = pr[5]; pv[3] = pr[7];
#pragma unroll
                        for (int v = 0; v < 4; v++) pv[4 + v] = pr[12 + v];
                    }
                    cr_step<R>(wr, pv, ea_, ec_, ed);
                }
                U16 *const bufA = RED, *const bufB = RED + 8 / UW * NQ;
                line_sync();   // every RED read of the line is done
                int n = 0;
#pragma unroll
                for (int st = 1; st < P; st <<= 1, n++) {
                    U16 *const bw = (n & 1) ? bufA : bufB;
                    const R mine[8] = {ea_[0], ec_[0], ea_[1], ec_[1], ed[0], ed[1], ed[2], ed[3]};
                    ustore(bw, q, mine, 8);
                    line_sync();
                    R mv[8], pv[8];
                    uload(bw, wc - st >= 0 ? q - st : q, mv, 8);
                    uload(bw, wc + st < P ? q + st : q, pv, 8);
                    pcr_update<R>(mv, pv, ea_, ec_, ed);
                }
                U16 *const bx = (n & 1) ? bufA : bufB;
                const R mine[8] = {ed[0], ed[1], ed[2], ed[3], R(0), R(0), R(0), R(0)};
                ustore(bx, q, mine, 8);
                line_sync();
                R nf[8];
                uload(bx, wc + 1 < P ? q + 1 : q, nf, 8);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const int m = v < 3 ? 0 : 1;
                    xo[v] = ed[v];
                    xo[4 + v] = wr.Dl[v] - wr.Al[m] * ed[v] - wr.Cl[m] * (wc + 1 < P ? nf[v] : R(0));
                }
            }
            ustore(XS, wl * (P + 1) + wc, xo, 8);
        }
        __syncthreads();
        R xf[4], xl[4];
        {
            R xo[8];
            uload(XS, li * (P + 1) + ch, xo, 8);
#pragma unroll
            for (int v = 0; v < 4; v++) { xf[v] = xo[v]; xl[v] = xo[4 + v]; }
        }

        // ---------------- write-back from registers ----------------
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int kd = (kinds >> (3 * i)) & 7;
            if (kd == R_NONE) continue;
            const long long off = lb + (long long)(p0 + i) * geo.stride;
            R c[4];   // correction from the chunk-end unknowns
            if constexpr (sizeof(R) == 4) {
                float2 c03, c12;
                if (i == 0) { c03 = neg2(p2(xf[0], xf[3])); c12 = neg2(p2(xf[1], xf[2])); }
                else if (i == K - 1) { c03 = neg2(p2(xl[0], xl[3])); c12 = neg2(p2(xl[1], xl[2])); }
                else {
                    c03 = fma2(p2(ec[0][i], ec[1][i]), p2(xl[0], xl[3]), mul2(p2(ea[0][i], ea[1][i]), p2(xf[0], xf[3])));
                    c12 = fma2(bc2(ec[0][i]), p2(xl[1], xl[2]), mul2(bc2(ea[0][i]), p2(xf[1], xf[2])));
                }
                const float2 x03 = add2(p2(dv[0][i], dv[3][i]), neg2(c03));
                const float2 x12 = add2(p2(dv[1][i], dv[2][i]), neg2(c12));
                R *const n0 = ld.nextp(geo, 0), *const n1 = ld.nextp(geo, 1), *const n2 = ld.nextp(geo, 2), *const n3 = ld.nextp(geo, 3);
                n0[off] = x03.x; n3[off] = x03.y; n1[off] = x12.x; n2[off] = x12.y;
                if (kd == R_IN) {
                    const float2 m03 = fma2(bc2(-gm), c03, p2(gv[0][i], gv[3][i]));
                    const float2 m12 = fma2(bc2(-gm), c12, p2(gv[1][i], gv[2][i]));
                    R *const t0 = ld.toutp(geo, 0), *const t1 = ld.toutp(geo, 1), *const t2 = ld.toutp(geo, 2), *const t3 = ld.toutp(geo, 3);
                    t0[off] = m03.x; t3[off] = m03.y; t1[off] = m12.x; t2[off] = m12.y;
                }
                (void)c;
            } else {
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const int m = v < 3 ? 0 : 1;
                    c[v] = i == 0 ? -xf[v] : (i == K - 1 ? -xl[v] : ea[m][i] * xf[v] + ec[m][i] * xl[v]);
                    ld.nextp(geo, v)[off] = dv[v][i] - c[v];
                    if (kd == R_IN) ld.toutp(geo, v)[off] = gv[v][i] - gm * c[v];
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host side: tensor maps and launch
// ---------------------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 get_encoder_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Box {w, 1, Lb} for X lines / {w, Lb, 1} for Y lines over a [nx][ny][nz] array.
// Encoded maps are cached by their arguments (the arrays live as long as their
// handle; a freed-and-reused address gets the same, still valid, map).
bool have_tensor_map_encoder() { return get_encoder_fn() != nullptr; }

namespace {
struct MapKey {
    const void *base;
    int kind, dir, nx, ny, nz, w, n, es, dt;
    bool operator==(const MapKey &o) const
    {
        return base == o.base && kind == o.kind && dir == o.dir && nx == o.nx && ny == o.ny && nz == o.nz &&
               w == o.w && n == o.n && es == o.es && dt == o.dt;
    }
};

struct MapKeyHash {
    size_t operator()(const MapKey &k) const
    {
        size_t h = std::hash<const void *>()(k.base);
        for (int v : {k.kind, k.dir, k.nx, k.ny, k.nz, k.w, k.n, k.es, k.dt}) h = h * 1000003u ^ (size_t)(unsigned)v;
        return h;
    }
};

// Encodes (or finds in the cache) a map of the given rank, dims, strides and box.
// The cache is a hash map: the adjoint's taped steps sweep over hundreds of tape
// slots, each with its own maps, and every launch looks up about ten.
bool encode_cached(CUtensorMap *m, const MapKey &key, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                   const cuuint32_t *box)
{
    static std::unordered_map<MapKey, CUtensorMap, MapKeyHash> cache;
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) { *m = it->second; return true; }
    }
    auto enc = get_encoder_fn();
    if (!enc) return false;
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(m, (CUtensorMapDataType)key.dt, rank, const_cast<void *>(key.base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    std::lock_guard<std::mutex> g(mu);
    if (cache.size() > 16384) cache.clear();
    cache.emplace(key, *m);
    return true;
}
} // namespace

bool make_tile_map(CUtensorMap *m, const void *base, int dir, int nx, int ny, int nz, int w, int Lb, int es,
                   CUtensorMapDataType dt)
{
    const MapKey key{base, 0, dir, nx, ny, nz, w, Lb, es, (int)dt};
    cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)nz * es, (cuuint64_t)ny * nz * es};
    cuuint32_t box[3] = {(cuuint32_t)w, (cuuint32_t)(dir == 0 ? 1 : Lb), (cuuint32_t)(dir == 0 ? Lb : 1)};
    return encode_cached(m, key, 3, dims, strides, box);
}

bool make_chunk_map(CUtensorMap *m, const void *base, int dir, int nx, int ny, int nz, int w, int K, int es,
                    CUtensorMapDataType dt, int box_rows)
{
    const MapKey key{base, 1 + box_rows, dir, nx, ny, nz, w, K, es, (int)dt};
    const cuuint64_t row = (cuuint64_t)(dir == 0 ? (size_t)ny * nz : (size_t)nz) * es;   // one step along the line
    const int P = (dir == 0 ? nx : ny) / K;
    if (dir == 0) {
        cuuint64_t dims[4] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)P, (cuuint64_t)K};
        cuuint64_t strides[3] = {(cuuint64_t)nz * es, row * K, row};
        cuuint32_t box[4] = {(cuuint32_t)w, 1, (cuuint32_t)P, (cuuint32_t)box_rows};
        return encode_cached(m, key, 4, dims, strides, box);
    }
    cuuint64_t dims[4] = {(cuuint64_t)nz, (cuuint64_t)P, (cuuint64_t)K, (cuuint64_t)nx};
    cuuint64_t strides[3] = {row * K, row, (cuuint64_t)ny * nz * es};
    cuuint32_t box[4] = {(cuuint32_t)w, (cuuint32_t)P, (cuuint32_t)box_rows, 1};
    return encode_cached(m, key, 4, dims, strides, box);
}

template <typename R, int NLT>
static size_t xytma_smem(int L, int P)
{
    return xy_tile_bytes<R, NLT>(L) + (size_t)NLT * (P + 1) * 24 * sizeof(R) + 16 /* mbarrier */;
}

size_t xytma_smem_bytes(int L, int P, int nlt, int elem_bytes)
{
    if (elem_bytes == 8) return nlt == 8 ? xytma_smem<double, 8>(L, P) : xytma_smem<double, 16>(L, P);
    return nlt == 8 ? xytma_smem<float, 8>(L, P) : xytma_smem<float, 16>(L, P);
}

bool xytma_supported(int dir, int nx, int ny, int nz, int K, int nlt, int elem_bytes)
{
    if (dir > 1 || !have_tensor_map_encoder()) return false;
    if (nlt != 8 && nlt != 16) return false;
    const int L = dir == 0 ? nx : ny;
    if (nz % 16 != 0) return false;             // CTA tiles of nlt lines; 16-byte code rows
    if (K != 4 && K != 8 && K != 16) return false;
    if (L % K != 0) return false;
    const int P = L / K;
    // compiled chunk counts; lines of 64 or 96 chunks (several warps per line) in float, K = 4, 8 lines
    const bool multi = (P == 64 || P == 96) && K == 4 && nlt == 8 && elem_bytes == 4;
    if (P != 4 && P != 8 && P != 16 && !(P == 32 && K == 4) && !multi) return false;
    const int threads = nlt * P;
    if (threads < 32 || threads > 1024) return false;
    // the CTAs per SM the shape is compiled for (228 KB per SM, 1 KB reserved per CTA)
    const size_t budget = 228 * 1024 / xy_ctas_per_sm(elem_bytes, K, nlt, P) - 1024;
    return xytma_smem_bytes(L, P, nlt, elem_bytes) <= (budget < 227 * 1024 ? budget : 227 * 1024);
}

namespace {
// Resident CTAs of one kernel instantiation per SM times the SM count, per device
// (the persistent grid of that instantiation).
struct PersistentGrid {
    std::mutex mu;
    int ctas[64] = {};
};

template <typename F>
int persistent_ctas(PersistentGrid &rec, F *kern, int threads, size_t smem)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    std::lock_guard<std::mutex> lock(rec.mu);
    if (!rec.ctas[dev]) {
        int per_sm = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess) return 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        rec.ctas[dev] = per_sm * sms;
    }
    return rec.ctas[dev];
}
} // namespace

template <typename R>
cudaError_t launch_sweep_xytma(int dir, const DomainView<R> &d, const int *line_lo, CLayer<R> cur, CLayer<R> tin,
                               Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges, int K, int nlt,
                               int *err_flag, cudaStream_t s)
{
    (void)line_lo;   // every tile is processed; lines without segments have no rows
    const int es = (int)sizeof(R);
    if (!xytma_supported(dir, d.nx, d.ny, d.nz, K, nlt, es)) return cudaErrorInvalidConfiguration;
    const LineGeom g = line_geom(dir, d.nx, d.ny, d.nz);
    const int L = g.len, P = L / K;
    const CUtensorMapDataType dt = es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const int wide = nlt == 8 ? XYTile<R, 8>::WIDE : XYTile<R, 16>::WIDE;
    XYMaps maps;
    for (int v = 0; v < 4; v++) {
        if (!make_chunk_map(&maps.cur[v], cur.f[v], dir, d.nx, d.ny, d.nz, nlt, K, es, dt, K))
            return cudaErrorInvalidValue;
        if (!make_chunk_map(&maps.tin[v], tin.f[v], dir, d.nx, d.ny, d.nz, nlt, K, es, dt, K))
            return cudaErrorInvalidValue;
    }
    if (!make_chunk_map(&maps.fwide, tin.f[dir], dir, d.nx, d.ny, d.nz, wide, K, es, dt, K))
        return cudaErrorInvalidValue;
    if (!make_chunk_map(&maps.code, d.code, dir, d.nx, d.ny, d.nz, 16, K, 1, CU_TENSOR_MAP_DATA_TYPE_UINT8, K))
        return cudaErrorInvalidValue;
    const size_t smem = xytma_smem_bytes(L, P, nlt, es);
    const int ntiles = (dir == 0 ? d.ny : d.nx) * (d.nz / nlt);
    const int threads = nlt * P;
#define XL(DD, KK, NN, PP)                                                                                       \
    if (dir == DD && K == KK && nlt == NN && P == PP) {                                                          \
        using Ld = XYTmaLoader<R, DD, KK, NN, PP, XYTile<R, NN>::WIDE, XYTile<R, NN>::WOFF>;                      \
        auto kern = sweep_xy_kernel<R, DD, KK, NN, PP, Ld>;                                                      \
        static SmemOptIn opt_in;                                                                                 \
        static PersistentGrid pgrid;                                                                             \
        cudaError_t e = ensure_dynamic_smem(opt_in, kern, smem);                                                 \
        if (e != cudaSuccess) return e;                                                                          \
        const int ctas = persistent_ctas(pgrid, kern, threads, smem);                                            \
        if (ctas <= 0) return cudaErrorInvalidConfiguration;                                                     \
        Ld ld;                                                                                                   \
        ld.maps = maps; ld.d = d; ld.next = next; ld.tout = tout; ld.kc = k; ld.kblocks = d.nz / NN;             \
        kern<<<ctas < ntiles ? ctas : ntiles, threads, smem, s>>>(ld, merges, ntiles, err_flag);                 \
        return cudaGetLastError();                                                                               \
    }
#define XLP(DD, KK, NN) XL(DD, KK, NN, 4) XL(DD, KK, NN, 8) XL(DD, KK, NN, 16)
    XLP(0, 8, 8) XLP(0, 16, 8) XLP(1, 8, 8) XLP(1, 16, 8)
    XLP(0, 8, 16) XLP(0, 16, 16) XLP(1, 8, 16) XLP(1, 16, 16)
    XLP(0, 4, 8) XLP(1, 4, 8) XLP(0, 4, 16) XLP(1, 4, 16)
    XL(0, 4, 8, 32) XL(1, 4, 8, 32) XL(0, 4, 16, 32) XL(1, 4, 16, 32)
    if constexpr (sizeof(R) == 4) {
        XL(0, 4, 8, 64) XL(1, 4, 8, 64) XL(0, 4, 8, 96) XL(1, 4, 8, 96)
    }
#undef XLP
#undef XL
    return cudaErrorInvalidConfiguration;
}

// ---------------------------------------------------------------------------
// element-wise (cp.async) tiles: any nz and line length, one domain or a batch
// ---------------------------------------------------------------------------

// Chunks per line of the cp.async shapes: 8 lines per CTA, K = 4 with 16 or 32
// chunks (lines up to 64 / 128 rows), K = 5 with 32 (up to 160 rows).
static int xycp_chunks(int L, int K)
{
    if (K == 4) return L <= 64 ? 16 : (L <= 128 ? 32 : 0);
    if (K == 5) return L <= 160 ? 32 : 0;
    return 0;
}

bool xycp_supported(int dir, int nx, int ny, int nz, int K, int elem_bytes)
{
    if (dir > 1 || nx < 3 || ny < 3 || nz < 3) return false;
    const int L = dir == 0 ? nx : ny;
    const int P = xycp_chunks(L, K);
    if (P == 0) return false;
    const size_t budget = 228 * 1024 / xy_ctas_per_sm(elem_bytes, K, 8, P) - 1024;
    return xytma_smem_bytes(P * K, P, 8, elem_bytes) <= (budget < 227 * 1024 ? budget : 227 * 1024);
}

template <typename R>
cudaError_t launch_sweep_xycp(int dir, const DomainView<R> &d, CLayer<R> cur, CLayer<R> tin, Layer<R> next,
                              Layer<R> tout, const SweepConst<R> &k, int merges, int K, int *err_flag, cudaStream_t s)
{
    const int es = (int)sizeof(R);
    if (!xycp_supported(dir, d.nx, d.ny, d.nz, K, es)) return cudaErrorInvalidConfiguration;
    const int L = dir == 0 ? d.nx : d.ny;
    const int P = xycp_chunks(L, K);
    const size_t smem = xytma_smem_bytes(P * K, P, 8, es);
    const int kblocks = (d.nz + 7) / 8;
    const int ntiles = (dir == 0 ? d.ny : d.nx) * kblocks;
    const int threads = 8 * P;
#define XC(DD, KK, PP)                                                                                           \
    if (dir == DD && K == KK && P == PP) {                                                                       \
        using Ld = XYCpLoader<R, DD, KK, 8, PP, XYTile<R, 8>::WIDE, XYTile<R, 8>::WOFF>;                          \
        auto kern = sweep_xy_kernel<R, DD, KK, 8, PP, Ld>;                                                       \
        static SmemOptIn opt_in;                                                                                 \
        static PersistentGrid pgrid;                                                                             \
        cudaError_t e = ensure_dynamic_smem(opt_in, kern, smem);                                                 \
        if (e != cudaSuccess) return e;                                                                          \
        const int ctas = persistent_ctas(pgrid, kern, threads, smem);                                            \
        if (ctas <= 0) return cudaErrorInvalidConfiguration;                                                     \
        Ld ld;                                                                                                   \
        ld.cur = cur; ld.tin = tin; ld.d = d; ld.next = next; ld.tout = tout; ld.kc = k;                         \
        ld.kblocks = kblocks; ld.L = L;                                                                          \
        kern<<<ctas < ntiles ? ctas : ntiles, threads, smem, s>>>(ld, merges, ntiles, err_flag);                 \
        return cudaGetLastError();                                                                               \
    }
    XC(0, 4, 16) XC(1, 4, 16) XC(0, 4, 32) XC(1, 4, 32) XC(0, 5, 32) XC(1, 5, 32)
#undef XC
    return cudaErrorInvalidConfiguration;
}

// The X or Y sweep of every domain of a batch in one persistent launch over the
// (domain, tile) work items; every domain's line length in the direction must be
// at most 32 K rows.
template <typename R>
cudaError_t launch_sweep_xy_batch(int dir, int K, const BatchDomain<R> *doms, const int2 *items, int nitems, int src,
                                  int tin, int dst, int tout, int merges, int *err_flag, cudaStream_t s)
{
    if (nitems == 0) return cudaSuccess;
    const int es = (int)sizeof(R);
    constexpr int P = 32;
    const size_t smem = xytma_smem_bytes(P * K, P, 8, es);
#define XB(DD, KK)                                                                                               \
    if (dir == DD && K == KK) {                                                                                  \
        using Ld = XYBatchLoader<R, DD, KK, 8, P, XYTile<R, 8>::WIDE, XYTile<R, 8>::WOFF>;                        \
        auto kern = sweep_xy_kernel<R, DD, KK, 8, P, Ld>;                                                        \
        static SmemOptIn opt_in;                                                                                 \
        static PersistentGrid pgrid;                                                                             \
        cudaError_t e = ensure_dynamic_smem(opt_in, kern, smem);                                                 \
        if (e != cudaSuccess) return e;                                                                          \
        const int ctas = persistent_ctas(pgrid, kern, 8 * P, smem);                                              \
        if (ctas <= 0) return cudaErrorInvalidConfiguration;                                                     \
        Ld ld;                                                                                                   \
        ld.doms = doms; ld.items = items; ld.src = src; ld.tin = tin; ld.dst = dst; ld.tout = tout;              \
        kern<<<ctas < nitems ? ctas : nitems, 8 * P, smem, s>>>(ld, merges, nitems, err_flag);                   \
        return cudaGetLastError();                                                                               \
    }
    XB(0, 4) XB(1, 4) XB(0, 5) XB(1, 5)
#undef XB
    return cudaErrorInvalidConfiguration;
}

template cudaError_t launch_sweep_xytma<float>(int, const DomainView<float> &, const int *, CLayer<float>,
                                               CLayer<float>, Layer<float>, Layer<float>, const SweepConst<float> &,
                                               int, int, int, int *, cudaStream_t);
template cudaError_t launch_sweep_xytma<double>(int, const DomainView<double> &, const int *, CLayer<double>,
                                                CLayer<double>, Layer<double>, Layer<double>,
                                                const SweepConst<double> &, int, int, int, int *, cudaStream_t);

template cudaError_t launch_sweep_xycp<float>(int, const DomainView<float> &, CLayer<float>, CLayer<float>,
                                              Layer<float>, Layer<float>, const SweepConst<float> &, int, int, int *,
                                              cudaStream_t);
template cudaError_t launch_sweep_xycp<double>(int, const DomainView<double> &, CLayer<double>, CLayer<double>,
                                               Layer<double>, Layer<double>, const SweepConst<double> &, int, int,
                                               int *, cudaStream_t);
template cudaError_t launch_sweep_xy_batch<float>(int, int, const BatchDomain<float> *, const int2 *, int, int, int,
                                                  int, int, int, int *, cudaStream_t);
template cudaError_t launch_sweep_xy_batch<double>(int, int, const BatchDomain<double> *, const int2 *, int, int, int,
                                                   int, int, int, int *, cudaStream_t);

} // namespace adi
