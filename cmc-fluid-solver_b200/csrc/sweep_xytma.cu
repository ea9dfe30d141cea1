// X and Y sweeps fed by the Tensor Memory Accelerator.
//
// A CTA owns NLT = 8 or 16 neighbouring lines (consecutive k at one j for X, at
// one i for Y) over their whole length L = P K.  One thread issues the tile loads
// (cp.async.bulk.tensor, no multicast) into shared memory:
//   cur   U V W T           NLT x L each
//   temp  three fields      NLT x L each
//   temp  advecting field   WIDE x L (the lines plus a k halo of at least one
//                                     line, x start kept 16-byte aligned)
//   temp  advecting field   NLT x L at j+-1 (X) / i+-1 (Y), the other off-line axis
//   codes                   16 x L bytes (16-byte aligned k start)
// Out-of-range boxes (first/last lines of the grid) are zero-filled by the
// hardware.  The threads then build and solve exactly as the generic fast sweep
// (sweep_fast.cu: increment form, chunk elimination, cyclic reduction + PCR of the
// chunk boundary unknowns through shared memory), reading every input from the
// tiles.  Results go back into the tiles they replace and leave as eight TMA tile
// stores (next U V W T, nonlinear layer U V W T) issued by one thread; nodes the
// sweep does not change are stored with the value they hold (see the write-back).
//
// Thread t owns chunk c = t / NLT (rows c K .. c K + K - 1) of line t % NLT, so the
// lanes of a warp read the same row-in-chunk of 32 / NLT neighbouring chunks.  The
// tensor maps split the line coordinate into (row-in-chunk, chunk) so that tiles
// land as [i][c][lines]: those lanes then read 32 consecutive words, where the
// row-major [row][lines] layout put rows K apart into the same banks.
//
// The wait for the tile is bounded: if it has not landed after about a second the
// CTA raises the handle's error flag and leaves before writing anything.  With 8
// lines a CTA needs about 54 KB for 128-row lines (four CTAs per SM, so one CTA's
// tile wait overlaps the others' arithmetic); with 16 lines about 108 KB (two).
#include "adi_internal.cuh"
#include "sweep_common.cuh"

#include "tma.cuh"

#include <mutex>
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
// register cap follows from it and the shared-memory budget per CTA must allow it.
__host__ __device__ constexpr int xy_ctas_per_sm(int es, int K, int NLT)
{
    return es != 4 ? 1 : (K == 4 ? (NLT == 8 ? 3 : 1) : (K == 8 ? (NLT == 8 ? 4 : 2) : 1));
}

} // namespace

// P (chunks per line) is a template parameter so that every tile offset is an
// immediate.  The register cap lets as many CTAs be resident as their shared
// memory allows (xy_ctas_per_sm): FP32 K = 8 four of 8 lines or two of 16, K = 4
// three of 8 lines.
template <typename R, int DIR, int K, int NLT, int P>
__global__ void __launch_bounds__(NLT * P, xy_ctas_per_sm((int)sizeof(R), K, NLT))
    sweep_xytma_kernel(const __grid_constant__ XYMaps maps, DomainView<R> d, LineGeom g,
                       const int *__restrict__ line_lo, Layer<R> next, Layer<R> tout, SweepConst<R> kc, int merges,
                       int *err_flag)
{
    using T = XYTile<R, NLT>;
    constexpr int WIDE = T::WIDE, WOFF = T::WOFF;
    extern __shared__ __align__(128) unsigned char smem[];
    const int L = g.len;
    const int t = threadIdx.x;
    const int ch = t / NLT, li = t - ch * NLT;
    // CTA -> (outer index, k0): X lines j*nz + k, Y lines i*nz + k
    const int kblocks = g.nz / NLT;
    const int outer = blockIdx.x / kblocks;
    const int k0 = (blockIdx.x - outer * kblocks) * NLT;
    const int line = outer * g.nz + k0 + li;

    // tile layout ([K][P][width] each; every tile starts on a 128-byte boundary)
    const size_t plane = round128((size_t)L * NLT * sizeof(R));
    R *tcur = reinterpret_cast<R *>(smem);                            // [4] cur fields
    R *ttin = reinterpret_cast<R *>(smem + 4 * plane);                // [3] temp fields other than DIR
    R *twide = reinterpret_cast<R *>(smem + 7 * plane);               // temp DIR field, WIDE columns
    const size_t wide_bytes = round128((size_t)L * WIDE * sizeof(R));
    R *thm = reinterpret_cast<R *>(smem + 7 * plane + wide_bytes);    // temp DIR field at outer-1
    R *thp = reinterpret_cast<R *>(smem + 8 * plane + wide_bytes);    // temp DIR field at outer+1
    uint8_t *tcode = smem + 9 * plane + wide_bytes;                   // codes, 16 columns
    const size_t code_bytes = round128((size_t)L * 16);
    R *buf0 = reinterpret_cast<R *>(smem + 9 * plane + wide_bytes + code_bytes);
    R *buf1 = buf0 + (size_t)NLT * P * 8;
    uint64_t *bar = reinterpret_cast<uint64_t *>(buf1 + (size_t)NLT * P * 8);

    const bool has = line < g.nlines && line_lo[line] >= 0;
    if (!__syncthreads_or(has)) return;   // no segment in these lines

    if (t == 0) {
        tma::mbar_init(bar, 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    if (t == 0) {
        // every box delivers its full size (zero fill included): cur 4, temp 3,
        // off-line halo 2 planes, the wide advecting tile and the code tile
        const uint32_t bytes = (uint32_t)(9 * (size_t)L * NLT * sizeof(R) + (size_t)L * WIDE * sizeof(R) +
                                          (size_t)L * 16);
        tma::arrive_expect_tx(bar, bytes);
        // coordinates (innermost first): X {k, j, c, i}, Y {k, c, i, x}
        const int c1 = DIR == 0 ? outer : 0, c3 = DIR == 0 ? 0 : outer;
        for (int v = 0; v < 4; v++) {
            load_4d(tcur + v * (plane / sizeof(R)), &maps.cur[v], k0, c1, 0, c3, bar);
            if (v != DIR)
                load_4d(ttin + (v < DIR ? v : v - 1) * (plane / sizeof(R)), &maps.tin[v], k0, c1, 0, c3, bar);
        }
        load_4d(twide, &maps.fwide, k0 - WOFF, c1, 0, c3, bar);
        if (DIR == 0) {
            load_4d(thm, &maps.tin[DIR], k0, outer - 1, 0, 0, bar);
            load_4d(thp, &maps.tin[DIR], k0, outer + 1, 0, 0, bar);
        } else {
            load_4d(thm, &maps.tin[DIR], k0, 0, 0, outer - 1, bar);
            load_4d(thp, &maps.tin[DIR], k0, 0, 0, outer + 1, bar);
        }
        load_4d(tcode, &maps.code, k0 & ~15, c1, 0, c3, bar);   // byte tiles start 16-byte aligned
    }
    // Bounded wait (phase 0).  A thread whose wait gave up computes on whatever the
    // tile holds; the CTA checks every thread's wait at its first barrier and
    // leaves before writing anything.
    const bool tiles_ok = tma::mbar_wait(bar, 0, 1 << 17);

    // ---------------- rows from the tiles: one pass, 3-row window ----------------
    using namespace sweep;
    const int p0 = ch * K;
    const int fs = (int)(plane / sizeof(R));      // elements between two fields of a tile
    const int code_col = li + (k0 & 15);          // this line's byte in a code row
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
    // window slots: 0 = row i-1, 1 = row i, 2 = row i+1.  cur is kept only for IN
    // rows (the reference vector of the increment form is 0 elsewhere).
    R cw[3][4], tw[3][4];
    uint8_t kw[3];
#define XY_LOAD_ROW(SLOT_, I_)                                                                       \
    {                                                                                                \
        const int ii = (I_);                                                                         \
        const bool ok = has && (ii >= 0 || ch > 0) && (ii < K || ch + 1 < P);                        \
        const int tr = trow(ii);                                                                     \
        const uint8_t c = ok ? tcode[tr * 16 + code_col] : uint8_t(NODE_OUT);                       \
        kw[SLOT_] = c;                                                                               \
        const bool in = code_is_in(c);                                                               \
        _Pragma("unroll") for (int v = 0; v < 4; v++)                                                \
        {                                                                                            \
            tw[SLOT_][v] = ok ? (v == DIR ? wT[tr * WIDE] : tin_of(v)[tr * NLT]) : R(0);             \
            cw[SLOT_][v] = in ? cT[v * fs + tr * NLT] : R(0);                                        \
        }                                                                                            \
    }
    int kind[K];
    unsigned freebits = 0;
    R rr[K], dv[4][K];
    XY_LOAD_ROW(0, -1)
    XY_LOAD_ROW(1, 0)
    // global offset of this line's node 0: X (0, j, k) = j*nz + k; Y (i, 0, k) = i*ny*nz + k
    const long long lb = DIR == 0 ? (long long)outer * g.nz + k0 + li : (long long)outer * g.ny * g.nz + k0 + li;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int p = p0 + i;
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
            // no row: the node keeps its value in the destination, which comes into
            // the (never read) cur slot of the tile so that the tile store writes it back
            const long long off = lb + (long long)p * g.stride;
            const int tr = i * P + ch;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                dv[v][i] = R(0);
                tma::cp_async<sizeof(R)>(tcur + v * fs + tr * NLT + li, next.f[v] + off);
            }
        } else {
            // boundary row; BC_FREE moves the IN neighbour's cur to the right side
            const bool vf = (kw[1] & CODE_VEL_FREE) != 0, tf = (kw[1] & CODE_TEMP_FREE) != 0;
            const bool from_left = kd == R_END;   // IN neighbour at p-1, else at p+1
            const long long off = lb + (long long)p * g.stride;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const bool fr = v < 3 ? vf : tf;
                const R cn = from_left ? cw[0][v] : cw[2][v];
                dv[v][i] = fr ? cn : (kc.nv_in_temp ? tw[1][v] : __ldg(d.nv[v] + off));
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
    tma::cp_async_commit();

    // ---------------- chunk elimination ----------------
    R ea[2][K], ec[2][K];
    Reduced<R> red;
    eliminate<R, K>(kind, rr, freebits, kc, dv, ea, ec, red);

    // ---------------- reduced system: one CR step + PCR through shared slots ----------------
    // Couplings to rows outside the line are exactly zero (the first row of a line
    // has a = 0, the last c = 0, and PCR keeps them zero), so a thread whose partner
    // row would lie outside reads its own slot instead: finite values times 0.
    R *const s0 = buf0 + li * 8, *const s1 = buf1 + li * 8;
    const int cs = NLT * 8;   // elements between the slots of two chunks
    slot_store<R>(s0 + ch * cs, red.Al[0], red.Cl[0], red.Al[1], red.Cl[1], red.Dl[0], red.Dl[1], red.Dl[2],
                  red.Dl[3]);
    if (__syncthreads_or(!tiles_ok)) {
        tma::cp_async_wait_all();
        if (t == 0) {
            atomicExch(err_flag, 1);
            tma::mbar_wait(bar, 0, 1 << 10);   // copies still in flight
        }
        return;
    }
    R ea_[2], ec_[2], ed[4];
    {
        R pv[8];
        slot_load<R>(s0 + (ch > 0 ? ch - 1 : ch) * cs, pv);
        if (ch == 0) {
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = R(0);
        }
        cr_step<R>(red, pv, ea_, ec_, ed);
    }
    int nstep = 0;
    for (int st = 1; st < P; st <<= 1, nstep++) {
        R *const bw = (nstep & 1) ? s0 : s1;
        slot_store<R>(bw + ch * cs, ea_[0], ec_[0], ea_[1], ec_[1], ed[0], ed[1], ed[2], ed[3]);
        __syncthreads();
        R mv[8], pv[8];
        slot_load<R>(bw + (ch - st >= 0 ? ch - st : ch) * cs, mv);
        slot_load<R>(bw + (ch + st < P ? ch + st : ch) * cs, pv);
        pcr_update<R>(mv, pv, ea_, ec_, ed);
    }
    R *const bx = (nstep & 1) ? s0 : s1;
    slot_store<R>(bx + ch * cs, ed[0], ed[1], ed[2], ed[3], R(0), R(0), R(0), R(0));
    __syncthreads();
    R xf[4], xl[4];
    {
        R nf[8];
        slot_load<R>(bx + (ch + 1 < P ? ch + 1 : ch) * cs, nf);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            xf[v] = ed[v];
            const int m = v < 3 ? 0 : 1;
            xl[v] = red.Dl[v] - red.Al[m] * xf[v] - red.Cl[m] * nf[v];   // Cl = 0 on the last chunk
        }
    }
    // ---------------- write-back through the tiles ----------------
    // Each thread overwrites its own rows (nobody reads them any more): cur slots
    // with the new values, the temp slots with the merged nonlinear layer (the DIR
    // field goes to the outer-1 halo tile, whose rows are free now).  Nodes that
    // are not IN keep the input temp value, which the output buffer holds too (both
    // nonlinear buffers start each step as copies of cur, and sweeps write only IN
    // nodes), and rows without a matrix row already hold the destination's value;
    // so the whole tile can be stored.
    if constexpr (sizeof(R) == 4) {
        // packed FP32: fields (U, T) and (V, W) two at a time, as the elimination left them
        const float2 xf03 = p2(xf[0], xf[3]), xf12 = p2(xf[1], xf[2]);
        const float2 xl03 = p2(xl[0], xl[3]), xl12 = p2(xl[1], xl[2]);
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int kd = kind[i];
            const int tr = i * P + ch;
            if (kd != R_IN) thm[tr * NLT + li] = wT[tr * WIDE];
            if (kd == R_NONE) continue;
            float2 x03, x12;
            if (i == 0) { x03 = xf03; x12 = xf12; }
            else if (i == K - 1) { x03 = xl03; x12 = xl12; }
            else {
                const float2 nea = p2(-ea[0][i], -ea[1][i]), nec = p2(-ec[0][i], -ec[1][i]);
                x03 = fma2(nec, xl03, fma2(nea, xf03, p2(dv[0][i], dv[3][i])));
                x12 = fma2(bc2(nec.x), xl12, fma2(bc2(nea.x), xf12, p2(dv[1][i], dv[2][i])));
            }
            R *const c0 = tcur + tr * NLT + li;
            if (kd == R_IN) {
                x03 = add2(x03, p2(c0[0], c0[3 * fs]));
                x12 = add2(x12, p2(c0[fs], c0[2 * fs]));
                auto tv = [&](int v) -> R { return v == DIR ? wT[tr * WIDE] : tin_of(v)[tr * NLT]; };
                float2 m03 = mul2(add2(p2(tv(0), tv(3)), x03), bc2(0.5f));
                float2 m12 = mul2(add2(p2(tv(1), tv(2)), x12), bc2(0.5f));
                if (merges == 2) {
                    m03 = mul2(add2(m03, x03), bc2(0.5f));
                    m12 = mul2(add2(m12, x12), bc2(0.5f));
                }
                const float mm[4] = {m03.x, m12.x, m12.y, m03.y};
#pragma unroll
                for (int v = 0; v < 4; v++) (v == DIR ? thm : ttin + (v < DIR ? v : v - 1) * fs)[tr * NLT + li] = mm[v];
            }
            c0[0] = x03.x;
            c0[fs] = x12.x;
            c0[2 * fs] = x12.y;
            c0[3 * fs] = x03.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int kd = kind[i];
            const int tr = i * P + ch;
            if (kd != R_IN) thm[tr * NLT + li] = wT[tr * WIDE];
            if (kd == R_NONE) continue;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const int m = v < 3 ? 0 : 1;
                R x = i == 0 ? xf[v] : (i == K - 1 ? xl[v] : dv[v][i] - ea[m][i] * xf[v] - ec[m][i] * xl[v]);
                R *const cslot = tcur + v * fs + tr * NLT + li;
                if (kd == R_IN) {
                    x += *cslot;
                    const R tv = v == DIR ? wT[tr * WIDE] : tin_of(v)[tr * NLT];
                    R mm = (tv + x) * R(0.5);
                    if (merges == 2) mm = (mm + x) * R(0.5);
                    (v == DIR ? thm : ttin + (v < DIR ? v : v - 1) * fs)[tr * NLT + li] = mm;
                }
                *cslot = x;
            }
        }
    }
    tma::cp_async_wait_all();
    tma::fence_proxy_async();
    __syncthreads();
    if (t == 0) {
        const int c1 = DIR == 0 ? outer : 0, c3 = DIR == 0 ? 0 : outer;
        for (int v = 0; v < 4; v++) {
            tma::store_4d(&maps.next[v], tcur + v * fs, k0, c1, 0, c3);
            tma::store_4d(&maps.tout[v], v == DIR ? thm : ttin + (v < DIR ? v : v - 1) * fs, k0, c1, 0, c3);
        }
        tma::bulk_commit();
        tma::bulk_wait_read();
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

// Encodes (or finds in the cache) a map of the given rank, dims, strides and box.
bool encode_cached(CUtensorMap *m, const MapKey &key, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                   const cuuint32_t *box)
{
    struct Ent {
        MapKey k;
        CUtensorMap m;
    };
    static std::vector<Ent> cache;
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> g(mu);
        for (const Ent &e : cache)
            if (e.k == key) { *m = e.m; return true; }
    }
    auto enc = get_encoder_fn();
    if (!enc) return false;
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(m, (CUtensorMapDataType)key.dt, rank, const_cast<void *>(key.base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    std::lock_guard<std::mutex> g(mu);
    if (cache.size() > 4096) cache.clear();
    cache.push_back({key, *m});
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
    using T = XYTile<R, NLT>;
    const size_t plane = round128((size_t)L * NLT * sizeof(R));
    return 9 * plane + round128((size_t)L * T::WIDE * sizeof(R)) + round128((size_t)L * 16) +
           2 * (size_t)NLT * P * 8 * sizeof(R) + 16 /* mbarrier */;
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
    if (P != 4 && P != 8 && P != 16 && !(P == 32 && K == 4)) return false;   // compiled chunk counts
    const int threads = nlt * P;
    if (threads < 32 || threads > 512) return false;
    // the CTAs per SM the shape is compiled for (228 KB per SM, 1 KB reserved per CTA)
    const size_t budget = 228 * 1024 / xy_ctas_per_sm(elem_bytes, K, nlt) - 1024;
    return xytma_smem_bytes(L, P, nlt, elem_bytes) <= (budget < 227 * 1024 ? budget : 227 * 1024);
}

template <typename R>
cudaError_t launch_sweep_xytma(int dir, const DomainView<R> &d, const int *line_lo, CLayer<R> cur, CLayer<R> tin,
                               Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges, int K, int nlt,
                               int *err_flag, cudaStream_t s)
{
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
    for (int v = 0; v < 4; v++) {
        if (!make_chunk_map(&maps.next[v], next.f[v], dir, d.nx, d.ny, d.nz, nlt, K, es, dt, K))
            return cudaErrorInvalidValue;
        if (!make_chunk_map(&maps.tout[v], tout.f[v], dir, d.nx, d.ny, d.nz, nlt, K, es, dt, K))
            return cudaErrorInvalidValue;
    }
    const size_t smem = xytma_smem_bytes(L, P, nlt, es);
    const int blocks = (dir == 0 ? d.ny : d.nx) * (d.nz / nlt);
    const int threads = nlt * P;
#define XL(DD, KK, NN, PP)                                                                                       \
    if (dir == DD && K == KK && nlt == NN && P == PP) {                                                          \
        auto kern = sweep_xytma_kernel<R, DD, KK, NN, PP>;                                                       \
        static SmemOptIn opt_in;                                                                                 \
        cudaError_t e = ensure_dynamic_smem(opt_in, kern, smem);                                                 \
        if (e != cudaSuccess) return e;                                                                          \
        kern<<<blocks, threads, smem, s>>>(maps, d, g, line_lo, next, tout, k, merges, err_flag);                \
        return cudaGetLastError();                                                                               \
    }
#define XLP(DD, KK, NN) XL(DD, KK, NN, 4) XL(DD, KK, NN, 8) XL(DD, KK, NN, 16)
    XLP(0, 8, 8) XLP(0, 16, 8) XLP(1, 8, 8) XLP(1, 16, 8)
    XLP(0, 8, 16) XLP(0, 16, 16) XLP(1, 8, 16) XLP(1, 16, 16)
    XLP(0, 4, 8) XLP(1, 4, 8) XLP(0, 4, 16) XLP(1, 4, 16)
    XL(0, 4, 8, 32) XL(1, 4, 8, 32) XL(0, 4, 16, 32) XL(1, 4, 16, 32)
#undef XLP
#undef XL
    return cudaErrorInvalidConfiguration;
}

template cudaError_t launch_sweep_xytma<float>(int, const DomainView<float> &, const int *, CLayer<float>,
                                               CLayer<float>, Layer<float>, Layer<float>, const SweepConst<float> &,
                                               int, int, int, int *, cudaStream_t);
template cudaError_t launch_sweep_xytma<double>(int, const DomainView<double> &, const int *, CLayer<double>,
                                                CLayer<double>, Layer<double>, Layer<double>,
                                                const SweepConst<double> &, int, int, int, int *, cudaStream_t);

} // namespace adi
