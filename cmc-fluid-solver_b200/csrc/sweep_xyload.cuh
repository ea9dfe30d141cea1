// Tile loaders of the X/Y sweep (sweep_xytma.cu).
//
// The sweep kernel works on tiles: NLT neighbouring lines (consecutive k at one j
// for X, at one i for Y) over their whole length, laid out in shared memory
// chunk-major ([row-in-chunk][chunk][line], sweep_xytma.cu).  How a tile gets there
// is the loader's business:
//   XYTmaLoader      one thread issues cp.async.bulk.tensor boxes (no multicast)
//                    completing on an mbarrier; needs nz a multiple of 16 and line
//                    lengths of exactly P K rows (the tensor maps' 16-byte rules).
//   XYCpLoader       every thread issues element-wise cp.async copies: any nz and
//                    any line length up to P K (rows past the line and lines past
//                    nz are padding with NODE_OUT codes, so they hold no matrix row).
//   XYBatchLoader    the same copies for the tiles of many domains of a batch
//                    (work items (domain, tile)), each with its own geometry,
//                    layers and sweep constants.
// Each loader also gives the kernel the per-tile context: where the tile's lines
// start in global memory, the destination layers, the node values and the sweep
// constants.
#pragma once

#include "adi_internal.cuh"
#include "tma.cuh"

namespace adi {

// Shared-memory tile of one X/Y launch.
template <typename R>
struct XYSmem {
    R *tcur;        // [4] cur fields, chunk-major
    R *ttin;        // [3] temp fields other than DIR
    R *twide;       // temp DIR field, WIDE columns (the lines plus a k halo)
    R *thm, *thp;   // temp DIR field at outer - 1 / outer + 1
    uint8_t *tcode; // codes, 16 columns per row
    uint64_t *bar;  // mbarrier (TMA loader)
};

// Where one tile's lines lie in global memory.  The solve reaches the rest of what
// it needs (sweep constants, node values, destination layers) through the loader's
// accessors, which read kernel parameters (one domain) or the tile's domain record
// (a batch) when used, so none of it is held in registers.
struct XYTileGeo {
    long long lb0;      // global offset of node 0 of the tile's line 0
    long long stride;   // element stride along the lines
    int code_off;       // column of line 0 in a code row of the tile
    int dom;            // domain of the tile (a batch's work item), else 0
};

namespace xyload {

// offsets of an X / Y line (outer index o, first line k0) in a [nx][ny][nz] array
template <int DIR>
__device__ __forceinline__ void line_axes(int ny, int nz, long long &sline, long long &souter)
{
    sline = DIR == 0 ? (long long)ny * nz : (long long)nz;    // along the line
    souter = DIR == 0 ? (long long)nz : (long long)ny * nz;   // along the outer axis (j for X, i for Y)
}

// Element-wise copies of one tile into the shared-memory layout (all threads of
// the CTA; cp.async, committed as one group).  Thread t = c NLT + l copies its own
// rows -- rows c K .. c K + K - 1 of line l -- of every plane, so its source offsets
// are one base plus multiples of the line stride and its destinations are
// consecutive words across the CTA; the two threads at the tile's sides also copy
// the k-halo columns of the advecting field.  L real rows, lines k0.. up to nz;
// other slots are zero (fields) or NODE_OUT (codes).  The codes are read into
// registers (K bytes per thread) and written to the tile by store_codes once the
// copies have landed, so the byte loads' latency passes while the CTA solves.
template <typename R, int DIR, int K, int NLT, int P, int WIDE, int WOFF>
__device__ __forceinline__ uint64_t issue_tile(const XYSmem<R> &sm, int fs, int t, const R *const *cur,
                                               const R *const *tin, const uint8_t *code, int ny, int nz,
                                               int n_outer, int L, int outer, int k0)
{
    constexpr int NT = NLT * P;
    long long sline, souter;
    line_axes<DIR>(ny, nz, sline, souter);
    const int ch = t / NLT, li = t - ch * NLT;
    const long long off0 = (long long)outer * souter + k0 + li + (long long)(ch * K) * sline;
    const bool line_ok = k0 + li < nz;
    const bool has_m = outer > 0, has_p = outer + 1 < n_outer;
    const int nrow = L - ch * K;   // rows of this chunk inside the line: i < nrow
#pragma unroll
    for (int i = 0; i < K; i++) {
        const bool ok = line_ok && i < nrow;
        const long long o = off0 + i * sline;
        const int q = t + i * NT;   // tile slot (i P + c) NLT + l
#pragma unroll
        for (int v = 0; v < 4; v++) {
            R *const dc = sm.tcur + v * fs + q;
            if (ok) tma::cp_async<sizeof(R)>(dc, cur[v] + o);
            else *dc = R(0);
            if (v == DIR) continue;
            R *const dt = sm.ttin + (v < DIR ? v : v - 1) * fs + q;
            if (ok) tma::cp_async<sizeof(R)>(dt, tin[v] + o);
            else *dt = R(0);
        }
        R *const dm = sm.thm + q, *const dp = sm.thp + q;
        if (ok && has_m) tma::cp_async<sizeof(R)>(dm, tin[DIR] + o - souter);
        else *dm = R(0);
        if (ok && has_p) tma::cp_async<sizeof(R)>(dp, tin[DIR] + o + souter);
        else *dp = R(0);
        // the advecting field with its k halo: own column, and the side columns
        R *const dw = sm.twide + (i * P + ch) * WIDE + WOFF + li;
        if (ok) tma::cp_async<sizeof(R)>(dw, tin[DIR] + o);
        else *dw = R(0);
        if (li == 0) {
            if (i < nrow && k0 > 0 && k0 - 1 < nz) tma::cp_async<sizeof(R)>(dw - 1, tin[DIR] + o - 1);
            else dw[-1] = R(0);
        }
        if (li == NLT - 1) {
            if (i < nrow && k0 + NLT < nz) tma::cp_async<sizeof(R)>(dw + 1, tin[DIR] + o + 1);
            else dw[1] = R(0);
        }
    }
    tma::cp_async_commit();
    uint64_t pack = 0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const uint8_t cd = (line_ok && i < nrow) ? __ldg(code + off0 + i * sline) : uint8_t(NODE_OUT);
        pack |= (uint64_t)cd << (8 * i);
    }
    return pack;
}

template <int K, int NLT, int P>
__device__ __forceinline__ void store_codes(uint8_t *tcode, int t, uint64_t pack)
{
    const int ch = t / NLT, li = t - ch * NLT;
#pragma unroll
    for (int i = 0; i < K; i++) tcode[(i * P + ch) * 16 + li] = (uint8_t)(pack >> (8 * i));
}

} // namespace xyload

// ---- TMA boxes (single domain, aligned dims) ----
template <typename R, int DIR, int K, int NLT, int P, int WIDE, int WOFF>
struct XYTmaLoader {
    XYMaps maps;
    DomainView<R> d;
    Layer<R> next, tout;
    SweepConst<R> kc;
    int kblocks;   // tiles per outer index

    static constexpr bool kTma = true;
    __device__ __forceinline__ void init(const XYSmem<R> &sm, int t) const
    {
        if (t == 0) {
            tma::mbar_init(sm.bar, 1);
            tma::fence_barrier_init();
        }
    }
    // Thread 0 issues the boxes; every box delivers its full size (zero fill
    // included): cur 4, temp 3, off-line halo 2 planes, the wide advecting tile and
    // the code tile.
    __device__ __forceinline__ uint64_t issue(int tile, const XYSmem<R> &sm, int fs, int t) const
    {
        if (t != 0 || kc.skip_tile_loads) return 0;   // fault injection: the tile never arrives
        constexpr int L = P * K;
        const int outer = tile / kblocks;
        const int k0 = (tile - outer * kblocks) * NLT;
        constexpr uint32_t bytes =
            (uint32_t)(9 * (size_t)L * NLT * sizeof(R) + (size_t)L * WIDE * sizeof(R) + (size_t)L * 16);
        tma::arrive_expect_tx(sm.bar, bytes);
        // coordinates (innermost first): X {k, j, c, i}, Y {k, c, i, x}
        const int c1 = DIR == 0 ? outer : 0, c3 = DIR == 0 ? 0 : outer;
        for (int v = 0; v < 4; v++) {
            tma::load_4d(sm.tcur + v * fs, &maps.cur[v], k0, c1, 0, c3, sm.bar);
            if (v != DIR) tma::load_4d(sm.ttin + (v < DIR ? v : v - 1) * fs, &maps.tin[v], k0, c1, 0, c3, sm.bar);
        }
        tma::load_4d(sm.twide, &maps.fwide, k0 - WOFF, c1, 0, c3, sm.bar);
        if (DIR == 0) {
            tma::load_4d(sm.thm, &maps.tin[DIR], k0, outer - 1, 0, 0, sm.bar);
            tma::load_4d(sm.thp, &maps.tin[DIR], k0, outer + 1, 0, 0, sm.bar);
        } else {
            tma::load_4d(sm.thm, &maps.tin[DIR], k0, 0, 0, outer - 1, sm.bar);
            tma::load_4d(sm.thp, &maps.tin[DIR], k0, 0, 0, outer + 1, sm.bar);
        }
        tma::load_4d(sm.tcode, &maps.code, k0 & ~15, c1, 0, c3, sm.bar);   // byte tiles start 16-byte aligned
        return 0;
    }
    // Bounded wait (phase it & 1).  A thread whose wait gave up computes on whatever
    // the tile holds; the CTA checks every thread's wait at its release barrier.
    __device__ __forceinline__ bool wait(int it, const XYSmem<R> &sm, int, uint64_t) const
    {
        return tma::mbar_wait(sm.bar, it & 1, kc.tile_wait_tries);
    }
    // After a wait that gave up: thread 0 waits, bounded, for copies still in flight
    // (none when the loads were never issued).
    __device__ __forceinline__ void abandon(int it, const XYSmem<R> &sm, int t) const
    {
        if (t == 0) tma::mbar_wait(sm.bar, it & 1, kc.tile_wait_tries < (1 << 10) ? kc.tile_wait_tries : 1 << 10);
    }
    __device__ __forceinline__ XYTileGeo geo(int tile) const
    {
        XYTileGeo g;
        const int outer = tile / kblocks;
        const int k0 = (tile - outer * kblocks) * NLT;
        g.lb0 = DIR == 0 ? (long long)outer * d.nz + k0 : (long long)outer * d.ny * d.nz + k0;
        g.stride = DIR == 0 ? (long long)d.ny * d.nz : (long long)d.nz;
        g.code_off = k0 & 15;
        g.dom = 0;
        return g;
    }
    __device__ __forceinline__ const SweepConst<R> &consts(const XYTileGeo &) const { return kc; }
    __device__ __forceinline__ const R *nv(const XYTileGeo &, int v) const { return d.nv[v]; }
    __device__ __forceinline__ R *nextp(const XYTileGeo &, int v) const { return next.f[v]; }
    __device__ __forceinline__ R *toutp(const XYTileGeo &, int v) const { return tout.f[v]; }
};

// ---- element-wise copies, one domain (any nz, lines up to P K rows) ----
template <typename R, int DIR, int K, int NLT, int P, int WIDE, int WOFF>
struct XYCpLoader {
    CLayer<R> cur, tin;
    DomainView<R> d;
    Layer<R> next, tout;
    SweepConst<R> kc;
    int kblocks;   // tiles per outer index: ceil(nz / NLT)
    int L;         // rows of a line

    static constexpr bool kTma = false;
    __device__ __forceinline__ void init(const XYSmem<R> &, int) const {}
    __device__ __forceinline__ uint64_t issue(int tile, const XYSmem<R> &sm, int fs, int t) const
    {
        const int outer = tile / kblocks;
        const int k0 = (tile - outer * kblocks) * NLT;
        return xyload::issue_tile<R, DIR, K, NLT, P, WIDE, WOFF>(sm, fs, t, cur.f, tin.f, d.code, d.ny, d.nz,
                                                                DIR == 0 ? d.ny : d.nx, L, outer, k0);
    }
    __device__ __forceinline__ bool wait(int, const XYSmem<R> &sm, int t, uint64_t codes) const
    {
        tma::cp_async_wait_all();
        xyload::store_codes<K, NLT, P>(sm.tcode, t, codes);
        __syncthreads();
        return true;
    }
    __device__ __forceinline__ void abandon(int, const XYSmem<R> &, int) const {}
    __device__ __forceinline__ XYTileGeo geo(int tile) const
    {
        XYTileGeo g;
        const int outer = tile / kblocks;
        const int k0 = (tile - outer * kblocks) * NLT;
        g.lb0 = DIR == 0 ? (long long)outer * d.nz + k0 : (long long)outer * d.ny * d.nz + k0;
        g.stride = DIR == 0 ? (long long)d.ny * d.nz : (long long)d.nz;
        g.code_off = 0;
        g.dom = 0;
        return g;
    }
    __device__ __forceinline__ const SweepConst<R> &consts(const XYTileGeo &) const { return kc; }
    __device__ __forceinline__ const R *nv(const XYTileGeo &, int v) const { return d.nv[v]; }
    __device__ __forceinline__ R *nextp(const XYTileGeo &, int v) const { return next.f[v]; }
    __device__ __forceinline__ R *toutp(const XYTileGeo &, int v) const { return tout.f[v]; }
};

// ---- element-wise copies, the tiles of all domains of a batch ----
// Work item q = (domain, tile of that domain); layer roles are indices into each
// domain's five layers, the same for the whole batch.
template <typename R, int DIR, int K, int NLT, int P, int WIDE, int WOFF>
struct XYBatchLoader {
    const BatchDomain<R> *doms;
    const int2 *items;
    int src, tin, dst, tout;

    static constexpr bool kTma = false;
    __device__ __forceinline__ void init(const XYSmem<R> &, int) const {}
    __device__ __forceinline__ void where(int q, const BatchDomain<R> *&bd, int &outer, int &k0) const
    {
        const int2 w = items[q];
        bd = doms + w.x;
        const int kb = (bd->d.nz + NLT - 1) / NLT;
        outer = w.y / kb;
        k0 = (w.y - outer * kb) * NLT;
    }
    __device__ __forceinline__ uint64_t issue(int q, const XYSmem<R> &sm, int fs, int t) const
    {
        const BatchDomain<R> *bd;
        int outer, k0;
        where(q, bd, outer, k0);
        const int nx = bd->d.nx, ny = bd->d.ny, nz = bd->d.nz;
        return xyload::issue_tile<R, DIR, K, NLT, P, WIDE, WOFF>(sm, fs, t, bd->L[src], bd->L[tin], bd->d.code, ny, nz,
                                                                DIR == 0 ? ny : nx, DIR == 0 ? nx : ny, outer, k0);
    }
    __device__ __forceinline__ bool wait(int, const XYSmem<R> &sm, int t, uint64_t codes) const
    {
        tma::cp_async_wait_all();
        xyload::store_codes<K, NLT, P>(sm.tcode, t, codes);
        __syncthreads();
        return true;
    }
    __device__ __forceinline__ void abandon(int, const XYSmem<R> &, int) const {}
    __device__ __forceinline__ XYTileGeo geo(int q) const
    {
        const BatchDomain<R> *bd;
        int outer, k0;
        where(q, bd, outer, k0);
        XYTileGeo g;
        const long long ny = bd->d.ny, nz = bd->d.nz;
        g.lb0 = DIR == 0 ? (long long)outer * nz + k0 : (long long)outer * ny * nz + k0;
        g.stride = DIR == 0 ? ny * nz : nz;
        g.code_off = 0;
        g.dom = items[q].x;
        return g;
    }
    __device__ __forceinline__ const SweepConst<R> &consts(const XYTileGeo &g) const { return doms[g.dom].kc[DIR]; }
    __device__ __forceinline__ const R *nv(const XYTileGeo &g, int v) const { return doms[g.dom].d.nv[v]; }
    __device__ __forceinline__ R *nextp(const XYTileGeo &g, int v) const { return doms[g.dom].L[dst][v]; }
    __device__ __forceinline__ R *toutp(const XYTileGeo &g, int v) const { return doms[g.dom].L[tout][v]; }
};

} // namespace adi
