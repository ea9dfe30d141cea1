// X and Y sweeps fed by the Tensor Memory Accelerator.
//
// A CTA owns NL = 16 neighbouring lines (16 consecutive k at one j for X, at one i
// for Y) over their whole length L.  One thread issues the tile loads
// (cp.async.bulk.tensor, no multicast) into shared memory:
//   cur   U V W T           16 x L each
//   temp  three fields      16 x L each
//   temp  advecting field   24 x L (k0-4 .. k0+19: the lines plus the k+-1 halo,
//                                   x start kept 16-byte aligned)
//   temp  advecting field   16 x L at j+-1 (X) / i+-1 (Y), the other off-line axis
//   codes                   16 x L bytes
// Out-of-range boxes (first/last lines of the grid) are zero-filled by the
// hardware.  The threads then build and solve exactly as the generic fast sweep
// (sweep_fast.cu: increment form, chunk elimination, cyclic reduction + PCR of the
// chunk boundary unknowns through shared memory), reading every input from the
// tiles, and store results straight to global memory (lanes run along k, so
// each warp store covers two 64-byte runs).
//
// The tile arrives as up to four boxes along the line, each on its own mbarrier,
// and a thread waits only for the boxes its rows need.  Every wait is bounded: if
// a box has not landed after about a second the CTA raises the handle's error flag
// and leaves before writing anything.
#include "adi_internal.cuh"
#include "sweep_common.cuh"

#include "tma.cuh"

#include <mutex>
#include <vector>

namespace adi {

using tma::smem_u32;
using tma::load_3d;

namespace {
constexpr int NLT = 16;   // lines per CTA
constexpr int WIDE = 24;  // width of the advecting-field tile (k0-4 .. k0+19)
} // namespace

template <typename R, int DIR, int K>
__global__ void __launch_bounds__(256)
    sweep_xytma_kernel(const __grid_constant__ XYMaps maps, DomainView<R> d, LineGeom g, int P, int Lb, int nbox,
                       const int *__restrict__ line_lo, Layer<R> next, Layer<R> tout, SweepConst<R> kc, int merges,
                       int *err_flag)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int L = g.len;
    const int t = threadIdx.x;
    const int ch = t / NLT, li = t - ch * NLT;
    // CTA -> (outer index, k0): X lines j*nz + k, Y lines i*nz + k
    const int kblocks = g.nz / NLT;
    const int outer = blockIdx.x / kblocks;
    const int k0 = (blockIdx.x - outer * kblocks) * NLT;
    const int line = outer * g.nz + k0 + li;

    // tile layout (L even, so every tile starts on a 128-byte boundary)
    const size_t plane = (size_t)L * NLT * sizeof(R);
    R *tcur = reinterpret_cast<R *>(smem);                       // [4][L][16]
    R *ttin = reinterpret_cast<R *>(smem + 4 * plane);            // [3][L][16]: the fields other than DIR
    R *twide = reinterpret_cast<R *>(smem + 7 * plane);           // [L][24]
    const size_t wide_bytes = ((size_t)L * WIDE * sizeof(R) + 127) / 128 * 128;
    R *thm = reinterpret_cast<R *>(smem + 7 * plane + wide_bytes);               // [L][16] at outer-1
    R *thp = reinterpret_cast<R *>(smem + 8 * plane + wide_bytes);               // [L][16] at outer+1
    uint8_t *tcode = smem + 9 * plane + wide_bytes;                               // [L][16]
    const size_t code_bytes = ((size_t)L * NLT + 127) / 128 * 128;
    R *buf0 = reinterpret_cast<R *>(smem + 9 * plane + wide_bytes + code_bytes);
    R *buf1 = buf0 + (size_t)NLT * P * 8;
    uint64_t *bar = reinterpret_cast<uint64_t *>(buf1 + (size_t)NLT * P * 8);   // one per box along the line

    const bool has = line < g.nlines && line_lo[line] >= 0;
    if (!__syncthreads_or(has)) return;   // no segment in these 16 lines

    if (t == 0) {
        for (int b = 0; b < nbox; b++) tma::mbar_init(&bar[b], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    if (t == 0) {
        // every box delivers its full size (zero fill included): cur 4, temp 3,
        // off-line halo 2 planes, the wide advecting tile and the code tile
        const uint32_t bytes = (uint32_t)(9 * (size_t)Lb * NLT * sizeof(R) + (size_t)Lb * WIDE * sizeof(R) +
                                          (size_t)Lb * NLT);
        for (int b = 0; b < nbox; b++) {
            uint64_t *bb = &bar[b];
            tma::arrive_expect_tx(bb, bytes);
            const int p0 = b * Lb;
            const size_t po = (size_t)p0 * NLT;        // row offset inside a [L][16] tile
            // coordinates (innermost first): X {k, j, x}, Y {k, y, i}
            const int c1 = DIR == 0 ? outer : p0, c2 = DIR == 0 ? p0 : outer;
            for (int v = 0; v < 4; v++) {
                load_3d(tcur + v * (plane / sizeof(R)) + po, &maps.cur[v], k0, c1, c2, bb);
                if (v != DIR)
                    load_3d(ttin + (v < DIR ? v : v - 1) * (plane / sizeof(R)) + po, &maps.tin[v], k0, c1, c2, bb);
            }
            load_3d(twide + (size_t)p0 * WIDE, &maps.fwide, k0 - 4, c1, c2, bb);
            if (DIR == 0) {
                load_3d(thm + po, &maps.tin[DIR], k0, outer - 1, p0, bb);
                load_3d(thp + po, &maps.tin[DIR], k0, outer + 1, p0, bb);
            } else {
                load_3d(thm + po, &maps.tin[DIR], k0, p0, outer - 1, bb);
                load_3d(thp + po, &maps.tin[DIR], k0, p0, outer + 1, bb);
            }
            load_3d(tcode + po, &maps.code, k0, c1, c2, bb);
        }
    }
    // Bounded waits (phase 0) for just the boxes holding this thread's rows and
    // their +-1 neighbours, so chunks near the start of the line begin while the
    // rest of the tile is still landing.  A thread whose wait gave up computes on
    // whatever the tile holds; the CTA checks every thread's wait at its first
    // barrier and leaves before writing anything.
    bool tiles_ok = true;
    {
        const int rlo = ch * K > 0 ? ch * K - 1 : 0;
        const int rhi = ch * K + K < L ? ch * K + K : L - 1;
        for (int b = rlo / Lb; b <= rhi / Lb; b++) tiles_ok &= tma::mbar_wait(&bar[b], 0, 1 << 17);
    }

    // ---------------- rows from the tiles: one pass, 3-row window ----------------
    using namespace sweep;
    const int p0 = ch * K;
    const int fs = L * NLT;                       // elements between two fields of a tile
    const R *__restrict__ cT = tcur + li;         // cur tile column of this line
    const R *__restrict__ tT = ttin + li;         // temp tiles (fields other than DIR)
    const R *__restrict__ wT = twide + li + 4;    // advecting field column (k halo at -1/+1)
    const R *__restrict__ hmT = thm + li;
    const R *__restrict__ hpT = thp + li;
    const uint8_t *__restrict__ kT = tcode + li;
    // window slots: 0 = row i-1, 1 = row i, 2 = row i+1.  cur is kept only for IN
    // rows (the reference vector of the increment form is 0 elsewhere).
    R cw[3][4], tw[3][4];
    uint8_t kw[3];
#define XY_LOAD_ROW(SLOT_, P_)                                                                       \
    {                                                                                                \
        const int pp = (P_);                                                                         \
        const bool ok = has && pp >= 0 && pp < L;                                                    \
        const uint8_t c = ok ? kT[pp * NLT] : uint8_t(NODE_OUT);                                     \
        kw[SLOT_] = c;                                                                               \
        const bool in = code_is_in(c);                                                               \
        _Pragma("unroll") for (int v = 0; v < 4; v++)                                                \
        {                                                                                            \
            tw[SLOT_][v] = ok ? (v == DIR ? wT[pp * WIDE] : tT[(v < DIR ? v : v - 1) * fs + pp * NLT]) : R(0); \
            cw[SLOT_][v] = in ? cT[v * fs + pp * NLT] : R(0);                                        \
        }                                                                                            \
    }
    int kind[K];
    unsigned freebits = 0;
    R rr[K], dv[4][K];
    XY_LOAD_ROW(0, p0 - 1)
    XY_LOAD_ROW(1, p0)
    // global offset of this line's node 0: X (0, j, k) = j*nz + k; Y (i, 0, k) = i*ny*nz + k
    const long long lb = DIR == 0 ? (long long)outer * g.nz + k0 + li : (long long)outer * g.ny * g.nz + k0 + li;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int p = p0 + i;
        XY_LOAD_ROW(2, p + 1)
        const int kd = row_kind(code_is_in(kw[0]), code_is_in(kw[1]), code_is_in(kw[2]));
        kind[i] = kd;
        if (kw[1] & CODE_VEL_FREE) freebits |= 1u << (2 * i);
        if (kw[1] & CODE_TEMP_FREE) freebits |= 2u << (2 * i);
        rr[i] = R(0);
        if (kd == R_IN) {
            // IN rows are never the first or last node of a line
            const R r = tw[1][DIR] * kc.inv_two_h;
            rr[i] = r;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const R vis = v < 3 ? kc.vis_v : kc.vis_t;
                dv[v][i] = vis * (cw[0][v] - R(2) * cw[1][v] + cw[2][v]) - r * (cw[2][v] - cw[0][v]);
            }
            dv[DIR][i] -= kc.v_T * ((tw[2][3] - tw[0][3]) * kc.inv_two_h);
            const R fa = (tw[2][0] - tw[0][0]) * kc.inv_two_h;
            const R fb = (tw[2][1] - tw[0][1]) * kc.inv_two_h;
            const R fc = (tw[2][2] - tw[0][2]) * kc.inv_two_h;
            const R g1 = (hpT[p * NLT] - hmT[p * NLT]) * (DIR == 0 ? kc.inv_two_dy : kc.inv_two_dx);
            const R g2 = (wT[p * WIDE + 1] - wT[p * WIDE - 1]) * kc.inv_two_dz;
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
        if (t == 0) {
            atomicExch(err_flag, 1);
            for (int b = 0; b < nbox; b++) tma::mbar_wait(&bar[b], 0, 1 << 10);   // copies still in flight
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
    if (!has) return;

    // ---------------- write-back ----------------
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int kd = kind[i];
        if (kd == R_NONE) continue;
        const int p = p0 + i;
        const long long off = lb + (long long)p * g.stride;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int m = v < 3 ? 0 : 1;
            R x = i == 0 ? xf[v] : (i == K - 1 ? xl[v] : dv[v][i] - ea[m][i] * xf[v] - ec[m][i] * xl[v]);
            if (kd == R_IN) {
                x += cT[v * fs + p * NLT];
                const R tv = v == DIR ? wT[p * WIDE] : tT[(v < DIR ? v : v - 1) * fs + p * NLT];
                R mm = (tv + x) * R(0.5);
                if (merges == 2) mm = (mm + x) * R(0.5);
                tout.f[v][off] = mm;
            }
            next.f[v][off] = x;
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

bool make_tile_map(CUtensorMap *m, const void *base, int dir, int nx, int ny, int nz, int w, int Lb, int es,
                   CUtensorMapDataType dt)
{
    struct Key {
        const void *base;
        int dir, nx, ny, nz, w, Lb, es, dt;
        bool operator==(const Key &o) const
        {
            return base == o.base && dir == o.dir && nx == o.nx && ny == o.ny && nz == o.nz && w == o.w &&
                   Lb == o.Lb && es == o.es && dt == o.dt;
        }
    };
    struct Ent {
        Key k;
        CUtensorMap m;
    };
    static std::vector<Ent> cache;
    static std::mutex mu;
    const Key key{base, dir, nx, ny, nz, w, Lb, es, (int)dt};
    {
        std::lock_guard<std::mutex> g(mu);
        for (const Ent &e : cache)
            if (e.k == key) { *m = e.m; return true; }
    }
    auto enc = get_encoder_fn();
    if (!enc) return false;
    cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)nz * es, (cuuint64_t)ny * nz * es};
    cuuint32_t box[3] = {(cuuint32_t)w, (cuuint32_t)(dir == 0 ? 1 : Lb), (cuuint32_t)(dir == 0 ? Lb : 1)};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    std::lock_guard<std::mutex> g(mu);
    if (cache.size() > 4096) cache.clear();
    cache.push_back({key, *m});
    return true;
}

size_t xytma_smem_bytes(int L, int P, int elem_bytes)
{
    const size_t plane = (size_t)L * NLT * elem_bytes;
    const size_t wide = ((size_t)L * WIDE * elem_bytes + 127) / 128 * 128;
    const size_t code = ((size_t)L * NLT + 127) / 128 * 128;
    return 9 * plane + wide + code + 2 * (size_t)NLT * P * 8 * elem_bytes + 64;   // + up to 4 mbarriers
}

bool xytma_supported(int dir, int nx, int ny, int nz, int K, int elem_bytes)
{
    if (dir > 1 || !have_tensor_map_encoder()) return false;
    const int L = dir == 0 ? nx : ny;
    if (nz % NLT != 0) return false;            // CTA tiles of 16 lines; code rows 16-byte strided
    if (K != 8 && K != 16) return false;
    if (L % K != 0) return false;
    const int P = L / K;
    if (NLT * P > 256 || NLT * P < 32) return false;
    if (L > 256 || L % 2 != 0) return false;    // boxes of <= 256 rows; 128-byte aligned tiles
    return xytma_smem_bytes(L, P, elem_bytes) <= 200 * 1024;
}

template <typename R>
cudaError_t launch_sweep_xytma(int dir, const DomainView<R> &d, const int *line_lo, CLayer<R> cur, CLayer<R> tin,
                               Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges, int K,
                               int *err_flag, cudaStream_t s)
{
    const int es = (int)sizeof(R);
    if (!xytma_supported(dir, d.nx, d.ny, d.nz, K, es)) return cudaErrorInvalidConfiguration;
    const LineGeom g = line_geom(dir, d.nx, d.ny, d.nz);
    const int L = g.len, P = L / K;
    // one box along the line (lines of up to 256 rows); the kernel also takes
    // several boxes per line, each on its own mbarrier, but splitting measured slower
    const int nbox = (L + 255) / 256, Lb = L / nbox;
    const CUtensorMapDataType dt = es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    XYMaps maps;
    for (int v = 0; v < 4; v++) {
        if (!make_tile_map(&maps.cur[v], cur.f[v], dir, d.nx, d.ny, d.nz, NLT, Lb, es, dt)) return cudaErrorInvalidValue;
        if (!make_tile_map(&maps.tin[v], tin.f[v], dir, d.nx, d.ny, d.nz, NLT, Lb, es, dt)) return cudaErrorInvalidValue;
    }
    if (!make_tile_map(&maps.fwide, tin.f[dir], dir, d.nx, d.ny, d.nz, WIDE, Lb, es, dt)) return cudaErrorInvalidValue;
    if (!make_tile_map(&maps.code, d.code, dir, d.nx, d.ny, d.nz, NLT, Lb, 1, CU_TENSOR_MAP_DATA_TYPE_UINT8))
        return cudaErrorInvalidValue;
    const size_t smem = xytma_smem_bytes(L, P, es);
    const int blocks = (dir == 0 ? d.ny : d.nx) * (d.nz / NLT);
    const int threads = NLT * P;
#define XL(DD, KK)                                                                                               \
    if (dir == DD && K == KK) {                                                                                  \
        auto kern = sweep_xytma_kernel<R, DD, KK>;                                                               \
        static int smem_set = 0;                                                                                 \
        if ((int)smem > smem_set) {                                                                              \
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
            if (e != cudaSuccess) return e;                                                                      \
            smem_set = (int)smem;                                                                                \
        }                                                                                                        \
        kern<<<blocks, threads, smem, s>>>(maps, d, g, P, Lb, nbox, line_lo, next, tout, k, merges, err_flag);   \
        return cudaGetLastError();                                                                               \
    }
    XL(0, 8) XL(0, 16) XL(1, 8) XL(1, 16)
#undef XL
    return cudaErrorInvalidConfiguration;
}

template cudaError_t launch_sweep_xytma<float>(int, const DomainView<float> &, const int *, CLayer<float>,
                                               CLayer<float>, Layer<float>, Layer<float>, const SweepConst<float> &,
                                               int, int, int *, cudaStream_t);
template cudaError_t launch_sweep_xytma<double>(int, const DomainView<double> &, const int *, CLayer<double>,
                                                CLayer<double>, Layer<double>, Layer<double>,
                                                const SweepConst<double> &, int, int, int *, cudaStream_t);

} // namespace adi
