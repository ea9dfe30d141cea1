// X and Y sweeps (FP32): persistent CTAs, double-buffered TMA tiles, two lines
// per thread.
//
// A tile is 16 neighbouring lines (k0 .. k0+15 at one j for X, at one i for Y)
// over their whole length L, loaded exactly as in sweep_xytma.cu (cur U V W T,
// the three temp fields other than the advecting one, the advecting field 24
// wide for the k +-1 halo, its off-line halo planes, the node codes), with
// cp.async.bulk.tensor (no multicast) completing on one mbarrier per buffer.
//
// One CTA per SM walks the tile list with two tile buffers: while it solves tile
// n from one buffer, the tile it will solve next is landing in the other, and the
// load of tile n+2 is issued as soon as tile n is done.  Thread (pair, chunk)
// owns lines k0+2*pair and k0+2*pair+1 over the K rows of its chunk, so every
// shared-memory read and every global store moves both lines at once (8 bytes),
// and the two independent systems give the scheduler instruction-level
// parallelism.  The arithmetic is that of the other fast sweeps (sweep_common.cuh:
// increment form, chunk elimination, one cyclic-reduction step and PCR over the
// chunk-first unknowns); the reduced rows travel through shared memory stored
// value-major, so neighbouring chunks' slots are read without bank conflicts.
//
// Every mbarrier wait is bounded; a CTA that gives up raises the handle's error
// flag, waits (bounded) for its other buffer's load if one is in flight, and
// leaves.
#include "adi_internal.cuh"
#include "sweep_common.cuh"
#include "tma.cuh"

namespace adi {

namespace {

constexpr int PT = 16;   // lines per tile
constexpr int PW = 24;   // advecting-field tile width (k0-4 .. k0+19)

// Byte layout of one tile buffer: cur planes 0-3, temp planes 4-6 (fields other
// than the advecting one, in field order), the wide advecting tile, the halo
// planes at outer-1 and outer+1, the code plane.
struct PairTile {
    size_t plane, wide, code, bytes;
};

__host__ __device__ inline PairTile pair_tile(int L)
{
    PairTile t;
    t.plane = (size_t)L * PT * sizeof(float);
    t.wide = ((size_t)L * PW * sizeof(float) + 127) / 128 * 128;
    t.code = ((size_t)L * PT + 127) / 128 * 128;
    t.bytes = (9 * t.plane + t.wide + t.code + 1023) / 1024 * 1024;
    return t;
}

// 8 reduced-row values of both lines of a thread, value-major slots:
// value j of chunk c, line li at S[j * sstride + c * PT + li].
template <int NV>
__device__ __forceinline__ void slots_put(float *S, int sstride, int c, int pr, const float (&a)[8],
                                          const float (&b)[8])
{
#pragma unroll
    for (int j = 0; j < NV; j++)
        *reinterpret_cast<float2 *>(S + j * sstride + c * PT + 2 * pr) = make_float2(a[j], b[j]);
}

template <int NV>
__device__ __forceinline__ void slots_get(const float *S, int sstride, int c, int pr, float (&a)[8], float (&b)[8])
{
#pragma unroll
    for (int j = 0; j < NV; j++) {
        const float2 x = *reinterpret_cast<const float2 *>(S + j * sstride + c * PT + 2 * pr);
        a[j] = x.x;
        b[j] = x.y;
    }
}

} // namespace

size_t xypair_smem_bytes(int L, int P)
{
    const PairTile t = pair_tile(L);
    return 2 * t.bytes + 2 * 8 * (size_t)P * PT * sizeof(float) + 64;
}

template <int DIR, int K>
__global__ void __launch_bounds__(256, 1)
    sweep_xypair_kernel(const __grid_constant__ XYMaps maps, DomainView<float> d, LineGeom g, int P, int ntiles,
                        const int *__restrict__ line_lo, Layer<float> next, Layer<float> tout, SweepConst<float> kc,
                        int merges, int *err_flag)
{
    using namespace sweep;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int L = g.len;
    const PairTile tl = pair_tile(L);
    const int t = threadIdx.x;
    const int pr = t & 7, ch = t >> 3;
    const int sstride = P * PT;
    float *const S0 = reinterpret_cast<float *>(smem + 2 * tl.bytes);
    float *const S1 = S0 + 8 * sstride;
    uint64_t *const bar = reinterpret_cast<uint64_t *>(S1 + 8 * sstride);
    int *const skip = reinterpret_cast<int *>(bar + 2);
    const int kblocks = g.nz / PT;
    const uint32_t tx_bytes = (uint32_t)(9 * tl.plane + (size_t)L * PW * sizeof(float) + (size_t)L * PT);
    const int fs = L * PT;   // floats per plane

    // Thread 0: starts the loads of `tile` into buffer b; false if none of its
    // 16 lines has a segment (nothing is loaded or solved for it).
    auto issue = [&](int b, int tile) -> bool {
        const int outer = tile / kblocks, k0 = (tile - outer * kblocks) * PT;
        bool any = false;
        for (int q = 0; q < PT; q++) any |= line_lo[outer * g.nz + k0 + q] >= 0;
        if (!any) return false;
        unsigned char *buf = smem + b * tl.bytes;
        tma::arrive_expect_tx(&bar[b], tx_bytes);
        // coordinates innermost first: X {k, j, x}, Y {k, y, i}; the whole line is one box
        const int c1 = DIR == 0 ? outer : 0, c2 = DIR == 0 ? 0 : outer;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            tma::load_3d(buf + v * tl.plane, &maps.cur[v], k0, c1, c2, &bar[b]);
            if (v != DIR) tma::load_3d(buf + (4 + (v < DIR ? v : v - 1)) * tl.plane, &maps.tin[v], k0, c1, c2, &bar[b]);
        }
        tma::load_3d(buf + 7 * tl.plane, &maps.fwide, k0 - 4, c1, c2, &bar[b]);
        unsigned char *hm = buf + 7 * tl.plane + tl.wide, *hp = hm + tl.plane;
        if (DIR == 0) {
            tma::load_3d(hm, &maps.tin[DIR], k0, outer - 1, 0, &bar[b]);
            tma::load_3d(hp, &maps.tin[DIR], k0, outer + 1, 0, &bar[b]);
        } else {
            tma::load_3d(hm, &maps.tin[DIR], k0, 0, outer - 1, &bar[b]);
            tma::load_3d(hp, &maps.tin[DIR], k0, 0, outer + 1, &bar[b]);
        }
        tma::load_3d(buf + 9 * tl.plane + tl.wide, &maps.code, k0, c1, c2, &bar[b]);
        return true;
    };

    if (t == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const int tile = blockIdx.x + b * gridDim.x;
            skip[b] = !(tile < ntiles && issue(b, tile));
        }
    }
    __syncthreads();

    unsigned ph = 0;   // bit b: parity of the next phase of bar[b]
    for (int n = 0;; n++) {
        const int tile = blockIdx.x + n * gridDim.x;
        if (tile >= ntiles) break;
        const int b = n & 1;
        if (!skip[b]) {
            const bool ok = tma::mbar_wait(&bar[b], (ph >> b) & 1u, 1 << 17);
            ph ^= 1u << b;
            if (__syncthreads_or(!ok)) {
                if (t == 0) {
                    atomicExch(err_flag, 1);
                    if (!skip[b ^ 1]) tma::mbar_wait(&bar[b ^ 1], (ph >> (b ^ 1)) & 1u, 1 << 10);
                }
                return;
            }

            const int outer = tile / kblocks, k0 = (tile - outer * kblocks) * PT;
            const unsigned char *buf = smem + b * tl.bytes;
            const float *__restrict__ cT = reinterpret_cast<const float *>(buf) + 2 * pr;
            const float *__restrict__ tT = reinterpret_cast<const float *>(buf + 4 * tl.plane) + 2 * pr;
            const float *__restrict__ wT = reinterpret_cast<const float *>(buf + 7 * tl.plane) + 4 + 2 * pr;
            const float *__restrict__ hmT = reinterpret_cast<const float *>(buf + 7 * tl.plane + tl.wide) + 2 * pr;
            const float *__restrict__ hpT = hmT + fs;
            const uint8_t *__restrict__ kT = buf + 9 * tl.plane + tl.wide + 2 * pr;

            // ---------------- rows from the tiles: one pass, 3-row window ----------------
            const int p0 = ch * K;
            float cw[3][4][2], tw[3][4][2];
            uint8_t kw[3][2];
#define XP_LOAD_ROW(SLOT_, P_)                                                                              \
    {                                                                                                       \
        const int pp = (P_);                                                                                \
        const bool ok_ = pp >= 0 && pp < L;                                                                 \
        const unsigned c2 = ok_ ? *reinterpret_cast<const uint16_t *>(kT + pp * PT)                         \
                                : unsigned(NODE_OUT) | (unsigned(NODE_OUT) << 8);                           \
        kw[SLOT_][0] = uint8_t(c2 & 0xffu);                                                                 \
        kw[SLOT_][1] = uint8_t(c2 >> 8);                                                                    \
        const bool i0 = code_is_in(kw[SLOT_][0]), i1 = code_is_in(kw[SLOT_][1]);                            \
        _Pragma("unroll") for (int v = 0; v < 4; v++)                                                       \
        {                                                                                                   \
            const float2 tv = !ok_ ? make_float2(0.f, 0.f)                                                  \
                                   : (v == DIR ? *reinterpret_cast<const float2 *>(wT + pp * PW)            \
                                               : *reinterpret_cast<const float2 *>(                         \
                                                     tT + (v < DIR ? v : v - 1) * fs + pp * PT));           \
            tw[SLOT_][v][0] = tv.x;                                                                         \
            tw[SLOT_][v][1] = tv.y;                                                                         \
            const float2 cv = (i0 || i1) ? *reinterpret_cast<const float2 *>(cT + v * fs + pp * PT)         \
                                         : make_float2(0.f, 0.f);                                           \
            cw[SLOT_][v][0] = i0 ? cv.x : 0.f;                                                              \
            cw[SLOT_][v][1] = i1 ? cv.y : 0.f;                                                              \
        }                                                                                                   \
    }
            int kind[2][K];
            unsigned freebits[2] = {0u, 0u};
            float rr[2][K], dv[2][4][K];
            XP_LOAD_ROW(0, p0 - 1)
            XP_LOAD_ROW(1, p0)
            // global offset of line A's node 0: X (0, j, k) = j*nz + k; Y (i, 0, k) = i*ny*nz + k
            const long long lb = (DIR == 0 ? (long long)outer * g.nz : (long long)outer * g.ny * g.nz) + k0 + 2 * pr;
#pragma unroll
            for (int i = 0; i < K; i++) {
                const int p = p0 + i;
                XP_LOAD_ROW(2, p + 1)
                float2 hm2 = make_float2(0.f, 0.f), hp2 = make_float2(0.f, 0.f);
                float wl = 0.f, wr = 0.f;
                if (code_is_in(kw[1][0]) || code_is_in(kw[1][1])) {
                    hm2 = *reinterpret_cast<const float2 *>(hmT + p * PT);
                    hp2 = *reinterpret_cast<const float2 *>(hpT + p * PT);
                    wl = wT[p * PW - 1];   // k-1 of line A
                    wr = wT[p * PW + 2];   // k+1 of line B
                }
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const int kd = row_kind(code_is_in(kw[0][q]), code_is_in(kw[1][q]), code_is_in(kw[2][q]));
                    kind[q][i] = kd;
                    if (kw[1][q] & CODE_VEL_FREE) freebits[q] |= 1u << (2 * i);
                    if (kw[1][q] & CODE_TEMP_FREE) freebits[q] |= 2u << (2 * i);
                    rr[q][i] = 0.f;
                    if (kd == R_IN) {
                        // IN rows are never the first or last node of a line
                        const float r = tw[1][DIR][q] * kc.inv_two_h;
                        rr[q][i] = r;
#pragma unroll
                        for (int v = 0; v < 4; v++) {
                            const float vis = v < 3 ? kc.vis_v : kc.vis_t;
                            dv[q][v][i] = vis * (cw[0][v][q] - 2.f * cw[1][v][q] + cw[2][v][q]) -
                                          r * (cw[2][v][q] - cw[0][v][q]);
                        }
                        dv[q][DIR][i] -= kc.v_T * ((tw[2][3][q] - tw[0][3][q]) * kc.inv_two_h);
                        const float fa = (tw[2][0][q] - tw[0][0][q]) * kc.inv_two_h;
                        const float fb = (tw[2][1][q] - tw[0][1][q]) * kc.inv_two_h;
                        const float fc = (tw[2][2][q] - tw[0][2][q]) * kc.inv_two_h;
                        const float g1 = ((q ? hp2.y : hp2.x) - (q ? hm2.y : hm2.x)) *
                                         (DIR == 0 ? kc.inv_two_dy : kc.inv_two_dx);
                        const float g2 = ((q ? wr : tw[1][DIR][1]) - (q ? tw[1][DIR][0] : wl)) * kc.inv_two_dz;
                        float diss;
                        if (DIR == 0) diss = 2.f * fa * fa + fb * fb + fc * fc + fb * g1 + fc * g2;
                        else diss = fa * fa + 2.f * fb * fb + fc * fc + fa * g1 + fc * g2;
                        dv[q][3][i] += kc.t_phi * diss;
                    } else if (kd == R_NONE) {
#pragma unroll
                        for (int v = 0; v < 4; v++) dv[q][v][i] = 0.f;
                    } else {
                        // boundary row; BC_FREE moves the IN neighbour's cur to the right side
                        const bool vf = (kw[1][q] & CODE_VEL_FREE) != 0, tf = (kw[1][q] & CODE_TEMP_FREE) != 0;
                        const bool from_left = kd == R_END;   // IN neighbour at p-1, else at p+1
                        const long long off = lb + q + (long long)p * g.stride;
#pragma unroll
                        for (int v = 0; v < 4; v++) {
                            const bool fr = v < 3 ? vf : tf;
                            const float cn = from_left ? cw[0][v][q] : cw[2][v][q];
                            dv[q][v][i] = fr ? cn : (kc.nv_in_temp ? tw[1][v][q] : __ldg(d.nv[v] + off));
                        }
                    }
                }
#pragma unroll
                for (int v = 0; v < 4; v++)
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        cw[0][v][q] = cw[1][v][q]; cw[1][v][q] = cw[2][v][q];
                        tw[0][v][q] = tw[1][v][q]; tw[1][v][q] = tw[2][v][q];
                    }
                kw[0][0] = kw[1][0]; kw[1][0] = kw[2][0];
                kw[0][1] = kw[1][1]; kw[1][1] = kw[2][1];
            }
#undef XP_LOAD_ROW

            // ---------------- chunk elimination, both lines ----------------
            float ea[2][2][K], ec[2][2][K];
            Reduced<float> red[2];
#pragma unroll
            for (int q = 0; q < 2; q++) eliminate<float, K>(kind[q], rr[q], freebits[q], kc, dv[q], ea[q], ec[q], red[q]);

            // ---------------- reduced system: one CR step + PCR through the slots ----------------
            // Couplings to rows outside the line are exactly zero (the first row of a
            // line has a = 0, the last c = 0, and PCR keeps them zero), so a thread
            // whose partner chunk would lie outside reads its own slot instead.
            {
                const float la[8] = {red[0].Al[0], red[0].Cl[0], red[0].Al[1], red[0].Cl[1],
                                     red[0].Dl[0], red[0].Dl[1], red[0].Dl[2], red[0].Dl[3]};
                const float lbv[8] = {red[1].Al[0], red[1].Cl[0], red[1].Al[1], red[1].Cl[1],
                                      red[1].Dl[0], red[1].Dl[1], red[1].Dl[2], red[1].Dl[3]};
                slots_put<8>(S0, sstride, ch, pr, la, lbv);
            }
            __syncthreads();
            float ea_[2][2], ec_[2][2], ed[2][4];
            {
                float pa[8], pb[8];
                slots_get<8>(S0, sstride, ch > 0 ? ch - 1 : ch, pr, pa, pb);
                if (ch == 0) {
#pragma unroll
                    for (int j = 0; j < 8; j++) pa[j] = pb[j] = 0.f;
                }
                cr_step<float>(red[0], pa, ea_[0], ec_[0], ed[0]);
                cr_step<float>(red[1], pb, ea_[1], ec_[1], ed[1]);
            }
            int nstep = 0;
            for (int st = 1; st < P; st <<= 1, nstep++) {
                float *const bw = (nstep & 1) ? S0 : S1;
                {
                    const float va[8] = {ea_[0][0], ec_[0][0], ea_[0][1], ec_[0][1], ed[0][0], ed[0][1], ed[0][2], ed[0][3]};
                    const float vb[8] = {ea_[1][0], ec_[1][0], ea_[1][1], ec_[1][1], ed[1][0], ed[1][1], ed[1][2], ed[1][3]};
                    slots_put<8>(bw, sstride, ch, pr, va, vb);
                }
                __syncthreads();
                float ma[8], mb[8], pa[8], pb[8];
                slots_get<8>(bw, sstride, ch - st >= 0 ? ch - st : ch, pr, ma, mb);
                slots_get<8>(bw, sstride, ch + st < P ? ch + st : ch, pr, pa, pb);
                pcr_update<float>(ma, pa, ea_[0], ec_[0], ed[0]);
                pcr_update<float>(mb, pb, ea_[1], ec_[1], ed[1]);
            }
            float *const bx = (nstep & 1) ? S0 : S1;
            {
                float va[8], vb[8];
#pragma unroll
                for (int v = 0; v < 4; v++) { va[v] = ed[0][v]; vb[v] = ed[1][v]; }
#pragma unroll
                for (int v = 4; v < 8; v++) va[v] = vb[v] = 0.f;
                slots_put<4>(bx, sstride, ch, pr, va, vb);
            }
            __syncthreads();
            float xf[2][4], xl[2][4];
            {
                float na[8], nbv[8];
                slots_get<4>(bx, sstride, ch + 1 < P ? ch + 1 : ch, pr, na, nbv);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const int m = v < 3 ? 0 : 1;
                    xf[0][v] = ed[0][v];
                    xf[1][v] = ed[1][v];
                    xl[0][v] = red[0].Dl[v] - red[0].Al[m] * xf[0][v] - red[0].Cl[m] * na[v];   // Cl = 0 on the last chunk
                    xl[1][v] = red[1].Dl[v] - red[1].Al[m] * xf[1][v] - red[1].Cl[m] * nbv[v];
                }
            }

            // ---------------- write-back, both lines per access ----------------
#pragma unroll
            for (int i = 0; i < K; i++) {
                const int kA = kind[0][i], kB = kind[1][i];
                if (kA == R_NONE && kB == R_NONE) continue;
                const int p = p0 + i;
                const long long off = lb + (long long)p * g.stride;
                const bool inA = kA == R_IN, inB = kB == R_IN;
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const int m = v < 3 ? 0 : 1;
                    float x[2];
#pragma unroll
                    for (int q = 0; q < 2; q++)
                        x[q] = i == 0 ? xf[q][v]
                                      : (i == K - 1 ? xl[q][v] : dv[q][v][i] - ea[q][m][i] * xf[q][v] - ec[q][m][i] * xl[q][v]);
                    if (inA || inB) {
                        const float2 c2 = *reinterpret_cast<const float2 *>(cT + v * fs + p * PT);
                        const float2 t2 = v == DIR ? *reinterpret_cast<const float2 *>(wT + p * PW)
                                                   : *reinterpret_cast<const float2 *>(tT + (v < DIR ? v : v - 1) * fs + p * PT);
                        if (inA) x[0] += c2.x;
                        if (inB) x[1] += c2.y;
                        float mA = (t2.x + x[0]) * 0.5f, mB = (t2.y + x[1]) * 0.5f;
                        if (merges == 2) {
                            mA = (mA + x[0]) * 0.5f;
                            mB = (mB + x[1]) * 0.5f;
                        }
                        if (inA && inB) *reinterpret_cast<float2 *>(tout.f[v] + off) = make_float2(mA, mB);
                        else if (inA) tout.f[v][off] = mA;
                        else tout.f[v][off + 1] = mB;
                    }
                    if (kA != R_NONE && kB != R_NONE) *reinterpret_cast<float2 *>(next.f[v] + off) = make_float2(x[0], x[1]);
                    else if (kA != R_NONE) next.f[v][off] = x[0];
                    else next.f[v][off + 1] = x[1];
                }
            }
        }
        __syncthreads();   // buffer b and the slots are free again
        if (t == 0) {
            const int nt = tile + 2 * gridDim.x;
            skip[b] = !(nt < ntiles && issue(b, nt));
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

bool xypair_supported(int dir, int nx, int ny, int nz, int K, int elem_bytes)
{
    if (dir > 1 || elem_bytes != 4 || !have_tensor_map_encoder()) return false;
    const int L = dir == 0 ? nx : ny;
    if (nz % PT != 0) return false;   // whole tiles of 16 lines
    if (K != 4 && K != 8) return false;
    if (L % K != 0 || L > 256 || L % 2 != 0) return false;   // one box along the line
    const int P = L / K;
    if (P < 2 || 8 * P > 256) return false;
    return xypair_smem_bytes(L, P) <= 227 * 1024;
}

cudaError_t launch_sweep_xypair(int dir, const DomainView<float> &d, const int *line_lo, CLayer<float> cur,
                                CLayer<float> tin, Layer<float> next, Layer<float> tout, const SweepConst<float> &k,
                                int merges, int K, int *err_flag, cudaStream_t s)
{
    if (!xypair_supported(dir, d.nx, d.ny, d.nz, K, 4)) return cudaErrorInvalidConfiguration;
    const LineGeom g = line_geom(dir, d.nx, d.ny, d.nz);
    const int L = g.len, P = L / K;
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    XYMaps maps;
    for (int v = 0; v < 4; v++) {
        if (!make_tile_map(&maps.cur[v], cur.f[v], dir, d.nx, d.ny, d.nz, PT, L, 4, dt)) return cudaErrorInvalidValue;
        if (!make_tile_map(&maps.tin[v], tin.f[v], dir, d.nx, d.ny, d.nz, PT, L, 4, dt)) return cudaErrorInvalidValue;
    }
    if (!make_tile_map(&maps.fwide, tin.f[dir], dir, d.nx, d.ny, d.nz, PW, L, 4, dt)) return cudaErrorInvalidValue;
    if (!make_tile_map(&maps.code, d.code, dir, d.nx, d.ny, d.nz, PT, L, 1, CU_TENSOR_MAP_DATA_TYPE_UINT8))
        return cudaErrorInvalidValue;
    const size_t smem = xypair_smem_bytes(L, P);
    const int ntiles = (dir == 0 ? d.ny : d.nx) * (d.nz / PT);
    const int threads = 8 * P;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
#define XP(DD, KK)                                                                                              \
    if (dir == DD && K == KK) {                                                                                 \
        auto kern = sweep_xypair_kernel<DD, KK>;                                                                \
        static SmemOptIn opt_in;                                                                                \
        e = ensure_dynamic_smem(opt_in, kern, smem);                                                            \
        if (e != cudaSuccess) return e;                                                                         \
        int per_sm = 0;                                                                                         \
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);                        \
        if (e != cudaSuccess) return e;                                                                         \
        if (per_sm < 1) return cudaErrorInvalidConfiguration;                                                   \
        const int grid = ntiles < sms * per_sm ? ntiles : sms * per_sm;                                         \
        kern<<<grid, threads, smem, s>>>(maps, d, g, P, ntiles, line_lo, next, tout, k, merges, err_flag);      \
        return cudaGetLastError();                                                                              \
    }
    XP(0, 4) XP(0, 8) XP(1, 4) XP(1, 8)
#undef XP
    return cudaErrorInvalidConfiguration;
}

} // namespace adi
