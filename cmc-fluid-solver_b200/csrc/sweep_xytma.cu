// X and Y sweeps fed by the Tensor Memory Accelerator.
//
// A CTA owns NL = 16 neighbouring lines (16 consecutive k at one j for X, at one i
// for Y) over their whole length L.  One thread issues the tile loads
// (cp.async.bulk.tensor, no multicast) into shared memory, all completing on one
// mbarrier:
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
// The mbarrier wait is bounded: if the tile has not landed after about a second
// the CTA raises the handle's error flag and leaves without computing.
#include "adi_internal.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>
#include <vector>

namespace adi {

namespace {

enum : int { T_NONE = 0, T_START = 1, T_IN = 2, T_END = 3, T_SHARED = 4 };

__device__ __forceinline__ int tkind(bool inm, bool in0, bool inp)
{
    if (in0) return T_IN;
    if (inm && inp) return T_SHARED;
    if (inp) return T_START;
    if (inm) return T_END;
    return T_NONE;
}

template <typename R>
__device__ __forceinline__ R trcp(R x)
{
    return R(1) / x;
}
template <>
__device__ __forceinline__ float trcp<float>(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return fmaf(r, fmaf(-x, r, 1.0f), r);   // one Newton-Raphson step for 1/x
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :
        : "r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

constexpr int NLT = 16;   // lines per CTA
constexpr int WIDE = 24;  // width of the advecting-field tile (k0-4 .. k0+19)

} // namespace

// Tensor maps of one launch (by value, in param space).
struct XYMaps {
    CUtensorMap cur[4];
    CUtensorMap tin[4];   // plain 16-wide boxes
    CUtensorMap fwide;    // advecting field of temp, 24-wide box
    CUtensorMap code;
};

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
    uint64_t *bar = reinterpret_cast<uint64_t *>(buf1 + (size_t)NLT * P * 8);

    const bool has = line < g.nlines && line_lo[line] >= 0;
    if (!__syncthreads_or(has)) return;   // no segment in these 16 lines

    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (t == 0) {
        // every box delivers its full size (zero fill included): cur 4, temp 3,
        // off-line halo 2 planes, the wide advecting tile and the code tile
        const uint32_t bytes = (uint32_t)(9 * plane + (size_t)L * WIDE * sizeof(R) + (size_t)L * NLT);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                     : "memory");
        for (int b = 0; b < nbox; b++) {
            const int p0 = b * Lb;
            const size_t po = (size_t)p0 * NLT;        // row offset inside a [L][16] tile
            // coordinates (innermost first): X {k, j, x}, Y {k, y, i}
            const int c1 = DIR == 0 ? outer : p0, c2 = DIR == 0 ? p0 : outer;
            for (int v = 0; v < 4; v++) {
                tma_load_3d(tcur + v * (plane / sizeof(R)) + po, &maps.cur[v], k0, c1, c2, bar);
                if (v != DIR)
                    tma_load_3d(ttin + (v < DIR ? v : v - 1) * (plane / sizeof(R)) + po, &maps.tin[v], k0, c1, c2, bar);
            }
            tma_load_3d(twide + (size_t)p0 * WIDE, &maps.fwide, k0 - 4, c1, c2, bar);
            if (DIR == 0) {
                tma_load_3d(thm + po, &maps.tin[DIR], k0, outer - 1, p0, bar);
                tma_load_3d(thp + po, &maps.tin[DIR], k0, outer + 1, p0, bar);
            } else {
                tma_load_3d(thm + po, &maps.tin[DIR], k0, p0, outer - 1, bar);
                tma_load_3d(thp + po, &maps.tin[DIR], k0, p0, outer + 1, bar);
            }
            tma_load_3d(tcode + po, &maps.code, k0, c1, c2, bar);
        }
    }
    // bounded wait for the tiles (phase 0): at most 2^17 tries of at most ~10 us
    {
        uint32_t done = 0;
        for (int it = 0; it < (1 << 17) && !done; it++) {
            asm volatile(
                "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0, 10000; selp.u32 %0, 1, 0, p; }"
                : "=r"(done)
                : "r"(smem_u32(bar))
                : "memory");
        }
        if (__syncthreads_or(!done)) {
            if (t == 0) atomicExch(err_flag, 1);
            return;
        }
    }

    // ---------------- rows from the tiles ----------------
    const int p0 = ch * K;
    auto TC = [&](int v, int p) -> R { return tcur[(size_t)v * L * NLT + (size_t)p * NLT + li]; };
    auto TT = [&](int v, int p) -> R {
        return v == DIR ? twide[(size_t)p * WIDE + li + 4]
                        : ttin[(size_t)(v < DIR ? v : v - 1) * L * NLT + (size_t)p * NLT + li];
    };
    auto CODE = [&](int p) -> uint8_t { return (p >= 0 && p < L) ? tcode[(size_t)p * NLT + li] : uint8_t(NODE_OUT); };

    int kind[K];
    unsigned freebits = 0;
    R rr[K], dv[4][K];
    bool inr[K + 2];
    uint8_t cc[K + 2];
#pragma unroll
    for (int q = 0; q < K + 2; q++) {
        cc[q] = has ? CODE(p0 - 1 + q) : uint8_t(NODE_OUT);
        inr[q] = code_is_in(cc[q]);
    }
#pragma unroll
    for (int i = 0; i < K; i++) {
        kind[i] = tkind(inr[i], inr[i + 1], inr[i + 2]);
        if (cc[i + 1] & CODE_VEL_FREE) freebits |= 1u << (2 * i);
        if (cc[i + 1] & CODE_TEMP_FREE) freebits |= 2u << (2 * i);
    }
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int p = p0 + i;
        const int kd = kind[i];
        rr[i] = R(0);
        if (kd == T_IN) {
            // IN rows are never the first or last node of a line
            const R r = TT(DIR, p) * kc.inv_two_h;
            rr[i] = r;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const R vis = v < 3 ? kc.vis_v : kc.vis_t;
                const R cm = inr[i] ? TC(v, p - 1) : R(0);
                const R cp = inr[i + 2] ? TC(v, p + 1) : R(0);
                dv[v][i] = vis * (cm - R(2) * TC(v, p) + cp) - r * (cp - cm);
            }
            dv[DIR][i] -= kc.v_T * ((TT(3, p + 1) - TT(3, p - 1)) * kc.inv_two_h);
            const R fa = (TT(0, p + 1) - TT(0, p - 1)) * kc.inv_two_h;
            const R fb = (TT(1, p + 1) - TT(1, p - 1)) * kc.inv_two_h;
            const R fc = (TT(2, p + 1) - TT(2, p - 1)) * kc.inv_two_h;
            const R g1 = (thp[(size_t)p * NLT + li] - thm[(size_t)p * NLT + li]) *
                         (DIR == 0 ? kc.inv_two_dy : kc.inv_two_dx);
            const R g2 = (twide[(size_t)p * WIDE + li + 5] - twide[(size_t)p * WIDE + li + 3]) * kc.inv_two_dz;
            R diss;
            if (DIR == 0) diss = R(2) * fa * fa + fb * fb + fc * fc + fb * g1 + fc * g2;
            else diss = fa * fa + R(2) * fb * fb + fc * fc + fa * g1 + fc * g2;
            dv[3][i] += kc.t_phi * diss;
        } else if (kd == T_NONE) {
#pragma unroll
            for (int v = 0; v < 4; v++) dv[v][i] = R(0);
        } else {
            const bool vf = (freebits >> (2 * i)) & 1u, tf = (freebits >> (2 * i + 1)) & 1u;
            const int pn = kd == T_END ? p - 1 : p + 1;   // the IN neighbour
            const long long off = line_base(DIR, g, line) + (long long)p * g.stride;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const bool fr = v < 3 ? vf : tf;
                dv[v][i] = fr ? TC(v, pn) : __ldg(d.nv[v] + off);
            }
        }
    }

    // ---------------- chunk elimination ----------------
    R ea[2][K], ec[2][K];
    R Af[2], Cf[2], Al[2], Cl[2], Df[4], Dl[4];
#pragma unroll
    for (int m = 0; m < 2; m++) {
        const R vis = m == 0 ? kc.vis_v : kc.vis_t;
        const R bin = m == 0 ? kc.b_v : kc.b_t;
        R A[K], B[K], C[K];
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int kd = kind[i];
            const bool fr = (freebits >> (2 * i + m)) & 1u;
            if (kd == T_IN) { A[i] = -rr[i] - vis; B[i] = bin; C[i] = rr[i] - vis; }
            else if (kd == T_NONE) { A[i] = R(0); B[i] = R(1); C[i] = R(0); }
            else {
                const bool first = kd != T_END;
                B[i] = fr ? R(2) : R(1);
                A[i] = (!first && fr) ? R(-1) : R(0);
                C[i] = (first && fr) ? R(-1) : R(0);
            }
        }
        {
            const R r = trcp<R>(B[1]);
            ea[m][1] = A[1] * r;
            ec[m][1] = C[1] * r;
            if (m == 0) { dv[0][1] *= r; dv[1][1] *= r; dv[2][1] *= r; }
            else dv[3][1] *= r;
        }
#pragma unroll
        for (int i = 2; i <= K - 2; i++) {
            const R r = trcp<R>(B[i] - A[i] * ec[m][i - 1]);
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) dv[v][i] = (dv[v][i] - A[i] * dv[v][i - 1]) * r;
            } else {
                dv[3][i] = (dv[3][i] - A[i] * dv[3][i - 1]) * r;
            }
            ea[m][i] = -A[i] * ea[m][i - 1] * r;
            ec[m][i] = C[i] * r;
        }
#pragma unroll
        for (int i = K - 3; i >= 1; i--) {
            const R ci = ec[m][i];
            ea[m][i] -= ci * ea[m][i + 1];
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) dv[v][i] -= ci * dv[v][i + 1];
            } else {
                dv[3][i] -= ci * dv[3][i + 1];
            }
            ec[m][i] = -ci * ec[m][i + 1];
        }
        const R rf = trcp<R>(B[0] - C[0] * ea[m][1]);
        Af[m] = A[0] * rf;
        Cf[m] = -C[0] * ec[m][1] * rf;
        const R rl = trcp<R>(B[K - 1] - A[K - 1] * ec[m][K - 2]);
        Al[m] = -A[K - 1] * ea[m][K - 2] * rl;
        Cl[m] = C[K - 1] * rl;
        if (m == 0) {
#pragma unroll
            for (int v = 0; v < 3; v++) {
                Df[v] = (dv[v][0] - C[0] * dv[v][1]) * rf;
                Dl[v] = (dv[v][K - 1] - A[K - 1] * dv[v][K - 2]) * rl;
            }
        } else {
            Df[3] = (dv[3][0] - C[0] * dv[3][1]) * rf;
            Dl[3] = (dv[3][K - 1] - A[K - 1] * dv[3][K - 2]) * rl;
        }
    }

    // ---------------- reduced system: one CR step + PCR, 8-value slots ----------------
    auto SLOT = [&](R *b, int c) -> R * { return b + ((size_t)c * NLT + li) * 8; };
    {
        R *w = SLOT(buf0, ch);
        w[0] = Al[0]; w[1] = Cl[0]; w[2] = Al[1]; w[3] = Cl[1];
        w[4] = Dl[0]; w[5] = Dl[1]; w[6] = Dl[2]; w[7] = Dl[3];
    }
    __syncthreads();
    R ea_[2], ec_[2], ed[4];
    {
        R pv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (ch > 0) {
            const R *r = SLOT(buf0, ch - 1);
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = r[q];
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const R pA = pv[2 * m], pC = pv[2 * m + 1];
            const R r = trcp<R>(R(1) - Af[m] * pC - Cf[m] * Al[m]);
            ea_[m] = -Af[m] * pA * r;
            ec_[m] = -Cf[m] * Cl[m] * r;
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) ed[v] = (Df[v] - Af[0] * pv[4 + v] - Cf[0] * Dl[v]) * r;
            } else {
                ed[3] = (Df[3] - Af[1] * pv[7] - Cf[1] * Dl[3]) * r;
            }
        }
    }
    int nstep = 0;
    for (int s = 1; s < P; s <<= 1, nstep++) {
        R *bw = (nstep & 1) ? buf0 : buf1;
        {
            R *w = SLOT(bw, ch);
            w[0] = ea_[0]; w[1] = ec_[0]; w[2] = ea_[1]; w[3] = ec_[1];
            w[4] = ed[0]; w[5] = ed[1]; w[6] = ed[2]; w[7] = ed[3];
        }
        __syncthreads();
        R mv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        R pv[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
        if (ch - s >= 0) {
            const R *r = SLOT(bw, ch - s);
#pragma unroll
            for (int q = 0; q < 8; q++) mv[q] = r[q];
        }
        if (ch + s < P) {
            const R *r = SLOT(bw, ch + s);
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = r[q];
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const R a = ea_[m], c = ec_[m];
            const R r = trcp<R>(R(1) - a * mv[2 * m + 1] - c * pv[2 * m]);
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) ed[v] = (ed[v] - a * mv[4 + v] - c * pv[4 + v]) * r;
            } else {
                ed[3] = (ed[3] - a * mv[7] - c * pv[7]) * r;
            }
            ea_[m] = -a * mv[2 * m] * r;
            ec_[m] = -c * pv[2 * m + 1] * r;
        }
    }
    R *bx = (nstep & 1) ? buf0 : buf1;
    {
        R *w = SLOT(bx, ch);
        w[0] = ed[0]; w[1] = ed[1]; w[2] = ed[2]; w[3] = ed[3];
    }
    __syncthreads();
    R xf[4], xl[4];
    {
        R nf[4] = {R(0), R(0), R(0), R(0)};
        if (ch + 1 < P) {
            const R *r = SLOT(bx, ch + 1);
#pragma unroll
            for (int v = 0; v < 4; v++) nf[v] = r[v];
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            xf[v] = ed[v];
            const int m = v < 3 ? 0 : 1;
            xl[v] = Dl[v] - Al[m] * xf[v] - Cl[m] * nf[v];
        }
    }
    if (!has) return;

    // ---------------- write-back ----------------
    const long long lb = line_base(DIR, g, line);
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int kd = kind[i];
        if (kd == T_NONE) continue;
        const int p = p0 + i;
        const long long off = lb + (long long)p * g.stride;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int m = v < 3 ? 0 : 1;
            R x = i == 0 ? xf[v] : (i == K - 1 ? xl[v] : dv[v][i] - ea[m][i] * xf[v] - ec[m][i] * xl[v]);
            if (kd == T_IN) {
                x += TC(v, p);
                R mm = (TT(v, p) + x) * R(0.5);
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

static PFN_cuTensorMapEncodeTiled_v12000 get_encoder()
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
static bool make_map(CUtensorMap *m, const void *base, int dir, int nx, int ny, int nz, int w, int Lb, int es,
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
    auto enc = get_encoder();
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
    return 9 * plane + wide + code + 2 * (size_t)NLT * P * 8 * elem_bytes + 16;
}

bool xytma_supported(int dir, int nx, int ny, int nz, int K, int elem_bytes)
{
    if (dir > 1 || !get_encoder()) return false;
    const int L = dir == 0 ? nx : ny;
    if (nz % NLT != 0) return false;            // CTA tiles of 16 lines; code rows 16-byte strided
    if (K != 8 && K != 16) return false;
    if (L % K != 0) return false;
    const int P = L / K;
    if (NLT * P > 256 || NLT * P < 32) return false;
    if (L > 256 || L % 2 != 0) return false;    // one box along the line; 128-byte aligned tiles
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
    const int nbox = (L + 255) / 256, Lb = L / nbox;
    const CUtensorMapDataType dt = es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    XYMaps maps;
    for (int v = 0; v < 4; v++) {
        if (!make_map(&maps.cur[v], cur.f[v], dir, d.nx, d.ny, d.nz, NLT, Lb, es, dt)) return cudaErrorInvalidValue;
        if (!make_map(&maps.tin[v], tin.f[v], dir, d.nx, d.ny, d.nz, NLT, Lb, es, dt)) return cudaErrorInvalidValue;
    }
    if (!make_map(&maps.fwide, tin.f[dir], dir, d.nx, d.ny, d.nz, WIDE, Lb, es, dt)) return cudaErrorInvalidValue;
    if (!make_map(&maps.code, d.code, dir, d.nx, d.ny, d.nz, NLT, Lb, 1, CU_TENSOR_MAP_DATA_TYPE_UINT8))
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
