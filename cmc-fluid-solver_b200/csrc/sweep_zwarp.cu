// Z sweep with warp-resident lines.
//
// Z lines are contiguous in memory.  A line of L = dimz nodes is held by P
// consecutive lanes of one warp (P in {4, 8, 16, 32}, the smallest with P*K >= L;
// 32/P lines per warp), lane `ch` owning rows [ch*K, ch*K + K) of the line; rows
// at or beyond L are padding (NODE_OUT, no loads or stores).  Where a lane's
// chunk lies whole inside the line and dimz keeps it 16-byte aligned, every
// global access is a 16-byte vector access: the own rows of cur and temp, the
// four off-line neighbour lines of the advecting component (x+-1, y+-1), and the
// stores when a whole chunk is written; otherwise the lane accesses its rows one
// by one.
// The rows just outside a chunk (stencil halo) come from the neighbouring lanes
// by shuffle, and the reduced system of the line -- one cyclic-reduction step
// then parallel cyclic reduction over the P chunk-first unknowns -- runs entirely
// in shuffles, so the kernel uses neither shared memory nor barriers.
//
// Rows, increment form, chunk elimination and boundary handling are those of the
// generic fast sweep (sweep_fast.cu); see the comments there.  The chunk
// elimination, the cyclic-reduction step and the PCR updates are the shared ones
// of sweep_common.cuh (packed FP32 in float).  Requirements
// (checked by the launcher): K in {4, 5, 8}, or 12 in FP32 for 256 < dimz <= 384;
// dimz <= 32*K; 16-byte aligned field arrays.
#include "adi_internal.cuh"
#include "sweep_common.cuh"

#include <climits>

namespace adi {

namespace {

enum : int { Z_NONE = 0, Z_START = 1, Z_IN = 2, Z_END = 3, Z_SHARED = 4 };

__device__ __forceinline__ int zkind(bool inm, bool in0, bool inp)
{
    if (in0) return Z_IN;
    if (inm && inp) return Z_SHARED;
    if (inp) return Z_START;
    if (inm) return Z_END;
    return Z_NONE;
}

template <typename R, int K>
__device__ __forceinline__ void vload(const R *p, R (&out)[K])
{
    if (sizeof(R) == 4) {
#pragma unroll
        for (int q = 0; q < K / 4; q++) {
            const float4 v = __ldg(reinterpret_cast<const float4 *>(p) + q);
            out[4 * q + 0] = v.x; out[4 * q + 1] = v.y; out[4 * q + 2] = v.z; out[4 * q + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < K / 2; q++) {
            const double2 v = __ldg(reinterpret_cast<const double2 *>(p) + q);
            out[2 * q + 0] = v.x; out[2 * q + 1] = v.y;
        }
    }
}

template <typename R, int K>
__device__ __forceinline__ void vstore(R *p, const R (&in)[K])
{
    if (sizeof(R) == 4) {
#pragma unroll
        for (int q = 0; q < K / 4; q++)
            reinterpret_cast<float4 *>(p)[q] = make_float4(in[4 * q], in[4 * q + 1], in[4 * q + 2], in[4 * q + 3]);
    } else {
#pragma unroll
        for (int q = 0; q < K / 2; q++)
            reinterpret_cast<double2 *>(p)[q] = make_double2(in[2 * q], in[2 * q + 1]);
    }
}

// shuffles within the P-lane segment of a line
template <typename T>
__device__ __forceinline__ T sh_up(T v, int d, int P) { return __shfl_up_sync(0xffffffffu, v, d, P); }
template <typename T>
__device__ __forceinline__ T sh_down(T v, int d, int P) { return __shfl_down_sync(0xffffffffu, v, d, P); }

} // namespace

// FIT: dimz == P K with 16-byte vector chunks (the launcher checks), so every lane
// holds a whole aligned chunk and the general row-by-row paths compile away.
template <typename R, int K, int P, bool FIT>
__global__ void __launch_bounds__(128)
    sweep_zwarp_kernel(DomainView<R> d, int nlines, const int *__restrict__ line_lo, const int *__restrict__ line_hi,
                       CLayer<R> cur, CLayer<R> tin, Layer<R> next, Layer<R> tout, SweepConst<R> kc, int merges)
{
    constexpr int LPW = 32 / P;  // lines per warp
    // a K-row chunk can be moved as 16-byte vectors
    constexpr bool KVEC = (K * sizeof(R)) % 16 == 0;
    constexpr bool FITV = FIT && KVEC;
    const int lane = threadIdx.x & 31;
    const int ch = lane % P;
    const int line = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * LPW + lane / P;
    const int L = d.nz;
    bool has = false;
    long long base = 0;
    if (line < nlines) {
        has = line_lo[line] >= 0;
        base = (long long)line * L;
    }
    // a warp whose lines are all empty or beyond the grid leaves together
    if (!__any_sync(0xffffffffu, has)) return;
    const int p0 = ch * K;
    const long long off0 = base + p0;
    const long long sx = (long long)d.ny * d.nz, sy = d.nz;
    // rows of this lane inside the line; vector accesses for a whole chunk when
    // dimz keeps every chunk start 16-byte aligned
    const int nr = FITV ? K : (p0 >= L ? 0 : (p0 + K <= L ? K : L - p0));
    const bool vec = FITV || (KVEC && nr == K && (L % (16 / (int)sizeof(R))) == 0);

    // ---- loads: own rows, four off-line neighbour chunks, codes ----
    R tv[4][K], cu[4][K], wxp[K], wxm[K], wyp[K], wym[K];
    uint8_t cc[K];
#pragma unroll
    for (int v = 0; v < 4; v++)
#pragma unroll
        for (int i = 0; i < K; i++) { tv[v][i] = R(0); cu[v][i] = R(0); }
#pragma unroll
    for (int i = 0; i < K; i++) { wxp[i] = wxm[i] = wyp[i] = wym[i] = R(0); cc[i] = NODE_OUT; }
    const R *W = tin.f[2];
    if constexpr (KVEC) {
        if (has && vec) {
#pragma unroll
            for (int v = 0; v < 4; v++) {
                vload<R, K>(tin.f[v] + off0, tv[v]);
                vload<R, K>(cur.f[v] + off0, cu[v]);
            }
            vload<R, K>(W + off0 + sx, wxp);
            vload<R, K>(W + off0 - sx, wxm);
            vload<R, K>(W + off0 + sy, wyp);
            vload<R, K>(W + off0 - sy, wym);
        }
    }
    if (has && !vec) {
#pragma unroll
        for (int i = 0; i < K; i++)
            if (i < nr) {
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    tv[v][i] = __ldg(tin.f[v] + off0 + i);
                    cu[v][i] = __ldg(cur.f[v] + off0 + i);
                }
                wxp[i] = __ldg(W + off0 + i + sx);
                wxm[i] = __ldg(W + off0 + i - sx);
                wyp[i] = __ldg(W + off0 + i + sy);
                wym[i] = __ldg(W + off0 + i - sy);
            }
    }
    if (has) {
        if (K == 4 && (FITV || (nr == K && L % 4 == 0))) {
            const uint32_t c4 = __ldg(reinterpret_cast<const uint32_t *>(d.code + off0));
#pragma unroll
            for (int i = 0; i < K; i++) cc[i] = (c4 >> (8 * i)) & 0xff;
        } else if (K == 8 && (FITV || (nr == K && L % 8 == 0))) {
#pragma unroll
            for (int q = 0; q < K / 8; q++) {
                const uint2 c8 = __ldg(reinterpret_cast<const uint2 *>(d.code + off0) + q);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    cc[8 * q + i] = (c8.x >> (8 * i)) & 0xff;
                    cc[8 * q + 4 + i] = (c8.y >> (8 * i)) & 0xff;
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < K; i++)
                if (i < nr) cc[i] = __ldg(d.code + off0 + i);
        }
    }
    // halo rows from the neighbouring lanes of the line
    R hm[4], hp[4], cm_[4], cp_[4];
    uint8_t ccm, ccp;
#pragma unroll
    for (int v = 0; v < 4; v++) {
        hm[v] = sh_up(tv[v][K - 1], 1, P);
        hp[v] = sh_down(tv[v][0], 1, P);
        cm_[v] = sh_up(cu[v][K - 1], 1, P);
        cp_[v] = sh_down(cu[v][0], 1, P);
    }
    ccm = (uint8_t)sh_up((int)cc[K - 1], 1, P);
    ccp = (uint8_t)sh_down((int)cc[0], 1, P);
    if (ch == 0) { ccm = NODE_OUT; }
    if (ch == P - 1) { ccp = NODE_OUT; }

    // ---- rows ----
    bool inr[K + 2];
    inr[0] = code_is_in(ccm);
    inr[K + 1] = code_is_in(ccp);
#pragma unroll
    for (int i = 0; i < K; i++) inr[i + 1] = code_is_in(cc[i]);
    int kind[K];
    R rr[K], dv[4][K];
#pragma unroll
    for (int i = 0; i < K; i++) {
        kind[i] = zkind(inr[i], inr[i + 1], inr[i + 2]);
        rr[i] = R(0);
        const R tprev[4] = {i > 0 ? tv[0][i - 1] : hm[0], i > 0 ? tv[1][i - 1] : hm[1], i > 0 ? tv[2][i - 1] : hm[2],
                            i > 0 ? tv[3][i - 1] : hm[3]};
        const R tnext[4] = {i < K - 1 ? tv[0][i + 1] : hp[0], i < K - 1 ? tv[1][i + 1] : hp[1],
                            i < K - 1 ? tv[2][i + 1] : hp[2], i < K - 1 ? tv[3][i + 1] : hp[3]};
        if (kind[i] == Z_IN) {
            const R r = tv[2][i] * kc.inv_two_h;
            rr[i] = r;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const R vis = v < 3 ? kc.vis_v : kc.vis_t;
                const R cm = inr[i] ? (i > 0 ? cu[v][i - 1] : cm_[v]) : R(0);
                const R cp = inr[i + 2] ? (i < K - 1 ? cu[v][i + 1] : cp_[v]) : R(0);
                dv[v][i] = vis * (cm - R(2) * cu[v][i] + cp) - r * (cp - cm);
            }
            dv[2][i] -= kc.v_T * ((tnext[3] - tprev[3]) * kc.inv_two_h);
            const R fa = (tnext[0] - tprev[0]) * kc.inv_two_h;
            const R fb = (tnext[1] - tprev[1]) * kc.inv_two_h;
            const R fc = (tnext[2] - tprev[2]) * kc.inv_two_h;
            const R g1 = (wxp[i] - wxm[i]) * kc.inv_two_dx;
            const R g2 = (wyp[i] - wym[i]) * kc.inv_two_dy;
            // DissFuncZ (TimeLayer3D.h:578-588)
            dv[3][i] += kc.t_phi * (fa * fa + fb * fb + R(2) * fc * fc + fa * g1 + fb * g2);
        } else if (kind[i] == Z_NONE) {
#pragma unroll
            for (int v = 0; v < 4; v++) dv[v][i] = R(0);
        } else {
            const bool vf = (cc[i] & CODE_VEL_FREE) != 0, tf = (cc[i] & CODE_TEMP_FREE) != 0;
            const long long off = off0 + i;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const R nb = kind[i] == Z_END ? (i > 0 ? cu[v][i - 1] : cm_[v]) : (i < K - 1 ? cu[v][i + 1] : cp_[v]);
                const bool fr = v < 3 ? vf : tf;
                dv[v][i] = fr ? nb : (kc.nv_in_temp ? tv[v][i] : __ldg(d.nv[v] + off));
            }
        }
    }

    // ---- chunk elimination and reduced system (shared with the X/Y sweeps) ----
    unsigned freebits = 0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        if (cc[i] & CODE_VEL_FREE) freebits |= 1u << (2 * i);
        if (cc[i] & CODE_TEMP_FREE) freebits |= 2u << (2 * i);
    }
    R ea[2][K], ec[2][K];
    sweep::Reduced<R> red;
    sweep::eliminate<R, K>(kind, rr, freebits, kc, dv, ea, ec, red);
    R (&Al)[2] = red.Al, (&Cl)[2] = red.Cl, (&Dl)[4] = red.Dl;

    // ---- reduced system in shuffles ----
    R ea_[2], ec_[2], ed[4];
    {
        // cyclic-reduction step: chunk-last row of the previous lane
        R pv[8] = {sh_up(Al[0], 1, P), sh_up(Cl[0], 1, P), sh_up(Al[1], 1, P), sh_up(Cl[1], 1, P),
                   sh_up(Dl[0], 1, P), sh_up(Dl[1], 1, P), sh_up(Dl[2], 1, P), sh_up(Dl[3], 1, P)};
        if (ch == 0) {
#pragma unroll
            for (int q = 0; q < 8; q++) pv[q] = R(0);
        }
        sweep::cr_step<R>(red, pv, ea_, ec_, ed);
    }
#pragma unroll
    for (int s = 1; s < P; s <<= 1) {
        // lanes whose partner lies outside the line receive their own row from the
        // shuffle; their coupling to it is exactly zero (first row a = 0, last row
        // c = 0, preserved by every step), so the finite values drop out.
        const R mv[8] = {sh_up(ea_[0], s, P), sh_up(ec_[0], s, P), sh_up(ea_[1], s, P), sh_up(ec_[1], s, P),
                         sh_up(ed[0], s, P),  sh_up(ed[1], s, P),  sh_up(ed[2], s, P),  sh_up(ed[3], s, P)};
        const R pv[8] = {sh_down(ea_[0], s, P), sh_down(ec_[0], s, P), sh_down(ea_[1], s, P), sh_down(ec_[1], s, P),
                         sh_down(ed[0], s, P),  sh_down(ed[1], s, P),  sh_down(ed[2], s, P),  sh_down(ed[3], s, P)};
        sweep::pcr_update<R>(mv, pv, ea_, ec_, ed);
    }
    R xf[4], xl[4];
#pragma unroll
    for (int v = 0; v < 4; v++) {
        R nf = sh_down(ed[v], 1, P);
        if (ch == P - 1) nf = R(0);
        xf[v] = ed[v];
        const int m = v < 3 ? 0 : 1;
        xl[v] = Dl[v] - Al[m] * xf[v] - Cl[m] * nf;
    }
    if (!has) return;

    // ---- write-back ----
    // merged nonlinear value: (temp + x) / 2, or with the extra merge (temp + 3 x) / 4
    const R gw_new = merges == 2 ? R(0.75) : R(0.5), gw_old = R(1) - gw_new;
    R xo[4][K], mo[4][K];
    bool all_seg = true, all_in = true;
#pragma unroll
    for (int i = 0; i < K; i++) {
        all_seg = all_seg && kind[i] != Z_NONE;
        all_in = all_in && kind[i] == Z_IN;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int m = v < 3 ? 0 : 1;
            R x = i == 0 ? xf[v] : (i == K - 1 ? xl[v] : dv[v][i] - ea[m][i] * xf[v] - ec[m][i] * xl[v]);
            if (kind[i] == Z_IN) x += cu[v][i];
            xo[v][i] = x;
            mo[v][i] = fma(x, gw_new, tv[v][i] * gw_old);
        }
    }
    // (padding rows are NONE: the row at L-1 is never IN, so the row at L is not a
    // segment end)
    bool done_next = false, done_tout = false;
    if constexpr (KVEC) {
        if (vec && all_seg) {
#pragma unroll
            for (int v = 0; v < 4; v++) vstore<R, K>(next.f[v] + off0, xo[v]);
            done_next = true;
        }
        if (vec && all_in) {
#pragma unroll
            for (int v = 0; v < 4; v++) vstore<R, K>(tout.f[v] + off0, mo[v]);
            done_tout = true;
        }
    }
    if (!done_next) {
#pragma unroll
        for (int i = 0; i < K; i++)
            if (kind[i] != Z_NONE) {
#pragma unroll
                for (int v = 0; v < 4; v++) next.f[v][off0 + i] = xo[v][i];
            }
    }
    if (!done_tout) {
#pragma unroll
        for (int i = 0; i < K; i++)
            if (kind[i] == Z_IN) {
#pragma unroll
                for (int v = 0; v < 4; v++) tout.f[v][off0 + i] = mo[v][i];
            }
    }
}

// Lanes per line: the smallest of 4, 8, 16, 32 whose chunks cover dimz (0: none).
int zwarp_lanes(int nz, int K)
{
    if (K != 4 && K != 5 && K != 8 && K != 12) return 0;
    for (int P = 4; P <= 32; P *= 2)
        if (P * K >= nz) return P;
    return 0;
}

// K = 12 is compiled for lines of 257 to 384 rows only (32 lanes), and only in
// FP32: in FP64 its rows do not fit in the registers.
bool zwarp_supported(int nz, int K, int elem_bytes)
{
    if (K == 12 && (elem_bytes != 4 || zwarp_lanes(nz, K) != 32 || nz <= 256)) return false;
    return nz >= 1 && zwarp_lanes(nz, K) > 0;
}

template <typename R>
cudaError_t launch_sweep_zwarp(const DomainView<R> &d, const int *line_lo, const int *line_hi, CLayer<R> cur,
                               CLayer<R> tin, Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges,
                               int K, cudaStream_t s)
{
    if (!zwarp_supported(d.nz, K, (int)sizeof(R))) return cudaErrorInvalidConfiguration;
    for (int v = 0; v < 4; v++)
        if (((uintptr_t)cur.f[v] | (uintptr_t)tin.f[v] | (uintptr_t)next.f[v] | (uintptr_t)tout.f[v]) % 16)
            return cudaErrorInvalidConfiguration;
    const int nlines = d.nx * d.ny;
    const int P = zwarp_lanes(d.nz, K);
    const int lines_per_block = 4 * (32 / P);  // 4 warps per block
    const int blocks = (nlines + lines_per_block - 1) / lines_per_block;
    const bool fit = d.nz == P * K && (K * sizeof(R)) % 16 == 0;
#define ZL(KK, PP)                                                                                              \
    if (K == KK && P == PP) {                                                                                   \
        if (fit)                                                                                                \
            sweep_zwarp_kernel<R, KK, PP, true><<<blocks, 128, 0, s>>>(d, nlines, line_lo, line_hi, cur, tin, next, \
                                                                      tout, k, merges);                         \
        else                                                                                                    \
            sweep_zwarp_kernel<R, KK, PP, false><<<blocks, 128, 0, s>>>(d, nlines, line_lo, line_hi, cur, tin,     \
                                                                       next, tout, k, merges);                  \
        return cudaGetLastError();                                                                              \
    }
    ZL(4, 4) ZL(4, 8) ZL(4, 16) ZL(4, 32) ZL(5, 4) ZL(5, 8) ZL(5, 16) ZL(5, 32) ZL(8, 4) ZL(8, 8) ZL(8, 16) ZL(8, 32)
    if constexpr (sizeof(R) == 4) {
        ZL(12, 32)
    }
#undef ZL
    return cudaErrorInvalidConfiguration;
}

template cudaError_t launch_sweep_zwarp<float>(const DomainView<float> &, const int *, const int *, CLayer<float>,
                                               CLayer<float>, Layer<float>, Layer<float>, const SweepConst<float> &,
                                               int, int, cudaStream_t);
template cudaError_t launch_sweep_zwarp<double>(const DomainView<double> &, const int *, const int *, CLayer<double>,
                                                CLayer<double>, Layer<double>, Layer<double>,
                                                const SweepConst<double> &, int, int, cudaStream_t);

} // namespace adi
