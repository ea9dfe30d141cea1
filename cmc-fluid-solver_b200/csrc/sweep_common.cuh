// Device building blocks shared by the fast sweep kernels (sweep_fast.cu,
// sweep_zwarp.cu, sweep_xytma.cu, sweep_xypair.cu) and the chunked adjoint sweep
// (adjoint_fast.cu).  In float the chunk elimination, the cyclic-reduction step and
// the PCR updates run in packed FP32 (sm_100 two-lane FMA/MUL), the velocity and
// temperature matrices (and the field pairs U,T / V,W) side by side.
//
// A chunk is K consecutive rows of one line system.  Row kinds follow the
// segment structure of Grid3D::GenerateListSegments (Grid3D.cpp:47-127): an IN
// node is an interior row (BuildMatrix, AdiSolver3D.cpp:755-801); the non-IN node
// before a run of IN nodes starts a segment (ApplyBC0, :804-827); the non-IN node
// after it ends the segment (ApplyBC1, :829-852); a non-IN node between two runs
// does both (Dirichlet by the solver contract); any other node has no row.
#pragma once

#include "adi_internal.cuh"

namespace adi {
namespace sweep {

enum : int { R_NONE = 0, R_START = 1, R_IN = 2, R_END = 3, R_SHARED = 4 };

__device__ __forceinline__ int row_kind(bool inm, bool in0, bool inp)
{
    if (in0) return R_IN;
    if (inm && inp) return R_SHARED;
    if (inp) return R_START;
    if (inm) return R_END;
    return R_NONE;
}

// Reciprocal: float uses the hardware approximation refined by one Newton-Raphson
// step r' = r + r(1 - x r); double uses IEEE division.
template <typename R>
__device__ __forceinline__ R rcp(R x)
{
    return R(1) / x;
}
template <>
__device__ __forceinline__ float rcp<float>(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return fmaf(r, fmaf(-x, r, 1.0f), r);
}

// Packed FP32 (two lanes per instruction, sm_100): lane x carries the velocity
// matrix (or variable U / V), lane y the temperature matrix (or T / W).
__device__ __forceinline__ float2 p2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 rcp2(float2 x)
{
    float2 r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(x.x));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(x.y));
    return fma2(r, fma2(neg2(x), r, bc2(1.0f)), r);   // one Newton-Raphson step per lane
}

// Matrix entries of one row of matrix m (velocity or temperature).
template <typename R>
__device__ __forceinline__ void row_abc(int kd, R r, bool free_bc, R vis, R b_in, R &a, R &b, R &c)
{
    if (kd == R_IN) {
        a = -r - vis;
        b = b_in;
        c = r - vis;
    } else if (kd == R_NONE) {
        a = R(0); b = R(1); c = R(0);
    } else {
        const bool first = kd != R_END;
        b = free_bc ? R(2) : R(1);
        a = (!first && free_bc) ? R(-1) : R(0);
        c = (first && free_bc) ? R(-1) : R(0);
    }
}

// The reduced rows of one chunk.  Unknowns of the line's reduced system are
// ordered (first0, last0, first1, last1, ...); rows are normalised (diagonal 1):
//   first: Af x(last of previous chunk) + x(first) + Cf x(last)   = Df
//   last:  Al x(first)                  + x(last)  + Cl x(first of next) = Dl
// Index m: 0 velocity matrix, 1 temperature matrix; D per variable U V W T.
template <typename R>
struct Reduced {
    R Af[2], Cf[2], Al[2], Cl[2], Df[4], Dl[4];
};

// Eliminates the interior rows 1..K-2 of a chunk so that each interior unknown is
// x_i = dv_i - ea_i x_first - ec_i x_last (per matrix), and forms the reduced rows.
// kind[i], rr[i] (advection term of IN rows), freebits (bit 2i velocity BC FREE,
// bit 2i+1 temperature) describe the rows; dv holds the right-hand sides on entry
// and d'' on exit.
// The same elimination in packed FP32: both matrices advance together (lanes x, y),
// and so do the right-hand sides (U, T) and (V, W).
template <int K>
__device__ __forceinline__ void eliminate_x2(const int (&kind)[K], const float (&rr)[K], unsigned freebits,
                                             const SweepConst<float> &kc, float (&dv)[4][K], float (&ea)[2][K],
                                             float (&ec)[2][K], Reduced<float> &red)
{
    float2 nA[K], B[K], C[K], EA[K], EC[K], D03[K], D12[K];
#pragma unroll
    for (int i = 0; i < K; i++) {
        float a0, b0, c0, a1, b1, c1;
        row_abc<float>(kind[i], rr[i], (freebits >> (2 * i)) & 1u, kc.vis_v, kc.b_v, a0, b0, c0);
        row_abc<float>(kind[i], rr[i], (freebits >> (2 * i + 1)) & 1u, kc.vis_t, kc.b_t, a1, b1, c1);
        nA[i] = p2(-a0, -a1);
        B[i] = p2(b0, b1);
        C[i] = p2(c0, c1);
        D03[i] = p2(dv[0][i], dv[3][i]);
        D12[i] = p2(dv[1][i], dv[2][i]);
    }
    {
        const float2 r = rcp2(B[1]);
        EA[1] = mul2(neg2(nA[1]), r);
        EC[1] = mul2(C[1], r);
        D03[1] = mul2(D03[1], r);
        D12[1] = mul2(D12[1], bc2(r.x));
    }
#pragma unroll
    for (int i = 2; i <= K - 2; i++) {
        const float2 r = rcp2(fma2(nA[i], EC[i - 1], B[i]));
        D03[i] = mul2(fma2(nA[i], D03[i - 1], D03[i]), r);
        D12[i] = mul2(fma2(bc2(nA[i].x), D12[i - 1], D12[i]), bc2(r.x));
        EA[i] = mul2(mul2(nA[i], EA[i - 1]), r);
        EC[i] = mul2(C[i], r);
    }
#pragma unroll
    for (int i = K - 3; i >= 1; i--) {
        const float2 nci = neg2(EC[i]);
        EA[i] = fma2(nci, EA[i + 1], EA[i]);
        D03[i] = fma2(nci, D03[i + 1], D03[i]);
        D12[i] = fma2(bc2(nci.x), D12[i + 1], D12[i]);
        EC[i] = mul2(nci, EC[i + 1]);
    }
    const float2 nC0 = neg2(C[0]);
    const float2 rf = rcp2(fma2(nC0, EA[1], B[0]));
    const float2 rl = rcp2(fma2(nA[K - 1], EC[K - 2], B[K - 1]));
    const float2 Af = mul2(neg2(nA[0]), rf), Cf = mul2(mul2(nC0, EC[1]), rf);
    const float2 Al = mul2(mul2(nA[K - 1], EA[K - 2]), rl), Cl = mul2(C[K - 1], rl);
    const float2 Df03 = mul2(fma2(nC0, D03[1], D03[0]), rf);
    const float2 Df12 = mul2(fma2(bc2(nC0.x), D12[1], D12[0]), bc2(rf.x));
    const float2 Dl03 = mul2(fma2(nA[K - 1], D03[K - 2], D03[K - 1]), rl);
    const float2 Dl12 = mul2(fma2(bc2(nA[K - 1].x), D12[K - 2], D12[K - 1]), bc2(rl.x));
    red.Af[0] = Af.x; red.Af[1] = Af.y; red.Cf[0] = Cf.x; red.Cf[1] = Cf.y;
    red.Al[0] = Al.x; red.Al[1] = Al.y; red.Cl[0] = Cl.x; red.Cl[1] = Cl.y;
    red.Df[0] = Df03.x; red.Df[3] = Df03.y; red.Df[1] = Df12.x; red.Df[2] = Df12.y;
    red.Dl[0] = Dl03.x; red.Dl[3] = Dl03.y; red.Dl[1] = Dl12.x; red.Dl[2] = Dl12.y;
#pragma unroll
    for (int i = 1; i <= K - 2; i++) {
        ea[0][i] = EA[i].x; ea[1][i] = EA[i].y;
        ec[0][i] = EC[i].x; ec[1][i] = EC[i].y;
        dv[0][i] = D03[i].x; dv[3][i] = D03[i].y;
        dv[1][i] = D12[i].x; dv[2][i] = D12[i].y;
    }
}

template <typename R, int K>
__device__ __forceinline__ void eliminate(const int (&kind)[K], const R (&rr)[K], unsigned freebits,
                                          const SweepConst<R> &kc, R (&dv)[4][K], R (&ea)[2][K], R (&ec)[2][K],
                                          Reduced<R> &red)
{
    static_assert(K >= 3, "chunks of at least three rows");
    if constexpr (sizeof(R) == 4) {
        eliminate_x2<K>(kind, rr, freebits, kc, dv, ea, ec, red);
    } else {
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const R vis = m == 0 ? kc.vis_v : kc.vis_t;
            const R bin = m == 0 ? kc.b_v : kc.b_t;
            R A[K], B[K], C[K];
#pragma unroll
            for (int i = 0; i < K; i++)
                row_abc<R>(kind[i], rr[i], (freebits >> (2 * i + m)) & 1u, vis, bin, A[i], B[i], C[i]);
            {
                const R r = rcp<R>(B[1]);
                ea[m][1] = A[1] * r;
                ec[m][1] = C[1] * r;
                if (m == 0) { dv[0][1] *= r; dv[1][1] *= r; dv[2][1] *= r; }
                else dv[3][1] *= r;
            }
#pragma unroll
            for (int i = 2; i <= K - 2; i++) {
                const R r = rcp<R>(B[i] - A[i] * ec[m][i - 1]);
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
            const R rf = rcp<R>(B[0] - C[0] * ea[m][1]);
            red.Af[m] = A[0] * rf;
            red.Cf[m] = -C[0] * ec[m][1] * rf;
            const R rl = rcp<R>(B[K - 1] - A[K - 1] * ec[m][K - 2]);
            red.Al[m] = -A[K - 1] * ea[m][K - 2] * rl;
            red.Cl[m] = C[K - 1] * rl;
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) {
                    red.Df[v] = (dv[v][0] - C[0] * dv[v][1]) * rf;
                    red.Dl[v] = (dv[v][K - 1] - A[K - 1] * dv[v][K - 2]) * rl;
                }
            } else {
                red.Df[3] = (dv[3][0] - C[0] * dv[3][1]) * rf;
                red.Dl[3] = (dv[3][K - 1] - A[K - 1] * dv[3][K - 2]) * rl;
            }
        }
    }
}

// eliminate() for explicitly given rows: A, B, C per matrix m (sub-diagonal,
// diagonal, super-diagonal of each of the chunk's K rows), right-hand sides dv
// (velocity columns 0-2 use m = 0, column 3 uses m = 1).  Used by the adjoint,
// whose transposed rows are not of the BuildMatrix / ApplyBC form.
template <typename R, int K>
__device__ __forceinline__ void eliminate_abc(const R (&A)[2][K], const R (&B)[2][K], const R (&C)[2][K],
                                              R (&dv)[4][K], R (&ea)[2][K], R (&ec)[2][K], Reduced<R> &red)
{
    static_assert(K >= 3, "chunks of at least three rows");
#pragma unroll
    for (int m = 0; m < 2; m++) {
        {
            const R r = rcp<R>(B[m][1]);
            ea[m][1] = A[m][1] * r;
            ec[m][1] = C[m][1] * r;
            if (m == 0) { dv[0][1] *= r; dv[1][1] *= r; dv[2][1] *= r; }
            else dv[3][1] *= r;
        }
#pragma unroll
        for (int i = 2; i <= K - 2; i++) {
            const R r = rcp<R>(B[m][i] - A[m][i] * ec[m][i - 1]);
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) dv[v][i] = (dv[v][i] - A[m][i] * dv[v][i - 1]) * r;
            } else {
                dv[3][i] = (dv[3][i] - A[m][i] * dv[3][i - 1]) * r;
            }
            ea[m][i] = -A[m][i] * ea[m][i - 1] * r;
            ec[m][i] = C[m][i] * r;
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
        const R rf = rcp<R>(B[m][0] - C[m][0] * ea[m][1]);
        red.Af[m] = A[m][0] * rf;
        red.Cf[m] = -C[m][0] * ec[m][1] * rf;
        const R rl = rcp<R>(B[m][K - 1] - A[m][K - 1] * ec[m][K - 2]);
        red.Al[m] = -A[m][K - 1] * ea[m][K - 2] * rl;
        red.Cl[m] = C[m][K - 1] * rl;
        if (m == 0) {
#pragma unroll
            for (int v = 0; v < 3; v++) {
                red.Df[v] = (dv[v][0] - C[m][0] * dv[v][1]) * rf;
                red.Dl[v] = (dv[v][K - 1] - A[m][K - 1] * dv[v][K - 2]) * rl;
            }
        } else {
            red.Df[3] = (dv[3][0] - C[m][0] * dv[3][1]) * rf;
            red.Dl[3] = (dv[3][K - 1] - A[m][K - 1] * dv[3][K - 2]) * rl;
        }
    }
}

// Cyclic-reduction step on the chunk-first row, given the previous chunk's last
// row (pv: Al[0] Cl[0] Al[1] Cl[1] Dl[0..3], zeros for the first chunk).  Returns
// the row of x(first) coupled to x(first) of the neighbouring chunks, normalised.
template <typename R>
__device__ __forceinline__ void cr_step(const Reduced<R> &red, const R (&pv)[8], R (&ea)[2], R (&ec)[2], R (&ed)[4])
{
    if constexpr (sizeof(R) == 4) {
        const float2 nAf = p2(-red.Af[0], -red.Af[1]), nCf = p2(-red.Cf[0], -red.Cf[1]);
        const float2 Al = p2(red.Al[0], red.Al[1]), Cl = p2(red.Cl[0], red.Cl[1]);
        const float2 r = rcp2(fma2(nCf, Al, fma2(nAf, p2(pv[1], pv[3]), bc2(1.0f))));
        const float2 a2 = mul2(mul2(nAf, p2(pv[0], pv[2])), r), c2 = mul2(mul2(nCf, Cl), r);
        const float2 e03 = mul2(fma2(nCf, p2(red.Dl[0], red.Dl[3]), fma2(nAf, p2(pv[4], pv[7]),
                                                                            p2(red.Df[0], red.Df[3]))), r);
        const float2 e12 = mul2(fma2(bc2(nCf.x), p2(red.Dl[1], red.Dl[2]),
                                     fma2(bc2(nAf.x), p2(pv[5], pv[6]), p2(red.Df[1], red.Df[2]))), bc2(r.x));
        ea[0] = a2.x; ea[1] = a2.y; ec[0] = c2.x; ec[1] = c2.y;
        ed[0] = e03.x; ed[3] = e03.y; ed[1] = e12.x; ed[2] = e12.y;
    } else {
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const R pA = pv[2 * m], pC = pv[2 * m + 1];
            const R r = rcp<R>(R(1) - red.Af[m] * pC - red.Cf[m] * red.Al[m]);
            ea[m] = -red.Af[m] * pA * r;
            ec[m] = -red.Cf[m] * red.Cl[m] * r;
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) ed[v] = (red.Df[v] - red.Af[0] * pv[4 + v] - red.Cf[0] * red.Dl[v]) * r;
            } else {
                ed[3] = (red.Df[3] - red.Af[1] * pv[7] - red.Cf[1] * red.Dl[3]) * r;
            }
        }
    }
}

// One parallel-cyclic-reduction update of a normalised row (ea, ec, ed) with the
// rows at distance s below (mv) and above (pv), each packed as a0 c0 a1 c1 d0..d3.
template <typename R>
__device__ __forceinline__ void pcr_update(const R (&mv)[8], const R (&pv)[8], R (&ea)[2], R (&ec)[2], R (&ed)[4])
{
    if constexpr (sizeof(R) == 4) {
        const float2 na = p2(-ea[0], -ea[1]), nc = p2(-ec[0], -ec[1]);
        const float2 r = rcp2(fma2(nc, p2(pv[0], pv[2]), fma2(na, p2(mv[1], mv[3]), bc2(1.0f))));
        const float2 e03 = mul2(fma2(nc, p2(pv[4], pv[7]), fma2(na, p2(mv[4], mv[7]), p2(ed[0], ed[3]))), r);
        const float2 e12 =
            mul2(fma2(bc2(nc.x), p2(pv[5], pv[6]), fma2(bc2(na.x), p2(mv[5], mv[6]), p2(ed[1], ed[2]))), bc2(r.x));
        const float2 a2 = mul2(mul2(na, p2(mv[0], mv[2])), r), c2 = mul2(mul2(nc, p2(pv[1], pv[3])), r);
        ed[0] = e03.x; ed[3] = e03.y; ed[1] = e12.x; ed[2] = e12.y;
        ea[0] = a2.x; ea[1] = a2.y; ec[0] = c2.x; ec[1] = c2.y;
    } else {
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const R a = ea[m], c = ec[m];
            const R r = rcp<R>(R(1) - a * mv[2 * m + 1] - c * pv[2 * m]);
            if (m == 0) {
#pragma unroll
                for (int v = 0; v < 3; v++) ed[v] = (ed[v] - a * mv[4 + v] - c * pv[4 + v]) * r;
            } else {
                ed[3] = (ed[3] - a * mv[7] - c * pv[7]) * r;
            }
            ea[m] = -a * mv[2 * m] * r;
            ec[m] = -c * pv[2 * m + 1] * r;
        }
    }
}

// 8-value slot store / load with 16-byte accesses (slot must be 16-byte aligned).
template <typename R>
__device__ __forceinline__ void slot_store(R *p, R v0, R v1, R v2, R v3, R v4, R v5, R v6, R v7)
{
    if (sizeof(R) == 4) {
        float4 *q = reinterpret_cast<float4 *>(p);
        q[0] = make_float4(v0, v1, v2, v3);
        q[1] = make_float4(v4, v5, v6, v7);
    } else {
        double2 *q = reinterpret_cast<double2 *>(p);
        q[0] = make_double2(v0, v1);
        q[1] = make_double2(v2, v3);
        q[2] = make_double2(v4, v5);
        q[3] = make_double2(v6, v7);
    }
}

template <typename R>
__device__ __forceinline__ void slot_load(const R *p, R (&v)[8])
{
    if (sizeof(R) == 4) {
        const float4 *q = reinterpret_cast<const float4 *>(p);
        const float4 a = q[0], b = q[1];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
        const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const double2 a = q[i];
            v[2 * i] = a.x;
            v[2 * i + 1] = a.y;
        }
    }
}

} // namespace sweep
} // namespace adi
