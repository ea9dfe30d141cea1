// Whole-layer kernels around the sweeps: boundary refresh, the per-step layer
// set-up, the standalone merge, the divergence error and the GetLayer fill.
// All are streaming HBM kernels: one pass, grid-stride, coalesced.
#include "adi_internal.cuh"

namespace adi {

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }

static int grid_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    long long cap = 148LL * 16;  // 16 resident 256-thread blocks per SM
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

// cur[BOUND|VALVE] = node values.  CPU semantics of UpdateBoundaries
// (Solver3D.cpp:27-34 / AdiSolver3D.cpp:290-294: CopyFromGrid for BOUND and VALVE).
template <typename R>
__global__ void update_boundaries_kernel(DomainView<R> d, Layer<R> cur)
{
    for (long long i = gtid(); i < d.n; i += gstride()) {
        if (code_is_bv(d.code[i])) {
#pragma unroll
            for (int v = 0; v < 4; v++) cur.f[v][i] = d.nv[v][i];
        }
    }
}

// Start of TimeStep (AdiSolver3D.cpp:310-320): next[BOUND|VALVE] = cur and
// temp = cur.  Both temp buffers of the double-buffered nonlinear layer get the
// copy, because the sweeps only ever write IN nodes of the buffer they fill.
// With update_boundaries, cur[BOUND|VALVE] is first refreshed from the node values
// (the driver calls UpdateBoundaries right before TimeStep, FluidSolver3D.cpp:241-242).
//
// bv_only (a step whose first sweep reads cur itself as its nonlinear layer, so
// the copy temp = cur is needed only where no sweep writes temp): cells that are
// not BOUND / VALVE are left alone.  The nonlinear buffers then differ from cur
// only where no sweep reads them: NODE_IN cells, which the first sweep reads from
// cur and every sweep writes before the next one reads them, and NODE_OUT cells,
// which no stencil of a NODE_IN row reaches.
template <typename R>
__device__ __forceinline__ void step_begin_at(const DomainView<R> &d, const Layer<R> &cur, const Layer<R> &next,
                                              const Layer<R> &ta, const Layer<R> &tb, bool update_boundaries,
                                              long long i, bool bv_only = false)
{
    bool bv = code_is_bv(d.code[i]);
    if (bv_only && !bv) return;
#pragma unroll
    for (int v = 0; v < 4; v++) {
        R x;
        if (update_boundaries && bv) {
            x = d.nv[v][i];
            cur.f[v][i] = x;
        } else {
            x = cur.f[v][i];
        }
        if (bv) next.f[v][i] = x;
        ta.f[v][i] = x;
        tb.f[v][i] = x;
    }
}

template <typename R>
__global__ void step_begin_kernel(DomainView<R> d, Layer<R> cur, Layer<R> next, Layer<R> ta, Layer<R> tb,
                                  bool update_boundaries, bool bv_only)
{
    for (long long i = gtid(); i < d.n; i += gstride())
        step_begin_at(d, cur, next, ta, tb, update_boundaries, i, bv_only);
}

// step_begin_at for four consecutive cells with 16-byte accesses (n a multiple
// of 4, every array 16-byte aligned; checked by the launcher).  Same values as
// four step_begin_at calls; cur and next are written only where those write.
// bv_only skips groups of four without a BOUND / VALVE cell and copies the groups
// with one whole (the extra temp cells are ones no sweep reads before writing).
template <typename R>
__global__ void step_begin_vec4_kernel(DomainView<R> d, Layer<R> cur, Layer<R> next, Layer<R> ta, Layer<R> tb,
                                       bool update_boundaries, bool bv_only)
{
    const long long n4 = d.n / 4;
    for (long long q = gtid(); q < n4; q += gstride()) {
        const long long i = 4 * q;
        const uint32_t c4 = __ldg(reinterpret_cast<const uint32_t *>(d.code + i));
        bool bv[4];
        bool any = false;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            bv[e] = code_is_bv((uint8_t)(c4 >> (8 * e)));
            any |= bv[e];
        }
        if (bv_only && !any) continue;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            R x[4];
            if (sizeof(R) == 4) {
                const float4 a = *reinterpret_cast<const float4 *>(cur.f[v] + i);
                x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
            } else {
                const double2 a = *reinterpret_cast<const double2 *>(cur.f[v] + i);
                const double2 b = *reinterpret_cast<const double2 *>(cur.f[v] + i + 2);
                x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
            }
            if (update_boundaries && any) {
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (bv[e]) {
                        x[e] = d.nv[v][i + e];
                        cur.f[v][i + e] = x[e];
                    }
            }
            if (any) {
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (bv[e]) next.f[v][i + e] = x[e];
            }
            if (sizeof(R) == 4) {
                const float4 a = make_float4((float)x[0], (float)x[1], (float)x[2], (float)x[3]);
                *reinterpret_cast<float4 *>(ta.f[v] + i) = a;
                *reinterpret_cast<float4 *>(tb.f[v] + i) = a;
            } else {
                const double2 a = make_double2((double)x[0], (double)x[1]), b = make_double2((double)x[2], (double)x[3]);
                *reinterpret_cast<double2 *>(ta.f[v] + i) = a;
                *reinterpret_cast<double2 *>(ta.f[v] + i + 2) = b;
                *reinterpret_cast<double2 *>(tb.f[v] + i) = a;
                *reinterpret_cast<double2 *>(tb.f[v] + i + 2) = b;
            }
        }
    }
}

template <typename R>
__device__ __forceinline__ Layer<R> batch_layer(const BatchDomain<R> &bd, int l)
{
    Layer<R> x;
#pragma unroll
    for (int v = 0; v < 4; v++) x.f[v] = bd.L[l][v];
    return x;
}

// The step start of every domain of a batch in one launch: blockIdx.y picks the
// domain, blockIdx.x / threadIdx.x stride over its cells.
template <typename R>
__global__ void step_begin_batch_kernel(const BatchDomain<R> *__restrict__ doms, int cur, int nxt, int ta, int tb,
                                        bool update_boundaries)
{
    const BatchDomain<R> &bd = doms[blockIdx.y];
    const Layer<R> c = batch_layer(bd, cur), n = batch_layer(bd, nxt), a = batch_layer(bd, ta), b = batch_layer(bd, tb);
    for (long long i = gtid(); i < bd.d.n; i += gstride()) step_begin_at(bd.d, c, n, a, b, update_boundaries, i);
}

// dest = (dest + src) / 2 where type == IN (TimeLayer3D.h:415-436).
template <typename R>
__global__ void merge_kernel(DomainView<R> d, CLayer<R> src, Layer<R> dest)
{
    for (long long i = gtid(); i < d.n; i += gstride()) {
        if (code_is_in(d.code[i])) {
#pragma unroll
            for (int v = 0; v < 4; v++) dest.f[v][i] = (dest.f[v][i] + src.f[v][i]) / R(2);
        }
    }
}

// TimeLayer3D::EvalDivError (TimeLayer3D.h:595-641).  The eight-corner sums are
// formed in the working precision, in the reference's operand order, then scaled
// and accumulated in double.  Per-block partial sums are reduced in a fixed order
// by a second single-block kernel, so the result is deterministic; it differs from
// the reference's sequential double sum only by summation order.
// Adds cell id's term of the divergence error to acc / cnt (IN cells off the
// upper faces only).
template <typename R>
__device__ __forceinline__ void div_cell(const DomainView<R> &d, const CLayer<R> &l, R dx, R dy, R dz, long long id,
                                         double &acc, unsigned long long &cnt)
{
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const long long sx = (long long)ny * nz, sy = nz;
    const R *U = l.f[0], *V = l.f[1], *W = l.f[2];
    int k = (int)(id % nz);
    long long r = id / nz;
    int j = (int)(r % ny);
    int i = (int)(r / ny);
    if (i >= nx - 1 || j >= ny - 1 || k >= nz - 1) return;
    if (!code_is_in(d.code[id])) return;
    // E(i,j,k) with the offsets the reference uses; IN nodes never sit on the
    // frame (solver contract), so i-1, j-1, k-1 >= 0.
#define E_(A, di, dj, dk) A[id + (di) * sx + (dj) * sy + (dk)]
    double err_x = (double)((R)((R)((R)((R)((R)((R)((R)(E_(U, 0, 0, 0) + E_(U, 0, -1, 0)) + E_(U, 0, -1, -1)) + E_(U, 0, 0, -1)) -
                            E_(U, -1, 0, 0)) - E_(U, -1, -1, 0)) - E_(U, -1, -1, -1)) - E_(U, -1, 0, -1)) * dz * dy) / 4.0;
    double err_y = (double)((R)((R)((R)((R)((R)((R)((R)(E_(V, 0, 0, 0) + E_(V, -1, 0, 0)) + E_(V, -1, 0, -1)) + E_(V, 0, 0, -1)) -
                            E_(V, 0, -1, 0)) - E_(V, -1, -1, 0)) - E_(V, -1, -1, -1)) - E_(V, 0, -1, -1)) * dx * dz) / 4.0;
    double err_z = (double)((R)((R)((R)((R)((R)((R)((R)(E_(W, 0, 0, 0) + E_(W, 0, -1, 0)) + E_(W, -1, -1, 0)) + E_(W, -1, 0, 0)) -
                            E_(W, 0, 0, -1)) - E_(W, 0, -1, -1)) - E_(W, -1, -1, -1)) - E_(W, -1, 0, -1)) * dx * dy) / 4.0;
#undef E_
    acc += fabs(err_x + err_y + err_z);
    cnt++;
}

// Block sum of (acc, cnt) in a fixed tree order into psum[slot], pcnt[slot].
__device__ __forceinline__ void block_sum_to(double acc, unsigned long long cnt, double *psum,
                                             unsigned long long *pcnt, long long slot)
{
    __shared__ double s_sum[256];
    __shared__ unsigned long long s_cnt[256];
    s_sum[threadIdx.x] = acc;
    s_cnt[threadIdx.x] = cnt;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s_sum[threadIdx.x] += s_sum[threadIdx.x + w];
            s_cnt[threadIdx.x] += s_cnt[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        psum[slot] = s_sum[0];
        pcnt[slot] = s_cnt[0];
    }
}

template <typename R>
__global__ void div_error_partial_kernel(DomainView<R> d, CLayer<R> l, R dx, R dy, R dz, double *psum,
                                         unsigned long long *pcnt)
{
    double acc = 0.0;
    unsigned long long cnt = 0;
    for (long long id = gtid(); id < d.n; id += gstride()) div_cell(d, l, dx, dy, dz, id, acc, cnt);
    block_sum_to(acc, cnt, psum, pcnt, blockIdx.x);
}

// Per-domain partial sums of a batch: blockIdx.y picks the domain; partials land
// at [domain][blockIdx.x].
template <typename R>
__global__ void div_error_batch_partial_kernel(const BatchDomain<R> *__restrict__ doms, int layer, double *psum,
                                               unsigned long long *pcnt)
{
    const BatchDomain<R> &bd = doms[blockIdx.y];
    CLayer<R> l;
#pragma unroll
    for (int v = 0; v < 4; v++) l.f[v] = bd.L[layer][v];
    double acc = 0.0;
    unsigned long long cnt = 0;
    for (long long id = gtid(); id < bd.d.n; id += gstride())
        div_cell(bd.d, l, (R)bd.dx, (R)bd.dy, (R)bd.dz, id, acc, cnt);
    block_sum_to(acc, cnt, psum, pcnt, (long long)blockIdx.y * gridDim.x + blockIdx.x);
}

__global__ void div_error_final_kernel(const double *psum, const unsigned long long *pcnt, int nblocks,
                                       double *out_sum, unsigned long long *out_cnt)
{
    // one warp per reduction: block b folds partials [b * nblocks, (b + 1) * nblocks)
    psum += (long long)blockIdx.x * nblocks;
    pcnt += (long long)blockIdx.x * nblocks;
    out_sum += blockIdx.x;
    out_cnt += blockIdx.x;
    const int lane = threadIdx.x;
    double s = 0.0;
    unsigned long long c = 0;
    for (int b = lane; b < nblocks; b += 32) {
        s += psum[b];
        c += pcnt[b];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
        *out_sum = s;
        *out_cnt = c;
    }
}

// Nonlinear-iteration residual: the largest |x - t| and |x| over NODE_IN cells and
// the four fields, where x is the layer a global iteration produced and t the
// nonlinear layer its last sweep linearised about.  Each thread keeps running
// maxima over a grid-stride range, a warp combines them with shuffles, and lane 0
// folds them into out[0], out[1] with atomicMax on the bit patterns (non-negative
// floating-point values order like their unsigned bit patterns; a NaN has larger
// bits than every finite value and infinity, so it survives the reduction).
template <typename R>
struct Bits;
template <>
struct Bits<float> {
    using T = unsigned int;
    __device__ static T of(float x) { return __float_as_uint(x); }
};
template <>
struct Bits<double> {
    using T = unsigned long long;
    __device__ static T of(double x) { return (unsigned long long)__double_as_longlong(x); }
};

template <typename R>
__device__ __forceinline__ R max_keep_nan(R a, R b)
{
    return (b > a || b != b) ? b : a;
}

template <typename R>
__global__ void residual_kernel(DomainView<R> d, CLayer<R> x, CLayer<R> t, unsigned long long *out)
{
    R dm = R(0), xm = R(0);
    for (long long i = gtid(); i < d.n; i += gstride()) {
        if (!code_is_in(d.code[i])) continue;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const R a = x.f[v][i];
            dm = max_keep_nan(dm, fabs(a - t.f[v][i]));
            xm = max_keep_nan(xm, fabs(a));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dm = max_keep_nan(dm, __shfl_xor_sync(0xffffffffu, dm, o));
        xm = max_keep_nan(xm, __shfl_xor_sync(0xffffffffu, xm, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, (unsigned long long)Bits<R>::of(dm));
        atomicMax(out + 1, (unsigned long long)Bits<R>::of(xm));
    }
}

// Solver3D::GetLayer clears OUT cells of the layer to MISSING_VALUE first
// (Solver3D.cpp:23, TimeLayer3D.h:974-998).
template <typename R>
__global__ void fill_missing_kernel(DomainView<R> d, Layer<R> l)
{
    for (long long i = gtid(); i < d.n; i += gstride()) {
        if ((d.code[i] & CODE_TYPE) == NODE_OUT) {
#pragma unroll
            for (int v = 0; v < 4; v++) l.f[v][i] = R(99999.0f);
        }
    }
}

// FilterToArrays point sampling (TimeLayer3D.h:869-881) of a layer onto an
// ox x oy x oz grid: output cell (i, j, k) takes node (i*nx/ox, j*ny/oy, k*nz/oz);
// velocity in the layer's precision (3 values per cell), T as double.
template <typename R>
__global__ void sample_layer_kernel(CLayer<R> l, int nx, int ny, int nz, int ox, int oy, int oz, R *vout,
                                    double *Tout)
{
    const long long m = (long long)ox * oy * oz;
    for (long long idx = gtid(); idx < m; idx += gstride()) {
        const int i = (int)(idx / ((long long)oy * oz)), j = (int)((idx / oz) % oy), k = (int)(idx % oz);
        const long long x = (long long)i * nx / ox, y = (long long)j * ny / oy, z = (long long)k * nz / oz;
        const long long src = (x * ny + y) * nz + z;
        vout[3 * idx + 0] = l.f[0][src];
        vout[3 * idx + 1] = l.f[1][src];
        vout[3 * idx + 2] = l.f[2][src];
        Tout[idx] = (double)l.f[3][src];
    }
}

template <typename R>
cudaError_t launch_sample_layer(CLayer<R> l, int nx, int ny, int nz, int ox, int oy, int oz, R *vout, double *Tout,
                                cudaStream_t s)
{
    const long long m = (long long)ox * oy * oz;
    sample_layer_kernel<R><<<grid_for(m, 256), 256, 0, s>>>(l, nx, ny, nz, ox, oy, oz, vout, Tout);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_update_boundaries(const DomainView<R> &d, Layer<R> cur, cudaStream_t s)
{
    update_boundaries_kernel<R><<<grid_for(d.n, 256), 256, 0, s>>>(d, cur);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_step_begin(const DomainView<R> &d, Layer<R> cur, Layer<R> next, Layer<R> ta, Layer<R> tb,
                              bool update_boundaries, cudaStream_t s, bool bv_only)
{
    bool vec = d.n % 4 == 0 && (reinterpret_cast<uintptr_t>(d.code) & 3) == 0;
    for (int v = 0; v < 4; v++)
        for (const void *p : {(const void *)cur.f[v], (const void *)next.f[v], (const void *)ta.f[v],
                              (const void *)tb.f[v], (const void *)d.nv[v]})
            vec &= (reinterpret_cast<uintptr_t>(p) & 15) == 0;
    if (vec)
        step_begin_vec4_kernel<R><<<grid_for(d.n / 4, 256), 256, 0, s>>>(d, cur, next, ta, tb, update_boundaries,
                                                                         bv_only);
    else
        step_begin_kernel<R><<<grid_for(d.n, 256), 256, 0, s>>>(d, cur, next, ta, tb, update_boundaries, bv_only);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_merge(const DomainView<R> &d, CLayer<R> src, Layer<R> dest, cudaStream_t s)
{
    merge_kernel<R><<<grid_for(d.n, 256), 256, 0, s>>>(d, src, dest);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_div_error(const DomainView<R> &d, CLayer<R> l, R dx, R dy, R dz, double *partial_sum,
                             unsigned long long *partial_cnt, int nblocks, double *out_sum,
                             unsigned long long *out_cnt, cudaStream_t s)
{
    div_error_partial_kernel<R><<<nblocks, 256, 0, s>>>(d, l, dx, dy, dz, partial_sum, partial_cnt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    div_error_final_kernel<<<1, 32, 0, s>>>(partial_sum, partial_cnt, nblocks, out_sum, out_cnt);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_fill_missing(const DomainView<R> &d, Layer<R> l, cudaStream_t s)
{
    fill_missing_kernel<R><<<grid_for(d.n, 256), 256, 0, s>>>(d, l);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_step_begin_batch(const BatchDomain<R> *doms, int ndom, long long max_cells, int cur, int nxt,
                                   int ta, int tb, bool update_boundaries, cudaStream_t s)
{
    if (ndom == 0) return cudaSuccess;
    long long per = (max_cells + 255) / 256;
    long long cap = (148LL * 16 + ndom - 1) / ndom;   // about 16 blocks per SM overall
    if (cap < 8) cap = 8;
    const int bx = (int)(per < cap ? (per < 1 ? 1 : per) : cap);
    step_begin_batch_kernel<R><<<dim3(bx, ndom), 256, 0, s>>>(doms, cur, nxt, ta, tb, update_boundaries);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_div_error_batch(const BatchDomain<R> *doms, int ndom, int layer, int nblocks, double *psum,
                                   unsigned long long *pcnt, double *out_sum, unsigned long long *out_cnt,
                                   cudaStream_t s)
{
    if (ndom == 0) return cudaSuccess;
    div_error_batch_partial_kernel<R><<<dim3(nblocks, ndom), 256, 0, s>>>(doms, layer, psum, pcnt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    div_error_final_kernel<<<ndom, 32, 0, s>>>(psum, pcnt, nblocks, out_sum, out_cnt);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_residual(const DomainView<R> &d, CLayer<R> x, CLayer<R> t, unsigned long long *out, cudaStream_t s)
{
    residual_kernel<R><<<DIV_BLOCKS, 256, 0, s>>>(d, x, t, out);
    return cudaGetLastError();
}

// Up to 8 same-sized arrays copied in one launch (16-byte accesses; the arrays
// start on 16-byte boundaries, as every layer and workspace piece does).
struct CopySet {
    const void *src[8];
    void *dst[8];
};

__global__ void __launch_bounds__(256) copy_fields_kernel(CopySet cs, int nf, long long n16, long long tail)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += stride) {
        uint4 v[8];
#pragma unroll
        for (int f = 0; f < 8; f++)
            if (f < nf) v[f] = reinterpret_cast<const uint4 *>(cs.src[f])[i];
#pragma unroll
        for (int f = 0; f < 8; f++)
            if (f < nf) reinterpret_cast<uint4 *>(cs.dst[f])[i] = v[f];
    }
    if (blockIdx.x == 0 && threadIdx.x < tail)
        for (int f = 0; f < nf; f++)
            reinterpret_cast<unsigned char *>(cs.dst[f])[n16 * 16 + threadIdx.x] =
                reinterpret_cast<const unsigned char *>(cs.src[f])[n16 * 16 + threadIdx.x];
}

cudaError_t launch_copy_fields(int nf, const void *const *src, void *const *dst, size_t bytes, cudaStream_t s)
{
    if (nf < 1 || nf > 8) return cudaErrorInvalidValue;
    CopySet cs{};
    for (int f = 0; f < nf; f++) {
        if (((uintptr_t)src[f] | (uintptr_t)dst[f]) % 16) return cudaErrorInvalidValue;
        cs.src[f] = src[f];
        cs.dst[f] = dst[f];
    }
    const long long n16 = (long long)(bytes / 16), tail = (long long)(bytes % 16);
    long long blocks = (n16 + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    copy_fields_kernel<<<(unsigned)blocks, 256, 0, s>>>(cs, nf, n16, tail);
    return cudaGetLastError();
}

#define INST(R)                                                                                                  \
    template cudaError_t launch_step_begin_batch<R>(const BatchDomain<R> *, int, long long, int, int, int, int,  \
                                                    bool, cudaStream_t);                                          \
    template cudaError_t launch_div_error_batch<R>(const BatchDomain<R> *, int, int, int, double *,               \
                                                   unsigned long long *, double *, unsigned long long *,          \
                                                   cudaStream_t);                                                 \
    template cudaError_t launch_residual<R>(const DomainView<R> &, CLayer<R>, CLayer<R>, unsigned long long *,   \
                                            cudaStream_t);                                                        \
    template cudaError_t launch_update_boundaries<R>(const DomainView<R> &, Layer<R>, cudaStream_t);            \
    template cudaError_t launch_step_begin<R>(const DomainView<R> &, Layer<R>, Layer<R>, Layer<R>, Layer<R>,    \
                                              bool, cudaStream_t, bool);                                          \
    template cudaError_t launch_merge<R>(const DomainView<R> &, CLayer<R>, Layer<R>, cudaStream_t);             \
    template cudaError_t launch_div_error<R>(const DomainView<R> &, CLayer<R>, R, R, R, double *,                \
                                             unsigned long long *, int, double *, unsigned long long *,          \
                                             cudaStream_t);                                                        \
    template cudaError_t launch_fill_missing<R>(const DomainView<R> &, Layer<R>, cudaStream_t);               \
    template cudaError_t launch_sample_layer<R>(CLayer<R>, int, int, int, int, int, int, R *, double *,        \
                                                cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace adi
