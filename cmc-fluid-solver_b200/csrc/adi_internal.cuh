// Internal declarations shared by the CUDA translation units of libadi_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>

namespace adi {

// Largest dynamic shared-memory size one kernel has been opened to, per device.
// cudaFuncSetAttribute acts on the current device only, so a process that drives
// several GPUs must open the kernel on each of them.  The mutex keeps the
// attribute monotone when two host threads launch the same kernel at once.
struct SmemOptIn {
    std::mutex mu;
    int bytes[64] = {};
};

template <typename F>
inline cudaError_t ensure_dynamic_smem(SmemOptIn &rec, F *kern, size_t bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    std::lock_guard<std::mutex> lock(rec.mu);
    if ((int)bytes <= rec.bytes[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) rec.bytes[dev] = (int)bytes;
    return e;
}

// Node types and BC codes of the reference (Common/Geometry.h:31-41).
enum : uint8_t { NODE_IN = 0, NODE_OUT = 1, NODE_BOUND = 2, NODE_VALVE = 3 };
enum : uint8_t { BC_NOSLIP = 0, BC_FREE = 1 };

// One byte per node on the device: bits 0-1 node type, bit 2 bc_vel == FREE,
// bit 3 bc_temp == FREE.  Replaces the 28-byte (FP32) Node AoS (Grid3D.h:73-88)
// on the sweep's read path; the node values live in four separate arrays.
constexpr uint8_t CODE_TYPE = 0x3;
constexpr uint8_t CODE_VEL_FREE = 0x4;
constexpr uint8_t CODE_TEMP_FREE = 0x8;

__host__ __device__ inline bool code_is_in(uint8_t c) { return (c & CODE_TYPE) == NODE_IN; }
__host__ __device__ inline bool code_is_bv(uint8_t c)
{
    uint8_t t = c & CODE_TYPE;
    return t == NODE_BOUND || t == NODE_VALVE;
}

// Four fields U, V, W, T of one time layer; element (i,j,k) at (i*ny + j)*nz + k.
template <typename R>
struct Layer {
    R *f[4];
};
template <typename R>
struct CLayer {
    const R *f[4];
};

// Geometry of the lines of one sweep direction.  Lines are numbered in the
// order Grid3D::GenerateListSegments visits them (Grid3D.cpp:64-65):
//   X: line = j*nz + k, Y: line = i*nz + k, Z: line = i*ny + j.
struct LineGeom {
    int nx, ny, nz;
    int len;          // nodes per line
    int nlines;
    long long stride; // element stride along the line
};

__host__ __device__ inline LineGeom line_geom(int dir, int nx, int ny, int nz)
{
    LineGeom g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    if (dir == 0) { g.len = nx; g.nlines = ny * nz; g.stride = (long long)ny * nz; }
    else if (dir == 1) { g.len = ny; g.nlines = nx * nz; g.stride = nz; }
    else { g.len = nz; g.nlines = nx * ny; g.stride = 1; }
    return g;
}

__host__ __device__ inline long long line_base(int dir, const LineGeom &g, int line)
{
    if (dir == 0) return line;                                            // (0, j, k): j*nz + k
    if (dir == 1) return (long long)(line / g.nz) * g.ny * g.nz + (line % g.nz); // (i, 0, k)
    return (long long)line * g.nz;                                        // (i, j, 0)
}

// Per-sweep scalar constants, evaluated in the working precision with the same
// operations BuildMatrix uses (AdiSolver3D.cpp:744-752,760-797).
template <typename R>
struct SweepConst {
    R three;         // 3
    R dt;            // dt
    R two_h;         // 2 * h along the line
    R vis_v, vis_t;  // v_vis / (h*h), t_vis / (h*h)
    R b_v, b_t;      // 3/dt + 2*vis
    R v_T, t_phi;
    R two_dx, two_dy, two_dz;
    // reciprocal forms used by the fast sweep (multiply instead of divide)
    R three_dt;                          // 3/dt
    R inv_two_h;                         // 1/(2h) along the line
    R inv_two_dx, inv_two_dy, inv_two_dz;
    // 1 when cur equals the node values at every BOUND/VALVE node at the start of
    // the step (adi_update_boundaries ran since the state last changed).  The
    // nonlinear layers are copies of cur that sweeps never write off NODE_IN, so
    // Dirichlet boundary rows can then read their value from the temp tile they
    // already hold instead of loading the node-value arrays.
    int nv_in_temp;
    // Bounded wait of the TMA-fed X/Y sweep for its tiles: polls of about 10 us
    // each (2^17 normally).  skip_tile_loads (set only by adi_set_fault_injection,
    // to test failure detection) makes that sweep issue no tile load at all, so its
    // wait runs out and the step reports ADI_ERR_TIMEOUT with nothing in flight.
    int tile_wait_tries;
    int skip_tile_loads;
};

// Launch shape of the fast sweep: NL lines per CTA, chunks of K rows per thread,
// P chunks per line (P*K >= line length).
struct FastShape {
    int K, NL, P;
    int mode;   // 0: generic chunked kernel; 1: warp-resident Z lines (sweep_zwarp.cu);
                // 2: TMA-fed X/Y tiles of NL = 16 lines (sweep_xytma.cu); 3: persistent
                // double-buffered X/Y tiles, two lines per thread (sweep_xypair.cu, FP32);
                // 4: TMA-fed X/Y tiles of NL = 8 lines (sweep_xytma.cu)
};

// Device-side description of one domain, passed by value to kernels.
template <typename R>
struct DomainView {
    int nx, ny, nz;
    long long n;
    const uint8_t *code;
    const R *nv[4];   // node values v.x v.y v.z T
};

// One domain of a batch (adi_batch_*), as the batched kernels see it: geometry,
// node codes and values, the five layers, per-direction line ranges, sweep
// constants for the batch's dt and lines-per-CTA / chunks-per-line of the batched
// generic sweep (NL * P <= 256).
template <typename R>
struct BatchDomain {
    DomainView<R> d;
    R *L[5][4];
    const int *lo[3];
    const int *hi[3];
    SweepConst<R> kc[3];
    int NL[3], P[3];
    int vec_ok;
    double dx, dy, dz;
};

// ---- launchers (each returns cudaGetLastError()) ----
// bv_only: a step whose first sweep reads cur as its nonlinear layer; only groups
// of four cells with a BOUND / VALVE cell are written (layer_ops.cu says why that
// keeps every value a sweep reads).
template <typename R>
cudaError_t launch_step_begin(const DomainView<R> &d, Layer<R> cur, Layer<R> next, Layer<R> ta, Layer<R> tb,
                              bool update_boundaries, cudaStream_t s, bool bv_only = false);
template <typename R>
cudaError_t launch_update_boundaries(const DomainView<R> &d, Layer<R> cur, cudaStream_t s);
template <typename R>
cudaError_t launch_merge(const DomainView<R> &d, CLayer<R> src, Layer<R> dest, cudaStream_t s);
template <typename R>
cudaError_t launch_div_error(const DomainView<R> &d, CLayer<R> l, R dx, R dy, R dz, double *partial_sum,
                             unsigned long long *partial_cnt, int nblocks, double *out_sum,
                             unsigned long long *out_cnt, cudaStream_t s);
template <typename R>
cudaError_t launch_fill_missing(const DomainView<R> &d, Layer<R> l, cudaStream_t s);
// FilterToArrays point sampling onto ox x oy x oz (vout: 3 values per cell, Tout: doubles).
template <typename R>
cudaError_t launch_sample_layer(CLayer<R> l, int nx, int ny, int nz, int ox, int oy, int oz, R *vout, double *Tout,
                                cudaStream_t s);
// Batch versions: every domain of the batch in one launch (grid y = domain).
// The divergence partials take nblocks * ndom slots, the results ndom each.
template <typename R>
cudaError_t launch_step_begin_batch(const BatchDomain<R> *doms, int ndom, long long max_cells, int cur, int nxt,
                                   int ta, int tb, bool update_boundaries, cudaStream_t s);
template <typename R>
cudaError_t launch_div_error_batch(const BatchDomain<R> *doms, int ndom, int layer, int nblocks, double *psum,
                                   unsigned long long *pcnt, double *out_sum, unsigned long long *out_cnt,
                                   cudaStream_t s);
// out[0] |= max |x - t|, out[1] |= max |x| over NODE_IN cells (bit patterns, atomicMax;
// out must start at zero).
template <typename R>
cudaError_t launch_residual(const DomainView<R> &d, CLayer<R> x, CLayer<R> t, unsigned long long *out, cudaStream_t s);

template <typename R>
cudaError_t launch_sweep_exact(int dir, const DomainView<R> &d, const int *line_lo, const int *line_hi,
                               CLayer<R> cur, CLayer<R> temp_in, Layer<R> next, Layer<R> temp_out,
                               R *scratch, const SweepConst<R> &k, int merges, cudaStream_t s);

template <typename R>
cudaError_t launch_sweep_fast(int dir, const DomainView<R> &d, const int *line_lo, const int *line_hi,
                              CLayer<R> cur, CLayer<R> temp_in, Layer<R> next, Layer<R> temp_out,
                              const SweepConst<R> &k, int merges, FastShape shape, cudaStream_t s);
// Shapes the fast sweep is compiled for (K values); returns false if `shape` is not one.
bool fast_shape_supported(int dir, FastShape shape, int len, int elem_bytes);
// Batched generic sweep: one persistent launch over the (domain, first line) items
// of direction dir; K in {4, 8}; 256 threads per CTA.
template <typename R>
cudaError_t launch_sweep_fast_batch(int dir, int K, const BatchDomain<R> *doms, const int2 *items, int nitems,
                                    int grid, int src, int tin, int dst, int tout, int merges, cudaStream_t s);

template <typename R>
cudaError_t launch_sweep_zwarp(const DomainView<R> &d, const int *line_lo, const int *line_hi, CLayer<R> cur,
                               CLayer<R> tin, Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges,
                               int K, cudaStream_t s);
bool zwarp_supported(int nz, int K, int elem_bytes);
template <typename R>
cudaError_t launch_sweep_xytma(int dir, const DomainView<R> &d, const int *line_lo, CLayer<R> cur, CLayer<R> tin,
                               Layer<R> next, Layer<R> tout, const SweepConst<R> &k, int merges, int K, int nlt,
                               int *err_flag, cudaStream_t s);
bool xytma_supported(int dir, int nx, int ny, int nz, int K, int nlt, int elem_bytes);
// The same X/Y sweep with tiles copied element-wise by the CTA's threads (cp.async):
// any nz, lines up to 160 rows (K = 4: up to 128, K = 5: up to 160), 8 lines per CTA.
template <typename R>
cudaError_t launch_sweep_xycp(int dir, const DomainView<R> &d, CLayer<R> cur, CLayer<R> tin, Layer<R> next,
                              Layer<R> tout, const SweepConst<R> &k, int merges, int K, int *err_flag, cudaStream_t s);
bool xycp_supported(int dir, int nx, int ny, int nz, int K, int elem_bytes);
// ... and for every domain of a batch in one persistent launch (work items
// (domain, tile of 8 lines); each domain's line length at most 32 K rows).
template <typename R>
cudaError_t launch_sweep_xy_batch(int dir, int K, const BatchDomain<R> *doms, const int2 *items, int nitems, int src,
                                  int tin, int dst, int tout, int merges, int *err_flag, cudaStream_t s);
cudaError_t launch_sweep_xypair(int dir, const DomainView<float> &d, const int *line_lo, CLayer<float> cur,
                                CLayer<float> tin, Layer<float> next, Layer<float> tout, const SweepConst<float> &k,
                                int merges, int K, int *err_flag, cudaStream_t s);
bool xypair_supported(int dir, int nx, int ny, int nz, int K, int elem_bytes);

cudaError_t launch_segment_scan(int dir, int nx, int ny, int nz, const uint8_t *code, int *line_count,
                                int *line_lo, int *line_hi, int *line_maxlen, long long *line_nodes,
                                cudaStream_t s);
cudaError_t launch_segment_write(int dir, int nx, int ny, int nz, const uint8_t *code,
                                 const long long *line_offset, int32_t *out7, cudaStream_t s);

// ---- adjoint (adjoint.cu) ----
// Adjoint of one sweep of direction dir with its tape (ti: the nonlinear layer
// the sweep read, xs: the layer it wrote): dbar consumed on the segment nodes,
// tbar turned from the adjoint of the written temp into that of the read temp,
// sbar and nvbar accumulated; ga, gb are two full-size work planes.
// chunk_K > 0 selects the fused chunked kernel (adjoint_fast.cu) when the line
// length allows it, chunk_K < 0 the split chunked kernels (a solve with chunks of
// -chunk_K rows that stores lambda into lam, then one thread per cell for the
// accumulations), 0 the one-thread-per-line kernel.
template <typename R>
cudaError_t launch_adjoint_sweep(int dir, const DomainView<R> &d, const int *lo, const int *hi, CLayer<R> ti,
                                 CLayer<R> xs, Layer<R> sbar, Layer<R> dbar, Layer<R> tbar, Layer<R> nvbar, R *ga, R *gb,
                                 R *scratch, const SweepConst<R> &k, int merges, int chunk_K, Layer<R> lam,
                                 cudaStream_t s);
// The same adjoint sweep with the chunked parallel structure of the fast forward
// sweep (adjoint_fast.cu); K in {4, 8}; lines up to 256 * K.  Fused (split
// false): the caller zeroes ga, gb and folds them in afterwards
// (launch_adjoint_sweep does both).  Split: the solve stores lambda into lamo and
// the accumulation kernel does the rest, off-line terms included (ga, gb unused).
bool adjoint_chunk_supported(int len, int K, int elem_bytes, int &NL, int &P);
template <typename R>
cudaError_t launch_adjoint_chunk(int dir, int K, const DomainView<R> &d, const int *lo, const int *hi, CLayer<R> ti,
                                 CLayer<R> xs, Layer<R> sbar, Layer<R> dbar, Layer<R> tbar, Layer<R> nvbar, R *ga, R *gb,
                                 const SweepConst<R> &k, int merges, bool split, Layer<R> lamo, cudaStream_t s);
// Adjoint of the step start and UpdateBoundaries (cbar: in, adjoint of cur after
// them; out, before them).
template <typename R>
cudaError_t launch_adjoint_step_start(const DomainView<R> &d, Layer<R> cbar, Layer<R> nbar, Layer<R> tbar,
                                      Layer<R> nvbar, cudaStream_t s);
// Kinetic energy of the NODE_IN cells of the box [lo, hi) of x into *out, and its
// gradient into cbar (psum: nblocks doubles of scratch).
template <typename R>
cudaError_t launch_objective(const DomainView<R> &d, CLayer<R> x, const int lo[3], const int hi[3], Layer<R> cbar,
                             double *psum, int nblocks, double *out, cudaStream_t s);

// nf (<= 8) arrays of `bytes` each, src[f] -> dst[f], in one launch; every pointer
// 16-byte aligned (cudaErrorInvalidValue otherwise).
cudaError_t launch_copy_fields(int nf, const void *const *src, void *const *dst, size_t bytes, cudaStream_t s);

// ---- mask builders (masks.cu) ----
// Shape3D: types (n bytes of scratch) <- NODE_IN, triangles rasterised as
// NODE_BOUND, outside flood-filled as NODE_OUT.  verts: 3 floats per vertex in
// grid coordinates; tris: 3 vertex indices per triangle (checked by the caller).
// status[0]: writes outside the grid, status[1]: loops stopped at their bound;
// changed: one int of scratch; the flood fill stops after max_passes.
cudaError_t launch_mask_shape3d(uint8_t *types, int nx, int ny, int nz, const float *verts, int nverts,
                                const int *tris, int ntris, int *status, int *changed, int max_passes,
                                int *passes_out, cudaStream_t s);
// Shape2D: a 2D node grid (nx x ny, i-major) from segments (8 floats each: p1, p2,
// v1, v2 in grid coordinates) in the reference's write order, with their node
// types (color).  key: nx*ny 64-bit scratch; vel: 2 floats per cell.
cudaError_t launch_mask_shape2d(const float *segs, const uint8_t *color, int nseg, int nx, int ny, float startT,
                                unsigned long long *key, uint8_t *type, float *vel, float *T, uint8_t *bc,
                                int *status, int *changed, int max_passes, int *passes_out, cudaStream_t s);
template <typename R>
cudaError_t launch_mask_shape3d_install(const uint8_t *types, uint8_t *code, Layer<R> nv, Layer<R> cur, long long n,
                                        R baseT, cudaStream_t s);
// SeaNetCDF from a depth map (snap: n bytes of scratch).
template <typename R>
cudaError_t launch_mask_sea(uint8_t *code, uint8_t *snap, Layer<R> nv, Layer<R> cur, int nx, int ny, int nz,
                            const float *depth, int dnx, int dny, float zmin, float baseT, const float in_vel[3],
                            float in_T, int *status, cudaStream_t s);
// Shape2D extrusion of a 2D node grid (t2: types, v2: 2 floats, T2: 1 float per cell).
template <typename R>
cudaError_t launch_mask_extrude2d(uint8_t *code, Layer<R> nv, Layer<R> cur, int nx, int ny, int nz,
                                  const uint8_t *t2, const float *v2, const float *T2, int active_nz, double depth_var,
                                  float baseT, int *status, cudaStream_t s);

// Solver contract and NODE_IN count of a node grid on the device: out2[0] = min
// over cells breaking the contract of (index << 2 | rule), rule 1: NODE_IN on the
// frame, 2: NODE_IN next to NODE_OUT, 3: BC_FREE cell between two fluid runs
// (~0 if none); out2[1] = NODE_IN cells.  The caller synchronises before reading.
cudaError_t launch_mask_census(const uint8_t *code, int nx, int ny, int nz, unsigned long long *out2,
                               cudaStream_t s);

constexpr int DIV_BLOCKS = 592;  // 4 x 148 SMs

} // namespace adi
