/*
 * adi_b200.h — C ABI of the B200-native 3D ADI time step.
 *
 * This is the drop-in boundary for the reference solver's hot path
 * (samech-git/cmc-fluid-solver, src/FluidSolver3D).  A C++ host that keeps the
 * reference's Solver3D surface (Solver3D.h:24-49) calls these functions instead of
 * the reference's host<->CUDA launchers.  Plain C types only: opaque handle,
 * host pointers, sizes, status codes.  No exceptions cross this boundary and
 * nothing here calls exit().
 *
 * Conventions
 *   - Arrays are [i][j][k] with k fastest, i.e. index = (i*dimy + j)*dimz + k,
 *     the layout of ScalarField3D::elem and Grid3D::GetType
 *     (TimeLayer3D.h:256-259, Grid3D.cpp:242-245).
 *   - Node types / BC codes are the reference enums (Common/Geometry.h:31-41):
 *     NODE_IN=0 NODE_OUT=1 NODE_BOUND=2 NODE_VALVE=3; BC_NOSLIP=0 BC_FREE=1.
 *   - "field buffers" for get/set are in the handle's precision (float for
 *     ADI_FP32, double for ADI_FP64), four separate arrays u, v, w, T.
 *   - Every call is asynchronous on the handle's stream except those that return
 *     data to the host (get_*, div_error, build_segments statistics), which
 *     synchronise that stream.
 *   - A handle is not thread-safe; distinct handles are independent.
 */
#ifndef ADI_B200_H
#define ADI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum adi_status {
    ADI_OK = 0,
    ADI_ERR_BAD_ARG = 1,       /* invalid argument or a mask the solver contract rejects */
    ADI_ERR_CAPACITY = 2,      /* a size beyond a stated maximum */
    ADI_ERR_NONFINITE = 3,     /* NaN/Inf found in a field after a step */
    ADI_ERR_NOT_CONVERGED = 4, /* tolerance mode: max global iterations reached */
    ADI_ERR_CUDA = 5,          /* a CUDA runtime call failed; see adi_last_error_string */
    ADI_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up */
    ADI_ERR_DIVERGENCE = 7,    /* divergence error above 0.01 (the reference throws,
                                  AdiSolver3D.cpp:371-374); layers are left unswapped */
    ADI_ERR_STATE = 8,         /* call order: e.g. a step before adi_set_mask */
    ADI_ERR_NO_DEVICE = 9      /* no CUDA device, or not an sm_100 device */
} adi_status;

typedef enum adi_precision { ADI_FP32 = 4, ADI_FP64 = 8 } adi_precision;

/* Sweep implementation.
 * ADI_SOLVER_EXACT: Thomas elimination per segment in the reference's operation
 *   order (Common/Algorithms.h:21-39) without fused multiply-add; results equal the
 *   reference CPU solver's bit for bit.
 * ADI_SOLVER_FAST: chunked elimination with register-resident coefficients; same
 *   equations, different rounding (within the documented tolerance). */
typedef enum adi_solver_kind { ADI_SOLVER_EXACT = 0, ADI_SOLVER_FAST = 1 } adi_solver_kind;

typedef enum adi_dir { ADI_X = 0, ADI_Y = 1, ADI_Z = 2 } adi_dir;

typedef struct adi_handle adi_handle;

/* Grid3D geometry: dims and spacing (Grid3D.h:97-98), plus the run precision
 * (replaces the compile-time FTYPE, Common/Geometry.h:21). */
typedef struct adi_grid_desc {
    int dimx, dimy, dimz;
    double dx, dy, dz;
    int precision; /* adi_precision */
} adi_grid_desc;

/* FluidParams (Common/Geometry.h:538-562). */
typedef struct adi_fluid_params {
    double v_T, v_vis, t_vis, t_phi;
} adi_fluid_params;

/* Per-direction segment statistics from adi_build_segments. */
typedef struct adi_seg_stats {
    int64_t num_segments[3];   /* per direction X, Y, Z */
    int64_t num_nodes[3];      /* sum of segment sizes (endpoints included) */
    int32_t max_size[3];       /* longest segment */
    int32_t max_per_line[3];   /* most segments on one line */
    int64_t num_in;            /* NODE_IN cells */
} adi_seg_stats;

/* ---- parameters -------------------------------------------------------- */

/* FluidParams(Re, Pr, lambda): v_T=1, v_vis=1/Re, t_vis=1/(Re*Pr),
 * t_phi=(lambda-1)/(lambda*Re).  Replaces Geometry.h:545-552. */
adi_status adi_fluid_params_normalized(double Re, double Pr, double lambda, adi_fluid_params *out);

/* FluidParams(vis, rho, R, k, cv).  Replaces Geometry.h:554-561. */
adi_status adi_fluid_params_dimensional(double vis, double rho, double R, double k, double cv,
                                        adi_fluid_params *out);

/* ---- lifetime ---------------------------------------------------------- */

/* Allocates every device buffer of one domain on the current CUDA device.
 * Replaces AdiSolver3D::Init (AdiSolver3D.cpp:166-268) for the single-GPU case. */
adi_status adi_create(const adi_grid_desc *grid, const adi_fluid_params *params, adi_handle **out);

/* Frees all device memory of the handle.  Replaces AdiSolver3D::~AdiSolver3D /
 * FreeMemory (AdiSolver3D.cpp:103-158). */
adi_status adi_destroy(adi_handle *h);

/* Binds the handle to a cudaStream_t (NULL = legacy default stream). */
adi_status adi_set_stream(adi_handle *h, void *cuda_stream);

/* Selects the sweep implementation (adi_solver_kind).  Default ADI_SOLVER_FAST. */
adi_status adi_set_solver(adi_handle *h, int kind);

/* Message for the last non-OK status of this handle (static storage). */
const char *adi_last_error_string(const adi_handle *h);

/* Fault injection, for testing failure detection (no counterpart in the
 * reference).  ADI_FAULT_SKIP_TILE_LOADS: the TMA-fed X/Y sweeps (fast solver,
 * 8- or 16-line tile shapes) issue no tile loads, so their bounded wait for the
 * tiles gives up after about 160 us; the step's next synchronising call returns
 * ADI_ERR_TIMEOUT and the sweep writes nothing.  Nothing is left in flight and
 * the context stays usable: ADI_FAULT_NONE restores normal steps.  Rebuilds the
 * handle's step graphs. */
typedef enum adi_fault { ADI_FAULT_NONE = 0, ADI_FAULT_SKIP_TILE_LOADS = 1 } adi_fault;
adi_status adi_set_fault_injection(adi_handle *h, int what);

/* ---- grid / mask ------------------------------------------------------- */

/* Uploads the Grid3D node array as SoA: node type, bc_vel, bc_temp and the
 * node values v.x, v.y, v.z, T (Grid3D.h:73-88).  The values are the boundary
 * data and also the initial state of every field (TimeLayer3D(grid) ->
 * CopyFromGrid, TimeLayer3D.h:1077-1090).  Values are rounded to the handle's
 * precision.  Also checks the solver contract: no IN cell on the outer frame, no
 * IN cell next to an OUT cell, no BC_FREE cell between two fluid runs; a mask
 * that breaks it is stored but adi_time_step returns ADI_ERR_BAD_ARG for it. */
adi_status adi_set_mask(adi_handle *h, const uint8_t *node_type, const uint8_t *bc_vel,
                        const uint8_t *bc_temp, const double *vx, const double *vy,
                        const double *vz, const double *T);

/* ---- mask builders on the GPU ------------------------------------------- *
 * Each builds the node grid on the device and then behaves as adi_set_mask with
 * that grid (initial state = node values, contract check, segments to be rebuilt).
 * The arithmetic is the reference's FTYPE = float arithmetic, so the node grid is
 * bit-identical to the reference's for the same input.  Inputs the reference
 * cannot finish (a scanline walk that stops advancing on a near-degenerate
 * triangle, a write outside the node array) return ADI_ERR_BAD_ARG. */

/* Grid3D::Build (Grid3D.cpp:854-898; Prepare3D_Shape :947-964 and
 * ComputeSubframeInfo :900-945, the choice of frame and its vertices, are the
 * caller's): all cells NODE_IN; the triangles rasterised as NODE_BOUND
 * (RasterPolygon :710-788 and RasterLine on the three edges :790-809); NODE_IN
 * cells connected to cell (0,0,0) become NODE_OUT (FloodFill :811-852);
 * NODE_IN/NODE_OUT cells get no-slip, v = 0, T = (float)base_T; NODE_BOUND cells
 * keep their BCs and values (zero, no-slip on a handle that had no mask, as
 * Grid3D::Init leaves them).
 * verts: 3 floats per vertex in grid coordinates ((x - bbox.min) / dx, ...,
 * Grid3D.cpp:420-428); tris: 3 vertex indices per triangle of the inactive shapes.
 * *fill_passes (may be NULL): flood-fill passes run. */
adi_status adi_mask_shape3d(adi_handle *h, const float *verts, int nverts, const int *tris,
                            int ntris, double base_T, int *fill_passes);

/* Grid3D::Prepare3D_NetCDF (Grid3D.cpp:966-1075) from the depth map the NetCDF
 * file holds (depth[dj + di * depth_ny], negative under water) and bbox.pMin.z
 * (zmin): water columns NODE_IN, water next to NODE_OUT and NODE_OUT next to the
 * resulting walls turned into no-slip walls, NODE_IN cells of the faces y = ny-1
 * and then x = nx-1 into valves with (in_vel, in_T) below the middle of their
 * water column and (-in_vel, 2 - in_T) above it. */
adi_status adi_mask_sea(adi_handle *h, const float *depth, int depth_nx, int depth_ny, float zmin,
                        double base_T, const float in_vel[3], double in_T);

/* Grid3D::Prepare2D (Grid3D.cpp:608-665): the 2D node grid of FluidSolver2D::Grid2D
 * (types, velocities (2 floats) and T per (i, j), i-major, of the handle's nx x ny)
 * extruded over active_nz of the nz levels, with a no-slip/free lid at
 * active_nz - 2 and a curved bottom of relative height depth_var. */
adi_status adi_mask_extrude2d(adi_handle *h, const uint8_t *type2d, const float *vel2d,
                              const float *T2d, int active_nz, double depth_var, double base_T);

/* FluidSolver2D::Grid2D::Build (Grid2D.cpp:231-266) on the GPU, for the no-slip
 * grids of the 2D solver and of 2D shapes extruded in depth (Grid3D's 2D grid):
 * every cell NODE_IN, the segments rasterised (RasterLine, Grid2D.cpp:109-141:
 * the cell takes the velocity interpolated along the segment, later segments and
 * steps overwriting earlier ones), the outside flood-filled from cell (0,0)
 * (FloodFill, :156-195), NODE_IN/NODE_OUT cells v = 0; T = (float)start_T and a
 * no-slip BC everywhere.  segs: 8 floats per segment (p1, p2, v1, v2, grid
 * coordinates) in the reference's order -- the segments of the moving shapes,
 * then those of the fixed ones (Grid2D.cpp:237-252); seg_type: NODE_VALVE or
 * NODE_BOUND per segment.  The grid (nx x ny, i-major) comes back in host arrays:
 * node type, BC, velocity (2 floats) and T per cell.  Runs on cuda_stream (NULL:
 * the default stream) of the current device.  A segment that leaves the grid
 * (the reference writes outside its node array) returns ADI_ERR_BAD_ARG. */
adi_status adi_mask_shape2d(const float *segs, const uint8_t *seg_type, int nseg, int nx, int ny, double start_T,
                            void *cuda_stream, uint8_t *type2d, uint8_t *bc2d, float *vel2d, float *T2d);

/* Reads the node grid back (types, BCs, node values in double). */
adi_status adi_get_mask(adi_handle *h, uint8_t *type, uint8_t *bc_vel, uint8_t *bc_temp,
                        double *vx, double *vy, double *vz, double *T);

/* Builds the per-direction segment lists on the GPU from the mask, once.
 * Replaces AdiSolver3D::CreateSegments / Grid3D::GenerateListSegments /
 * GenerateGridBoundaries (AdiSolver3D.cpp:553-562, Grid3D.cpp:47-146).
 * stats may be NULL. */
adi_status adi_build_segments(adi_handle *h, adi_seg_stats *stats);

/* Copies one direction's segment list to the host, in Grid3D::GenerateListSegments
 * order, 7 int32 per segment: posx posy posz endx endy endz size.  If out7 is NULL
 * only *count is written.  ADI_ERR_CAPACITY if cap < count. */
adi_status adi_get_segments(adi_handle *h, int dir, int32_t *out7, int64_t cap, int64_t *count);

/* ---- time stepping ----------------------------------------------------- */

/* cur[BOUND|VALVE] = node values.  Replaces AdiSolver3D::UpdateBoundaries
 * (AdiSolver3D.cpp:286-304; CPU semantics Solver3D.cpp:27-34). */
adi_status adi_update_boundaries(adi_handle *h);

/* One time step with num_global nonlinear iterations of Z, Y, X sweeps, each
 * repeated num_local times.  Replaces AdiSolver3D::TimeStep (AdiSolver3D.cpp:306-391)
 * with the CPU backend's merge schedule.  compute_error != 0 evaluates the
 * divergence error of the result on the GPU; a value above 0.01 (the last one
 * evaluated, as in the reference) returns ADI_ERR_DIVERGENCE. */
adi_status adi_time_step(adi_handle *h, double dt, int num_global, int num_local, int compute_error);

/* adi_update_boundaries + adi_time_step: one pass of the reference driver loop
 * (FluidSolver3D.cpp:241-242). */
adi_status adi_step(adi_handle *h, double dt, int num_global, int num_local, int compute_error);

/* Runs n_steps driver-loop passes (adi_step); compute_error every err_every steps
 * (0 = never) and on the last, like the driver loop
 * (FluidSolver3D.cpp:224-262) without output. */
adi_status adi_run(adi_handle *h, double dt, int num_global, int num_local, int n_steps, int err_every);

/* adi_step in tolerance mode (no counterpart in the reference's 3D solver, whose
 * TimeStep runs a fixed num_global; its 2D solver loops on a divergence threshold,
 * AdiSolver2D.cpp:290-314).  Global iterations run until the residual
 *   r = max |x - t| / max |x|   over NODE_IN cells and the four fields,
 * x the layer the iteration produced and t the nonlinear layer its last sweep
 * linearised about, is <= tol, or max_global iterations have run.  *iters_used and
 * *residual (either may be NULL) report the count and the last r.  The residual is
 * a warp-shuffle max-reduction on the GPU read back after each iteration. */
adi_status adi_step_tol(adi_handle *h, double dt, int max_global, int num_local, double tol, int compute_error,
                        int *iters_used, double *residual);

/* adi_step, adi_time_step and adi_run replay one CUDA graph per step shape (dt,
 * iteration counts, error flag, layer roles), captured on first use on a private
 * stream and launched on the handle's stream; a step that computes the divergence
 * error waits for it, any other step returns without synchronising.  on = 0 issues
 * every kernel directly instead (as does profiling, adi_set_profiling).  Graphs are
 * rebuilt after adi_set_mask, adi_build_segments, adi_autotune, adi_set_fast_shape
 * and adi_set_solver.  Default on. */
adi_status adi_set_graphs(adi_handle *h, int on);

/* ---- step phases --------------------------------------------------------- */

/* The parts of adi_step one at a time, for hosts that split a domain over
 * several handles and exchange data between sweeps (no counterpart in the
 * reference's single-process step; the reference's multi-GPU slab solver,
 * AdiSolver3D.cu:523-881, exchanges inside its sweeps).  A step is:
 *   adi_phase_begin(h, 1)                 UpdateBoundaries + the step start
 *   per global iteration: adi_phase_sweep for Z, Y, X, each num_local times
 *                         (merges = 2 on the last X sweep of the iteration)
 *   adi_phase_div_sum(h, ADI_ROLE_NEXT)   optional: divergence sum and IN count
 *   adi_phase_end(h)                      the new state becomes cur
 * Sweeps read and write the handle's layers by role; adi_role_pointers gives a
 * role's four field arrays (U, V, W, T) on the device, valid until the roles next
 * change (every sweep swaps the two nonlinear layers; adi_phase_end swaps cur and
 * next).  Asynchronous on the handle's stream, except adi_phase_div_sum. */
enum { ADI_ROLE_CUR = 0, ADI_ROLE_NEXT = 1, ADI_ROLE_HALF = 2, ADI_ROLE_TEMP_IN = 3, ADI_ROLE_TEMP_OUT = 4 };
adi_status adi_phase_begin(adi_handle *h, int update_boundaries);
adi_status adi_phase_sweep(adi_handle *h, int dir, double dt, int merges);
adi_status adi_phase_div_sum(adi_handle *h, int role, double *sum, uint64_t *count);
adi_status adi_phase_end(adi_handle *h);
adi_status adi_role_pointers(adi_handle *h, int role, void **out4);

/* ---- fields ------------------------------------------------------------ */

/* Layers: 0 = cur (latest state), 1 = next (scratch layer of the last step). */
adi_status adi_get_state(adi_handle *h, int layer, void *u, void *v, void *w, void *T);
adi_status adi_set_state(adi_handle *h, const void *u, const void *v, const void *w, const void *T);

/* adi_set_state + adi_step + adi_get_state(h, 0, ...) as one pipelined call: the
 * state is uploaded from in4[0..3] (u, v, w, T host arrays) on an upload stream,
 * the step runs on the handle's stream, the result is copied aside on the device
 * and downloaded into out4[0..3] on a download stream, each field in four pieces.
 * Returns once the work is queued (after the divergence check when
 * compute_error, which waits for the step); call adi_io_wait before reading out4.
 * Each upload piece waits for the same piece of the previous call's download, so
 * a call may take the previous call's out4 as its in4 (a host-side time march):
 * the download of one piece then overlaps the upload of the one before it.  Host
 * arrays should be page-locked (cudaHostAlloc / cudaHostRegister) for the copies
 * to run asynchronously; results equal the three separate calls bit for bit. */
adi_status adi_step_io(adi_handle *h, const void *const *in4, void *const *out4, double dt, int num_global,
                       int num_local, int compute_error);
/* Waits for the last adi_step_io download; work queued on the handle's stream
 * afterwards follows it. */
adi_status adi_io_wait(adi_handle *h);

/* Solver3D::GetLayer (Solver3D.cpp:21-25 + TimeLayer3D::FilterToArrays,
 * TimeLayer3D.h:819-924): OUT cells of the layer the reference reads (`next`,
 * which after a step holds the state the step started from) are set to 99999
 * (MISSING_VALUE), then the layer is point-sampled onto an outdimx x outdimy x
 * outdimz grid (0 = full size) at x = i*dimx/outdimx (integer division), etc.
 * v receives 3 interleaved values per point (Vec3D) in the handle's precision,
 * T one double per point.  Both steps run on the GPU; only the sampled grid is
 * copied to the host. */
adi_status adi_get_layer(adi_handle *h, int outdimx, int outdimy, int outdimz, void *v, double *T);

/* Mean absolute finite-volume divergence of cur over IN cells
 * (TimeLayer3D::EvalDivError, TimeLayer3D.h:595-641), computed on the GPU. */
adi_status adi_div_error(adi_handle *h, double *out);

/* ---- fast-sweep launch shapes (autotuner) -------------------------------- */

/* Launch shape of the fast sweep for one direction: each thread owns K
 * consecutive rows of a line, a CTA holds NL lines, P = ceil(len/K) chunks per
 * line.  NL = 0 selects the warp-resident Z kernel (Z only; K in {4, 5, 8}, or
 * 12 in float for 256 < dimz <= 384; a line in the smallest P in {4, 8, 16, 32}
 * lanes with P K >= dimz, so dimz <= 32 K); NL = -16 and NL = -8 select the TMA-fed X/Y
 * kernel with 16 or 8 lines per CTA (dimz a multiple of 16, K in {4, 8, 16},
 * line length = P K with P in {4, 8, 16} or P = 32 at K = 4, or, in float with
 * K = 4 and 8 lines, P = 64 or 96 (lines of 256 or 384 rows), tiles within the
 * shared memory of the CTAs per SM the shape is compiled for); NL = -1 selects
 * the same X/Y kernel with tiles of 8 lines copied element by element by the
 * CTA's threads (cp.async), for any dimz and lines up to 128 rows (K = 4) or
 * 160 rows (K = 5);
 * NL = -32 selects the persistent, double-buffered X/Y kernel with
 * two lines per thread (FP32 only; dimz a multiple of 16, K in {4, 8}, 2 <= P <= 32,
 * both tile buffers within 227 KB of shared memory, e.g. line length <= 136 at
 * K = 4).  adi_build_segments times the candidate shapes on
 * the domain (the autotuner) and keeps the fastest per direction; these calls
 * read or override the choice.  adi_set_fast_shape returns ADI_ERR_BAD_ARG for a
 * shape no kernel is compiled for (generic: K in {4, 8, 12, 16},
 * 32 <= NL*P <= 256). */
adi_status adi_get_fast_shape(adi_handle *h, int dir, int *K, int *NL, int *P);
adi_status adi_set_fast_shape(adi_handle *h, int dir, int K, int NL);

/* Re-runs the autotuner for all three directions (reps timed launches per
 * candidate); also called by adi_build_segments when the solver is ADI_SOLVER_FAST. */
adi_status adi_autotune(adi_handle *h, int reps);

/* ---- profiling ----------------------------------------------------------- */

/* Kernel classes timed by the built-in profiler; the names follow the reference's
 * Profiler events (AdiSolver3D.cpp:297-301,319-321,592-652). */
typedef enum adi_kernel_class {
    ADI_K_STEP_BEGIN = 0,   /* UpdateBoundaries + CopyLayer (fused) */
    ADI_K_SWEEP_X = 1,      /* SolveSegments_X */
    ADI_K_SWEEP_Y = 2,      /* SolveSegments_Y */
    ADI_K_SWEEP_Z = 3,      /* SolveSegments_Z */
    ADI_K_MERGE = 4,        /* MergeLayer (only when not fused into a sweep) */
    ADI_K_DIV_ERROR = 5,    /* EvalDivError */
    ADI_K_OTHER = 6,
    ADI_K_NUM = 7
} adi_kernel_class;

typedef struct adi_profile {
    int64_t launches[ADI_K_NUM];  /* kernel launches since the last reset */
    double ms[ADI_K_NUM];         /* summed CUDA-event time (profiling on only) */
    int64_t bytes[ADI_K_NUM];     /* algorithmic HBM bytes of those launches */
} adi_profile;

/* on != 0: record a CUDA event pair around every kernel launch on the handle's
 * stream.  Launch counts and algorithmic bytes are always kept. */
adi_status adi_set_profiling(adi_handle *h, int on);

/* Synchronises the stream, folds pending event pairs into the totals and copies
 * them out; reset != 0 zeroes the totals afterwards. */
adi_status adi_get_profile(adi_handle *h, adi_profile *out, int reset);

/* Device pointers of the current layers (zero-copy, for a torch test harness):
 * cur u, v, w, T then next u, v, w, T.  The state may be written through them
 * between steps; the next adi_step (or adi_update_boundaries) re-applies the
 * boundary values. */
adi_status adi_device_pointers(adi_handle *h, void *out8[8]);

/* ---- adjoint --------------------------------------------------------------- */

/* Discrete adjoint of n_steps adi_step calls (no counterpart in the reference).
 * Runs the steps from the current state (no divergence guard), evaluates
 *   J = 1/2 sum over NODE_IN cells of the box [box_lo, box_hi) of u^2 + v^2 + w^2
 * on the final state, and returns dJ/d(node values) (nv_grad: 4 fields, handle
 * precision, [i][j][k]; the inflow, wall and outflow data are node values) and
 * dJ/d(initial state) (state_grad), either may be NULL.  The backward pass runs
 * the sweeps in reverse order, each as a transposed tridiagonal solve over the same
 * segments, recomputing the steps of each window of ckpt_every steps from a
 * stored state.  Device memory: (n_steps/ckpt_every + 12) layers plus the tape of
 * one window, ckpt_every * num_global * num_local * 3 * 8 fields, in one
 * allocation that the handle keeps for later calls (grown when a call needs more,
 * freed by adi_destroy).  The handle ends at the final state. */
adi_status adi_adjoint_run(adi_handle *h, double dt, int num_global, int num_local, int n_steps, int ckpt_every,
                           const int box_lo[3], const int box_hi[3], double *J, void *nv_grad, void *state_grad);

/* Adjoint sweep variant: K = 4 or 8 runs the chunked transposed solve fused with
 * its accumulations (K rows per thread, cyclic reduction across chunks; lines up
 * to 256 * K); K = -4 or -8 the same solve split from the accumulations (the
 * solve stores the adjoint solution, one thread per cell then accumulates it,
 * off-line terms included); K = 0 one thread per line (any length).  Lines too
 * long for a chunked variant take the one-thread-per-line kernel. */
adi_status adi_set_adjoint_chunk(adi_handle *h, int K);

/* Replaces the node values (the boundary data of every node; Grid3D node v, T)
 * without touching the state; the next adi_step applies them. */
adi_status adi_set_node_values(adi_handle *h, const double *vx, const double *vy, const double *vz,
                               const double *T);

/* ---- 2D solver ------------------------------------------------------------ */

/* The reference's 2D ADI solver (FluidSolver2D/AdiSolver2D.cpp) on the GPU, with
 * its own semantics, which differ from the 3D solver's: one segment per grid row /
 * column spanning every interior obstacle, 1/dt in the rows, FREE rows x0 - x1 = 0,
 * temp_local copy-then-merge per local iteration, a global loop that runs
 * num_global iterations and then continues while the divergence error exceeds 0.1,
 * layer copies that skip the last row and column.  Float results equal the
 * reference's bit for bit.  Surface: Solver2D / AdiSolver2D (Solver2D.h:23-44). */
typedef struct adi2d_handle adi2d_handle;

/* Replaces AdiSolver2D::Init's allocation (AdiSolver2D.cpp:20-33). */
adi_status adi2d_create(int nx, int ny, double dx, double dy, int precision, const adi_fluid_params *params,
                        adi2d_handle **out);
adi_status adi2d_destroy(adi2d_handle *h);
adi_status adi2d_set_stream(adi2d_handle *h, void *cuda_stream);

/* Grid2D node data as arrays [i][j] (j fastest): cell type, BC type, velocity,
 * temperature (CondData2D, Grid2D.h:31-45); startT is Grid2D::startT.  The state
 * starts at the node data (AdiSolver2D::Init, AdiSolver2D.cpp:35-47); the segments
 * are built here (CreateSegments, :228-277). */
adi_status adi2d_set_grid(adi2d_handle *h, const uint8_t *node_type, const uint8_t *bc_type, const double *vx,
                          const double *vy, const double *T, double startT);

/* Segmentation of the 2D sweeps.  mode 0 (the default): the reference's, one
 * segment per row / column spanning every interior obstacle
 * (AdiSolver2D::CreateSegments, AdiSolver2D.cpp:228-277).  mode 1: masked
 * segments, the 3D solver's segmentation (Grid3D::GenerateListSegments,
 * Grid3D.cpp:47-127) applied to 2D lines -- each maximal run of IN nodes with the
 * non-IN node on each side as its boundary rows, so solid cells are never solved
 * as fluid; everything else (rows, 1/dt, merges, the error loop) is unchanged.
 * The reference has no mode 1.  Rebuilds the segment lists from the node types
 * of adi2d_set_grid (ADI_ERR_STATE before it); the state is kept. */
adi_status adi2d_set_segments(adi2d_handle *h, int mode);

/* Solver2D::UpdateBoundaries (Solver2D.cpp:40-54). */
adi_status adi2d_update_boundaries(adi2d_handle *h);

/* AdiSolver2D::TimeStep (AdiSolver2D.cpp:279-323); *iters_used (may be NULL) gets
 * the global iterations run.  Where the reference calls exit(1) this returns
 * ADI_ERR_DIVERGENCE (error above 1.0) or ADI_ERR_NOT_CONVERGED (over 100
 * iterations) and leaves the state unspecified. */
adi_status adi2d_time_step(adi2d_handle *h, double dt, int num_global, int num_local, int *iters_used);

/* adi2d_update_boundaries + adi2d_time_step (FluidSolver2D.cpp:131-132). */
adi_status adi2d_step(adi2d_handle *h, double dt, int num_global, int num_local, int *iters_used);

/* adi2d_update_boundaries + the step in tolerance mode (no counterpart in the
 * reference, whose loop runs num_global iterations and then continues while the
 * divergence error exceeds 0.1): global iterations run until the change of the
 * iterate
 *   r = max |x_k - x_(k-1)| / max |x_k|   over NODE_IN nodes and the three fields
 * (x_k the layer after global iteration k, x_0 the state the step starts from) is
 * <= tol, at most max_global of them.  The divergence guard stays (error above
 * 1.0: ADI_ERR_DIVERGENCE).  *iters_used and *residual (either may be NULL) get
 * the count and the last r.  Synchronises after every iteration. */
adi_status adi2d_step_tol(adi2d_handle *h, double dt, int max_global, int num_local, double tol, int *iters_used,
                          double *residual);

/* which 0: cur (the state), 1: next; handle precision, [i][j]. */
adi_status adi2d_get_state(adi2d_handle *h, int which, void *u, void *v, void *T);
/* Solver2D::SetLayer (Solver2D.cpp:30-38): the state. */
adi_status adi2d_set_state(adi2d_handle *h, const void *u, const void *v, const void *T);
/* Solver2D::GetLayer (Solver2D.cpp:19-29): next point-sampled on outdimx x outdimy
 * (0 = full); vel2 gets interleaved (x, y) doubles, T doubles. */
adi_status adi2d_get_layer(adi2d_handle *h, int outdimx, int outdimy, double *vel2, double *T);
/* Divergence error and global iterations of the last step. */
adi_status adi2d_last_error(adi2d_handle *h, double *err, int *iters);
const char *adi2d_last_error_string(const adi2d_handle *h);

/* ---- batches of domains ------------------------------------------------ */

/* Many independent domains stepped together (no counterpart in the reference,
 * which steps one domain per process).  Each member is an ordinary handle (created,
 * masked and segmented as usual; its own fluid parameters and grid); the batch
 * borrows them, so they must outlive it.  A batch step runs, for all members at
 * once: one step-start launch, one persistent launch per sweep (the generic
 * chunked sweep over a work list of (domain, first line) items in longest-first
 * order, K rows per thread and 256 threads per CTA, lines per CTA fitted to each
 * domain), and the per-domain divergence errors; the whole step is replayed as a
 * CUDA graph.  Members step in lock step: all start with the same layer roles
 * (e.g. freshly set up) and must not be stepped on their own while batched. */
typedef struct adi_batch adi_batch;

/* Builds the batch's descriptors and work lists.  All handles: same precision and
 * device, mask and segments set, solver contract satisfied.  The batch uses the
 * first handle's stream. */
adi_status adi_batch_create(adi_handle *const *handles, int n, adi_batch **out);
adi_status adi_batch_destroy(adi_batch *b);
adi_status adi_batch_set_stream(adi_batch *b, void *cuda_stream);

/* adi_step for every member: boundary update, num_global x (Z, Y, X sweeps,
 * num_local each), divergence errors when compute_error.  If any member's
 * (last computed) divergence error exceeds 0.01 the call returns
 * ADI_ERR_DIVERGENCE and no member advances. */
adi_status adi_batch_step(adi_batch *b, double dt, int num_global, int num_local, int compute_error);

/* adi_batch_step with host buffers: member q's state is uploaded from in[4 q + f]
 * (f = u, v, w, T; the member's precision) and its new state downloaded into
 * out[4 q + f].  With the member-graph schedule each branch runs, member after
 * member, the upload, the member's step and the download, so copies overlap other
 * members' sweeps; with the persistent schedule all uploads precede the step and
 * all downloads follow it.  Returns once queued (after the divergence check when
 * compute_error); call adi_batch_io_wait before reading out.  A call may take the
 * previous call's out as its in.  On ADI_ERR_DIVERGENCE no member advances (out
 * then holds the rejected step's results). */
adi_status adi_batch_step_io(adi_batch *b, const void *const *in, void *const *out, double dt, int num_global,
                             int num_local, int compute_error);
adi_status adi_batch_io_wait(adi_batch *b);

/* Last computed divergence error of each member (n values). */
adi_status adi_batch_div_errors(adi_batch *b, double *out);

/* Kernel and chunk length of the batched sweep per direction (segment-to-thread
 * binning): K in {4, 8} runs the generic chunked kernel over (domain, lines)
 * items; for X and Y, K = -4 or -5 runs the tile kernel over (domain, tile of 8
 * lines) items, tiles copied element-wise, chunks of |K| rows, every member's
 * line length at most 32 |K| (else ADI_ERR_CAPACITY).  The autotuner times every
 * choice per direction at dt and keeps the fastest. */
adi_status adi_batch_set_chunk(adi_batch *b, int dir, int K);
adi_status adi_batch_get_chunk(adi_batch *b, int dir, int *K);

/* How a batch step is scheduled.  ADI_BATCH_PERSISTENT (the default): the
 * multi-domain launches above, one per sweep.  ADI_BATCH_MEMBER_GRAPHS: every
 * member's own step (its solver, its autotuned kernels and shapes: what adi_step
 * runs), the members spread over `branches` (1..4) concurrent streams, largest
 * first by cells, forked from and joined back into the batch's stream; captured,
 * the streams are parallel branches of one graph, so one member's launch tails
 * and launch gaps overlap another member's sweeps.  Results are those of each
 * member's adi_step; the divergence guard is the same (no member advances). */
enum { ADI_BATCH_PERSISTENT = 0, ADI_BATCH_MEMBER_GRAPHS = 1 };
adi_status adi_batch_set_schedule(adi_batch *b, int schedule, int branches);
adi_status adi_batch_get_schedule(adi_batch *b, int *schedule, int *branches);

/* Picks the chunk length per direction by timing one batched sweep per choice,
 * then the schedule by timing whole steps (num_global 1, num_local 2) of the
 * persistent schedule and of the member-graph schedule with 1 to 4 branches
 * (replayed graphs, reps each after one untimed).  The timed steps rewrite the
 * next, half and nonlinear layers only and apply the boundary update to the
 * current state, as the next step would. */
adi_status adi_batch_autotune(adi_batch *b, double dt, int reps);

/* Mean time in ms of one whole batch step (num_global, num_local, no divergence
 * error) with the current schedule: reps replays of its graph after one untimed. */
adi_status adi_batch_time_step(adi_batch *b, double dt, int num_global, int num_local, int reps, float *ms_out);

/* Mean time in ms of one batched sweep launch per direction X, Y, Z (reps timed
 * launches after one untimed, at dt; the launches write half and the nonlinear
 * buffers only, which every step rewrites before reading). */
adi_status adi_batch_time_sweeps(adi_batch *b, double dt, int reps, float *ms_out3);

/* Graph replay on (default) or off; kernel launches issued so far. */
adi_status adi_batch_set_graphs(adi_batch *b, int on);
adi_status adi_batch_launches(adi_batch *b, int64_t *out);
const char *adi_batch_last_error_string(const adi_batch *b);

/* ---- allocation-free sweep ----------------------------------------------- */

/* This entry point has no counterpart in the reference: it exists for callers
 * that cannot allocate device memory while they run -- hosts whose device memory
 * is owned by their own pool allocator, time loops that must not pay cudaMalloc's
 * implicit synchronisation and latency, and code running where allocation is not
 * allowed.  It performs one exact sweep of one direction (the arithmetic of the
 * ADI_SOLVER_EXACT path: Thomas per segment, reference operation order) on device
 * arrays the caller owns and allocates nothing:
 *   - no handle and no segment lists: each line finds its own segments;
 *   - the elimination scratch is one fixed static device array of
 *     adi_static_scratch_bytes() (16 MiB), compiled into the library; every GPU
 *     that loads the library holds it until the process exits.  Lines are
 *     processed in batches that fit it (one launch per batch, in stream order).
 *     A line longer than 16 MiB / (6 * 128 * element size) nodes (5461 in float,
 *     2730 in double) is rejected with ADI_ERR_CAPACITY.
 *   - every call shares that array and leaves its last contents behind; each
 *     scratch value a launch reads was written earlier in the same launch by the
 *     same thread, so nothing needs clearing.  Calls whose work overlaps on the GPU
 *     (different streams, or different host threads on one device) race on the
 *     array: serialise them, e.g. issue them on one stream.
 *   - every call looks up the array's device address (cudaGetSymbolAddress)
 *     with the caller's device current, so it stays right after a device reset
 *     or in a non-primary driver context; the first call on a device also loads
 *     the library's module there, so make that first call before any stream
 *     capture.
 * All pointers are device pointers in the precision's element type, except the
 * three uint8 node arrays (Grid3D Node SoA).  temp_in and temp_out must not
 * alias each other or cur; next must not alias cur or temp_in.  merges is 1, or 2
 * for the sweep that also carries the per-iteration extra merge.  Asynchronous
 * on `stream`.
 * The node arrays should meet adi_set_mask's solver contract (no NODE_IN cell on
 * the outer frame or next to NODE_OUT, no BC_FREE cell between two fluid runs of
 * a line); they are not checked on the host.  Lines whose rows would read outside
 * the arrays -- a NODE_IN cell at either end of the line, or any NODE_IN cell in a
 * line on the outer frame -- are skipped by the kernel (left unwritten); other
 * violations give the reference's arithmetic on the given mask.
 * Errors: ADI_ERR_BAD_ARG, ADI_ERR_CAPACITY, or ADI_ERR_CUDA when a CUDA error is
 * pending before the call or a launch fails.  There is no handle and so no
 * message string; the CUDA error is left pending for the caller's
 * cudaGetLastError. */
typedef struct adi_static_sweep_args {
    int dir;                  /* ADI_X, ADI_Y or ADI_Z */
    int dimx, dimy, dimz;
    double dx, dy, dz, dt;
    adi_fluid_params params;
    int precision;            /* ADI_FP32 or ADI_FP64 */
    int merges;               /* 1 or 2 */
    const uint8_t *node_type, *bc_vel, *bc_temp;
    const void *node_value[4];  /* v.x v.y v.z T */
    const void *cur[4];
    const void *temp_in[4];
    void *next[4];
    void *temp_out[4];
    void *stream;             /* cudaStream_t; NULL = legacy default stream */
} adi_static_sweep_args;

adi_status adi_sweep_exact_static(const adi_static_sweep_args *args);

/* Size in bytes of the fixed scratch array used by adi_sweep_exact_static. */
size_t adi_static_scratch_bytes(void);

/* Library build/version string. */
const char *adi_version(void);

/* ---- result files ------------------------------------------------------- */

/* The reference's result file (Common/IO.h:136-276 OutputNetCDF3D_header and
 * :340-377 OutputNetCDF3D_layer, called from FluidSolver3D.cpp:206 and :258) with the
 * same dimensions (x, y, z, unlimited t), variables (x, y, z float axes; time double
 * [t]; u, v, w, T double [t][x][y][z]; d float [x][y]), attributes and values,
 * written as a NetCDF classic file (64-bit offset format) because no NetCDF-4 /
 * HDF5 library is available here; any NetCDF reader opens it.  Host code, no
 * device.
 *
 * adi_nc_write_header: creates `path`; vars is the reference's out_vars list as
 * comma-separated short names ("u,v,w,T,d"); the time axis holds time / timestep
 * records (their data the fill value until written); depth (depth_nx x depth_ny,
 * [x][y]) is point-sampled to the output grid as DepthInfo3D does and needed only
 * when vars names "d"; xy_degree_units: the x / y axes' units are degree_north /
 * degree_east instead of metres.  ADI_ERR_BAD_ARG for a file that cannot be written,
 * a negative time, more than 1e7 records, or one record of a variable above the
 * format's 4 GiB (outdimx * outdimy * outdimz * 8 bytes).
 * adi_nc_write_layer: writes record `layer` of every data variable vars names
 * (except d) from vel (3 values per cell, float or double: vel_elem_bytes 4 or 8,
 * as Vec3D holds FTYPE) and T (double), cells [x][y][z] as GetLayer gives them;
 * a layer past the last record extends the record count. */
typedef struct {
    float pmin[3], pmax[3];   /* BBox3D pMin, pMax */
} adi_bbox3d;
adi_status adi_nc_write_header(const char *path, const adi_bbox3d *bbox, const float *depth, int depth_nx,
                               int depth_ny, double timestep, double time, int outdimx, int outdimy, int outdimz,
                               const char *vars, int xy_degree_units);
adi_status adi_nc_write_layer(const char *path, const void *vel, int vel_elem_bytes, const double *T, int layer,
                              int outdimx, int outdimy, int outdimz, const char *vars);

#ifdef __cplusplus
}
#endif

#endif /* ADI_B200_H */
