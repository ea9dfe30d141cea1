/* CPU restatement oracle of the reference's 3D ADI time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load liboracle_adi.so, and only as the checker:
 * the product (libadi_b200.so) never links or calls it.
 *
 * The float instantiation is pinned bit for bit against the reference's own CPU
 * solver compiled from its sources (oracle/_ref/libref3d.so, built by
 * oracle/Makefile; tests/test_oracle_pin.py and the committed golden fixtures in
 * tests/golden/).  The double instantiation is the same code with REAL=double:
 * the FP64 oracle the product's float results are measured against.
 *
 * Segment lists restate Grid3D::GenerateListSegments (Grid3D.cpp:47-127) with
 * nblockZ = 1 (the single-domain path); the time step restates the CPU branch
 * of AdiSolver3D::TimeStep (AdiSolver3D.cpp:306-391); see adi_oracle_body.h for
 * the per-function citations.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Common/Geometry.h:31-41 */
enum { NODE_IN_ = 0, NODE_OUT_ = 1, NODE_BOUND_ = 2, NODE_VALVE_ = 3 };
enum { BC_NOSLIP_ = 0, BC_FREE_ = 1 };

typedef struct {
    int pos[3], end[3];
    int size;
} seg_t;

typedef struct {
    seg_t *seg;
    int count;
} seg_list;

/* Grid3D::GenerateListSegments for one direction (0 X, 1 Y, 2 Z).  Lines are
 * visited in the reference's order (X: y then z; Y: x then z; Z: x then y, the
 * second index fastest).  Along a line, a segment opens at the cell before the
 * first IN cell of a run and closes at the first non-IN cell after it; a run
 * that reaches the last cell of the line is dropped.  Returns the count, or -1
 * when cap is too small (out may be NULL to count only). */
int oracle_segments(const uint8_t *type, int nx, int ny, int nz, int dir, int32_t *out7, int cap)
{
    int dims[3] = {nx, ny, nz};
    int a2 = dir == 0 ? 1 : 0;       /* axis of the outer loop */
    int a3 = dir == 2 ? 1 : 2;       /* axis of the inner loop */
    int count = 0;
    for (int i = 0; i < dims[a2]; i++)
        for (int j = 0; j < dims[a3]; j++) {
            int p[3] = {0, 0, 0};
            p[a2] = i;
            p[a3] = j;
            int state = 0, start = 0;
            for (int q = 0; q + 1 < dims[dir]; q++) {
                p[dir] = q + 1;
                int in = type[((size_t)p[0] * ny + p[1]) * nz + p[2]] == NODE_IN_;
                if (in) {
                    if (!state) start = q;
                    state = 1;
                } else if (state) {
                    if (out7) {
                        if (count >= cap) return -1;
                        int32_t *o = out7 + 7 * (size_t)count;
                        o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
                        o[dir] = start;
                        o[3] = p[0]; o[4] = p[1]; o[5] = p[2];
                        o[6] = q + 1 - start + 1;
                    }
                    count++;
                    state = 0;
                }
            }
        }
    return count;
}

static int build_lists(const uint8_t *type, int nx, int ny, int nz, seg_list out[3])
{
    for (int dir = 0; dir < 3; dir++) {
        int n = oracle_segments(type, nx, ny, nz, dir, NULL, 0);
        int32_t *raw = (int32_t *)malloc(sizeof(int32_t) * 7 * (size_t)(n > 0 ? n : 1));
        out[dir].seg = (seg_t *)malloc(sizeof(seg_t) * (size_t)(n > 0 ? n : 1));
        out[dir].count = n;
        if (!raw || !out[dir].seg) { free(raw); return -1; }
        oracle_segments(type, nx, ny, nz, dir, raw, n);
        for (int s = 0; s < n; s++) {
            seg_t *g = &out[dir].seg[s];
            for (int c = 0; c < 3; c++) { g->pos[c] = raw[7 * s + c]; g->end[c] = raw[7 * s + 3 + c]; }
            g->size = raw[7 * s + 6];
        }
        free(raw);
    }
    return 0;
}

#define REAL float
#define SFX _f32
#include "adi_oracle_body.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX _f64
#include "adi_oracle_body.h"
#undef REAL
#undef SFX

#include "adi_oracle_adjoint.h"

/* ------------------------------------------------------------------------ */
/* C ABI used by the tests (ctypes).                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int precision; /* 4 float, 8 double */
    void *s;
} oracle_h;

#define ALLOC_SOLVER(T, SUFFIX)                                                                 \
    do {                                                                                         \
        T *s = (T *)calloc(1, sizeof(T));                                                        \
        size_t n = (size_t)nx * ny * nz;                                                         \
        s->nx = nx; s->ny = ny; s->nz = nz;                                                      \
        s->dx = dx; s->dy = dy; s->dz = dz;                                                      \
        s->type = h_type; s->bc_vel = h_bcv; s->bc_temp = h_bct;                                 \
        const double *src[4] = {vx, vy, vz, T_};                                                 \
        for (int v = 0; v < 4; v++) {                                                            \
            s->nv[v] = calloc(n, sizeof(*s->nv[v]));                                             \
            for (size_t q = 0; q < n; q++) s->nv[v][q] = src[v][q];                              \
        }                                                                                        \
        for (int l = 0; l < 4; l++)                                                              \
            for (int v = 0; v < 4; v++) s->L[l].f[v] = calloc(n, sizeof(*s->L[l].f[v]));         \
        s->cur = 0; s->next = 1; s->half = 2; s->temp = 3;                                       \
        for (int v = 0; v < 4; v++) memcpy(s->L[0].f[v], s->nv[v], n * sizeof(*s->nv[v]));      \
        s->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();                           \
        int mx = nx > ny ? nx : ny; mx = mx > nz ? mx : nz;                                      \
        s->scratch = calloc((size_t)s->nthreads * 5 * mx, sizeof(*s->scratch));                  \
        build_lists(h_type, nx, ny, nz, s->segs);                                                \
        h->s = s;                                                                                \
        (void)SUFFIX;                                                                            \
    } while (0)

/* Creates an oracle domain.  Node arrays are [i][j][k] with k fastest; the
 * initial state of every field is the node values (TimeLayer3D(grid) ->
 * CopyFromGrid, TimeLayer3D.h:1077-1090,734-781). */
void *oracle_create(int precision, int nthreads, int nx, int ny, int nz, double dx, double dy, double dz,
                    const uint8_t *type, const uint8_t *bc_vel, const uint8_t *bc_temp,
                    const double *vx, const double *vy, const double *vz, const double *T_)
{
    oracle_h *h = (oracle_h *)calloc(1, sizeof(oracle_h));
    size_t n = (size_t)nx * ny * nz;
    uint8_t *h_type = malloc(n), *h_bcv = malloc(n), *h_bct = malloc(n);
    memcpy(h_type, type, n); memcpy(h_bcv, bc_vel, n); memcpy(h_bct, bc_temp, n);
    h->precision = precision;
    if (precision == 8) ALLOC_SOLVER(solver_f64, 0);
    else ALLOC_SOLVER(solver_f32, 0);
    return h;
}

/* FluidParams values (v_T, v_vis, t_vis, t_phi) as doubles; they are rounded
 * to the working precision here, as FluidParams' (FTYPE) casts do. */
int oracle_set_params(void *vh, double v_T, double v_vis, double t_vis, double t_phi)
{
    oracle_h *h = (oracle_h *)vh;
    if (h->precision == 8) {
        solver_f64 *s = h->s; s->v_T = v_T; s->v_vis = v_vis; s->t_vis = t_vis; s->t_phi = t_phi;
    } else {
        solver_f32 *s = h->s; s->v_T = (float)v_T; s->v_vis = (float)v_vis; s->t_vis = (float)t_vis; s->t_phi = (float)t_phi;
    }
    return 0;
}

int oracle_step(void *vh, double dt, int num_global, int num_local, int compute_error)
{
    oracle_h *h = (oracle_h *)vh;
    if (h->precision == 8) return step_f64(h->s, dt, num_global, num_local, compute_error, 1);
    return step_f32(h->s, dt, num_global, num_local, compute_error, 1);
}

/* adi_step_tol's semantics (tolerance mode), for its parity tests. */
int oracle_step_tol(void *vh, double dt, int max_global, int num_local, double tol, int compute_error, int *iters,
                    double *res)
{
    oracle_h *h = (oracle_h *)vh;
    if (h->precision == 8) return step_tol_f64(h->s, dt, max_global, num_local, tol, compute_error, iters, res);
    return step_tol_f32(h->s, dt, max_global, num_local, tol, compute_error, iters, res);
}

/* TimeStep alone (AdiSolver3D.cpp:306-391), without UpdateBoundaries. */
int oracle_time_step(void *vh, double dt, int num_global, int num_local, int compute_error)
{
    oracle_h *h = (oracle_h *)vh;
    if (h->precision == 8) return step_f64(h->s, dt, num_global, num_local, compute_error, 0);
    return step_f32(h->s, dt, num_global, num_local, compute_error, 0);
}

/* which: 0 cur, 1 next, 2 half, 3 temp.  Output as double. */
int oracle_get_fields(void *vh, int which, double *u, double *v, double *w, double *T_)
{
    oracle_h *h = (oracle_h *)vh;
    double *dst[4] = {u, v, w, T_};
    if (h->precision == 8) {
        solver_f64 *s = h->s;
        int idx[4] = {s->cur, s->next, s->half, s->temp};
        size_t n = (size_t)s->nx * s->ny * s->nz;
        for (int f = 0; f < 4; f++) memcpy(dst[f], s->L[idx[which]].f[f], n * sizeof(double));
    } else {
        solver_f32 *s = h->s;
        int idx[4] = {s->cur, s->next, s->half, s->temp};
        size_t n = (size_t)s->nx * s->ny * s->nz;
        for (int f = 0; f < 4; f++)
            for (size_t q = 0; q < n; q++) dst[f][q] = s->L[idx[which]].f[f][q];
    }
    return 0;
}

int oracle_set_state(void *vh, const double *u, const double *v, const double *w, const double *T_)
{
    oracle_h *h = (oracle_h *)vh;
    const double *src[4] = {u, v, w, T_};
    if (h->precision == 8) {
        solver_f64 *s = h->s;
        size_t n = (size_t)s->nx * s->ny * s->nz;
        for (int f = 0; f < 4; f++) memcpy(s->L[s->cur].f[f], src[f], n * sizeof(double));
    } else {
        solver_f32 *s = h->s;
        size_t n = (size_t)s->nx * s->ny * s->nz;
        for (int f = 0; f < 4; f++)
            for (size_t q = 0; q < n; q++) s->L[s->cur].f[f][q] = (float)src[f][q];
    }
    return 0;
}

double oracle_div_error(void *vh)
{
    oracle_h *h = (oracle_h *)vh;
    if (h->precision == 8) { solver_f64 *s = h->s; return div_error_f64(s, &s->L[s->cur]); }
    solver_f32 *s = h->s;
    return div_error_f32(s, &s->L[s->cur]);
}

double oracle_last_div_error(void *vh)
{
    oracle_h *h = (oracle_h *)vh;
    if (h->precision == 8) return ((solver_f64 *)h->s)->diff_error;
    return ((solver_f32 *)h->s)->diff_error;
}

/* FP64 discrete adjoint of n_steps adi_step calls from the current state:
 * J = 1/2 sum over NODE_IN cells of the box [lo, hi) of u^2 + v^2 + w^2 after the
 * steps; nv_grad = dJ/d(node values), state_grad = dJ/d(initial state), each 4
 * fields [i][j][k].  The handle ends at the final state.  No divergence guard.
 * Returns 0, or -1 for a float handle. */
int oracle_adjoint_run(void *vh, double dt, int num_global, int num_local, int n_steps, const int *lo,
                       const int *hi, double *J, double *nv_grad, double *state_grad)
{
    oracle_h *h = (oracle_h *)vh;
    if (h->precision != 8) return -1;
    solver_f64 *s = h->s;
    size_t n = adj_n(s);
    int S = num_global * num_local * 3;
    layer_f64 *states = calloc((size_t)n_steps + 1, sizeof(layer_f64));
    for (int t = 0; t <= n_steps; t++) adj_alloc(&states[t], n);
    for (int t = 0; t < n_steps; t++) {
        adj_copy(&states[t], &s->L[s->cur], n);
        step_f64(s, dt, num_global, num_local, 0, 1);
    }
    adj_copy(&states[n_steps], &s->L[s->cur], n);
    layer_f64 cbar, nvbar, nbar, hbar, tbar, xb;
    adj_alloc(&cbar, n); adj_alloc(&nvbar, n); adj_alloc(&nbar, n);
    adj_alloc(&hbar, n); adj_alloc(&tbar, n); adj_alloc(&xb, n);
    double acc = 0.0;
    for (int i = lo[0]; i < hi[0]; i++)
        for (int j = lo[1]; j < hi[1]; j++)
            for (int k = lo[2]; k < hi[2]; k++) {
                size_t id = ((size_t)i * s->ny + j) * s->nz + k;
                if (s->type[id] != NODE_IN_) continue;
                for (int v = 0; v < 3; v++) {
                    double x = states[n_steps].f[v][id];
                    acc += x * x;
                    cbar.f[v][id] = x;
                }
            }
    *J = 0.5 * acc;
    layer_f64 *Ti = calloc((size_t)S, sizeof(layer_f64)), *X = calloc((size_t)S, sizeof(layer_f64));
    for (int q = 0; q < S; q++) { adj_alloc(&Ti[q], n); adj_alloc(&X[q], n); }
    for (int t = n_steps - 1; t >= 0; t--) {
        adj_copy(&s->L[s->cur], &states[t], n);
        adj_step_with_tape(s, dt, num_global, num_local, Ti, X);
        adj_step(s, dt, num_global, num_local, Ti, X, &cbar, &nvbar, &nbar, &hbar, &tbar, &xb);
    }
    adj_copy(&s->L[s->cur], &states[n_steps], n);
    for (int v = 0; v < 4; v++) {
        memcpy(nv_grad + (size_t)v * n, nvbar.f[v], n * sizeof(double));
        memcpy(state_grad + (size_t)v * n, cbar.f[v], n * sizeof(double));
    }
    for (int q = 0; q < S; q++) { adj_free(&Ti[q]); adj_free(&X[q]); }
    free(Ti); free(X);
    for (int t = 0; t <= n_steps; t++) adj_free(&states[t]);
    free(states);
    adj_free(&cbar); adj_free(&nvbar); adj_free(&nbar); adj_free(&hbar); adj_free(&tbar); adj_free(&xb);
    return 0;
}

/* Replaces the node values (boundary data) of a handle; the state is unchanged. */
int oracle_set_node_values(void *vh, const double *vx, const double *vy, const double *vz, const double *T_)
{
    oracle_h *h = (oracle_h *)vh;
    const double *src[4] = {vx, vy, vz, T_};
    if (h->precision == 8) {
        solver_f64 *s = h->s;
        size_t n = (size_t)s->nx * s->ny * s->nz;
        for (int v = 0; v < 4; v++) memcpy(s->nv[v], src[v], n * sizeof(double));
    } else {
        solver_f32 *s = h->s;
        size_t n = (size_t)s->nx * s->ny * s->nz;
        for (int v = 0; v < 4; v++)
            for (size_t q = 0; q < n; q++) s->nv[v][q] = (float)src[v][q];
    }
    return 0;
}

#define FREE_SOLVER(T)                                                              \
    do {                                                                             \
        T *s = (T *)h->s;                                                            \
        for (int v = 0; v < 4; v++) free(s->nv[v]);                                  \
        for (int l = 0; l < 4; l++) for (int v = 0; v < 4; v++) free(s->L[l].f[v]);  \
        for (int d = 0; d < 3; d++) free(s->segs[d].seg);                            \
        free(s->scratch);                                                            \
        free((void *)s->type); free((void *)s->bc_vel); free((void *)s->bc_temp);   \
        free(s);                                                                     \
    } while (0)

void oracle_destroy(void *vh)
{
    oracle_h *h = (oracle_h *)vh;
    if (!h) return;
    if (h->precision == 8) FREE_SOLVER(solver_f64);
    else FREE_SOLVER(solver_f32);
    free(h);
}
