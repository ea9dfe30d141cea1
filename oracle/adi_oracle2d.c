/* CPU restatement oracle of the reference's 2D ADI solver (AdiSolver2D).
 *
 * TEST INFRASTRUCTURE ONLY: only tests/ and the CPU-baseline leg of bench.py load
 * liboracle_adi2d.so, as the checker.  The float instantiation is pinned bit for
 * bit against the reference's own 2D solver compiled from its sources
 * (oracle/_ref/libref2d.so, oracle/ref2d_harness.cpp); the double instantiation is
 * the FP64 oracle.  Per-function citations are in adi_oracle2d_body.h.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Common/Geometry.h:31-41 */
enum { NODE_IN_ = 0, NODE_OUT_ = 1, NODE_BOUND_ = 2, NODE_VALVE_ = 3 };
enum { BC_NOSLIP_ = 0, BC_FREE_ = 1 };

typedef struct {
    int posx, posy, endx, endy, size;
    int dir; /* 0 X, 1 Y */
} seg2_t;

static float absr_f32(float x) { return fabsf(x); }
static double absr_f64(double x) { return fabs(x); }

#define REAL float
#define SFX _f32
#include "adi_oracle2d_body.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX _f64
#include "adi_oracle2d_body.h"
#undef REAL
#undef SFX

/* AdiSolver2D::CreateSegments (AdiSolver2D.cpp:228-277): listX holds one
 * Y-direction segment per column i, listY one X-direction segment per row j. */
static void make_segments_row_spanning(const uint8_t *type, int nx, int ny, seg2_t *segx, seg2_t *segy, int *ncx,
                                       int *ncy)
{
    int cx = 0, cy = 0;
#define T_(i, j) type[(size_t)(i) * ny + (j)]
    for (int i = 0; i < nx; i++) {
        seg2_t g;
        g.posx = i;
        g.dir = 1;
        int j = 0;
        while (j < ny && T_(i, j) == NODE_OUT_) j++;
        while (j + 1 < ny && T_(i, j + 1) != NODE_IN_) j++;
        if (j + 1 >= ny) continue;
        g.posy = j;
        j = ny - 1;
        while (j >= 0 && T_(i, j) == NODE_OUT_) j--;
        while (j - 1 >= 0 && T_(i, j - 1) != NODE_IN_) j--;
        g.size = j - g.posy + 1;
        g.endx = i;
        g.endy = j;
        segx[cx++] = g;
    }
    for (int j = 0; j < ny; j++) {
        seg2_t g;
        g.posy = j;
        g.dir = 0;
        int i = 0;
        while (i < nx && T_(i, j) == NODE_OUT_) i++;
        while (i + 1 < nx && T_(i + 1, j) != NODE_IN_) i++;
        if (i + 1 >= nx) continue;
        g.posx = i;
        i = nx - 1;
        while (i >= 0 && T_(i, j) == NODE_OUT_) i--;
        while (i - 1 >= 0 && T_(i - 1, j) != NODE_IN_) i--;
        g.size = i - g.posx + 1;
        g.endx = i;
        g.endy = j;
        segy[cy++] = g;
    }
#undef T_
    *ncx = cx;
    *ncy = cy;
}

/* Masked segments, the 3D solver's segmentation (Grid3D::GenerateListSegments,
 * Grid3D.cpp:47-127) applied to the 2D grid's columns and rows: every maximal run
 * of IN nodes with the non-IN node on each side as its boundary rows, so solid
 * cells inside the box are never solved as fluid.  A run that reaches the last
 * node of a line has no closing node and is dropped, as there. */
static void make_segments_masked(const uint8_t *type, int nx, int ny, seg2_t *segx, seg2_t *segy, int *ncx, int *ncy)
{
    int cx = 0, cy = 0;
    for (int dir = 1; dir >= 0; dir--) {
        const int nlines = dir == 1 ? nx : ny, len = dir == 1 ? ny : nx;
        for (int l = 0; l < nlines; l++) {
            int open = -1;
            for (int p = 0; p + 1 < len; p++) {
                const size_t nxt = dir == 1 ? (size_t)l * ny + (p + 1) : (size_t)(p + 1) * ny + l;
                const int in_next = type[nxt] == NODE_IN_;
                if (open < 0 && in_next) open = p;
                else if (open >= 0 && !in_next) {
                    seg2_t g;
                    g.dir = dir;
                    g.size = p + 1 - open + 1;
                    if (dir == 1) { g.posx = g.endx = l; g.posy = open; g.endy = p + 1; segx[cx++] = g; }
                    else { g.posy = g.endy = l; g.posx = open; g.endx = p + 1; segy[cy++] = g; }
                    open = -1;
                }
            }
        }
    }
    *ncx = cx;
    *ncy = cy;
}

/* mode 0: the reference's row-spanning segments; mode 1: masked segments. */
static void make_segments(const uint8_t *type, int nx, int ny, int mode, seg2_t **segx, seg2_t **segy, int *ncx,
                          int *ncy)
{
    /* a line of n nodes holds at most n / 2 masked segments */
    *segx = calloc((size_t)nx * (ny / 2 + 1), sizeof(seg2_t));
    *segy = calloc((size_t)ny * (nx / 2 + 1), sizeof(seg2_t));
    if (mode == 1) make_segments_masked(type, nx, ny, *segx, *segy, ncx, ncy);
    else make_segments_row_spanning(type, nx, ny, *segx, *segy, ncx, ncy);
}

typedef struct {
    int precision;
    void *s;
} oracle2d_h;

#define ALLOC2(T, SUF)                                                                    \
    do {                                                                                  \
        T *s = calloc(1, sizeof(T));                                                      \
        size_t n = (size_t)nx * ny;                                                       \
        s->nx = nx; s->ny = ny; s->dx = dx; s->dy = dy; s->startT = startT;               \
        uint8_t *t = malloc(n), *b = malloc(n);                                           \
        memcpy(t, type, n); memcpy(b, bct, n);                                            \
        s->type = t; s->bct = b;                                                          \
        s->du = calloc(n, sizeof(*s->du)); s->dv = calloc(n, sizeof(*s->dv));             \
        s->dt_ = calloc(n, sizeof(*s->dt_));                                              \
        for (size_t q = 0; q < n; q++) { s->du[q] = vx[q]; s->dv[q] = vy[q]; s->dt_[q] = T_[q]; } \
        l2_alloc##SUF(&s->cur, n); l2_alloc##SUF(&s->next, n); l2_alloc##SUF(&s->half, n); \
        l2_alloc##SUF(&s->temp, n); l2_alloc##SUF(&s->next_local, n);                     \
        /* AdiSolver2D::Init: cur = node data everywhere (AdiSolver2D.cpp:35-47) */        \
        for (size_t q = 0; q < n; q++) { s->cur.u[q] = s->du[q]; s->cur.v[q] = s->dv[q]; s->cur.t[q] = s->dt_[q]; } \
        make_segments(t, nx, ny, 0, &s->segx, &s->segy, &s->nsegx, &s->nsegy);            \
        h->s = s;                                                                         \
    } while (0)

void *oracle2d_create(int precision, int nx, int ny, double dx, double dy, double startT, const uint8_t *type,
                      const uint8_t *bct, const double *vx, const double *vy, const double *T_)
{
    oracle2d_h *h = calloc(1, sizeof(oracle2d_h));
    h->precision = precision;
    if (precision == 8) ALLOC2(solver2_f64, _f64);
    else ALLOC2(solver2_f32, _f32);
    return h;
}

int oracle2d_set_params(void *vh, double v_T, double v_vis, double t_vis, double t_phi)
{
    oracle2d_h *h = vh;
    if (h->precision == 8) {
        solver2_f64 *s = h->s; s->v_T = v_T; s->v_vis = v_vis; s->t_vis = t_vis; s->t_phi = t_phi;
    } else {
        solver2_f32 *s = h->s;
        s->v_T = (float)v_T; s->v_vis = (float)v_vis; s->t_vis = (float)t_vis; s->t_phi = (float)t_phi;
    }
    return 0;
}

/* UpdateBoundaries + TimeStep: the 2D driver loop (FluidSolver2D.cpp:131-132).
 * Returns the global iterations run, or -1 where the reference exits. */
int oracle2d_step(void *vh, double dt, int num_global, int num_local)
{
    oracle2d_h *h = vh;
    if (h->precision == 8) {
        solver2_f64 *s = h->s;
        update_bnd2_f64(s);
        return time_step2_f64(s, dt, num_global, num_local);
    }
    solver2_f32 *s = h->s;
    update_bnd2_f32(s);
    return time_step2_f32(s, (float)dt, num_global, num_local);
}

/* UpdateBoundaries + the tolerance-mode step (time_step2_tol). */
int oracle2d_step_tol(void *vh, double dt, int max_global, int num_local, double tol, double *res)
{
    oracle2d_h *h = vh;
    if (h->precision == 8) {
        solver2_f64 *s = h->s;
        update_bnd2_f64(s);
        return time_step2_tol_f64(s, dt, max_global, num_local, tol, res);
    }
    solver2_f32 *s = h->s;
    update_bnd2_f32(s);
    return time_step2_tol_f32(s, (float)dt, max_global, num_local, tol, res);
}

/* which: 0 cur, 1 next.  Output as double, [i][j]. */
int oracle2d_get_fields(void *vh, int which, double *u, double *v, double *T_)
{
    oracle2d_h *h = vh;
    if (h->precision == 8) {
        solver2_f64 *s = h->s;
        layer2_f64 *l = which ? &s->next : &s->cur;
        size_t n = (size_t)s->nx * s->ny;
        memcpy(u, l->u, n * 8); memcpy(v, l->v, n * 8); memcpy(T_, l->t, n * 8);
    } else {
        solver2_f32 *s = h->s;
        layer2_f32 *l = which ? &s->next : &s->cur;
        size_t n = (size_t)s->nx * s->ny;
        for (size_t q = 0; q < n; q++) { u[q] = l->u[q]; v[q] = l->v[q]; T_[q] = l->t[q]; }
    }
    return 0;
}

double oracle2d_last_err(void *vh)
{
    oracle2d_h *h = vh;
    return h->precision == 8 ? ((solver2_f64 *)h->s)->last_err : ((solver2_f32 *)h->s)->last_err;
}

/* Rebuilds the segment lists: mode 0 the reference's row-spanning segments
 * (the default), mode 1 masked segments.  Returns the segment count, -1 on a bad
 * mode. */
int oracle2d_set_segments(void *vh, int mode)
{
    oracle2d_h *h = vh;
    if (mode != 0 && mode != 1) return -1;
    if (h->precision == 8) {
        solver2_f64 *s = h->s;
        free(s->segx); free(s->segy);
        make_segments(s->type, s->nx, s->ny, mode, &s->segx, &s->segy, &s->nsegx, &s->nsegy);
        return s->nsegx + s->nsegy;
    }
    solver2_f32 *s = h->s;
    free(s->segx); free(s->segy);
    make_segments(s->type, s->nx, s->ny, mode, &s->segx, &s->segy, &s->nsegx, &s->nsegy);
    return s->nsegx + s->nsegy;
}

/* Segments as int32 [posx posy endx endy size dir] rows: listX then listY. */
int oracle2d_segments(void *vh, int32_t *out6, int cap)
{
    oracle2d_h *h = vh;
    seg2_t *a, *b;
    int na, nb;
    if (h->precision == 8) { solver2_f64 *s = h->s; a = s->segx; b = s->segy; na = s->nsegx; nb = s->nsegy; }
    else { solver2_f32 *s = h->s; a = s->segx; b = s->segy; na = s->nsegx; nb = s->nsegy; }
    if (!out6) return na + nb;
    if (cap < na + nb) return -1;
    for (int q = 0; q < na + nb; q++) {
        seg2_t *g = q < na ? &a[q] : &b[q - na];
        int32_t *o = out6 + 6 * q;
        o[0] = g->posx; o[1] = g->posy; o[2] = g->endx; o[3] = g->endy; o[4] = g->size; o[5] = g->dir;
    }
    return na + nb;
}

#define FREE2(T, SUF)                                                                   \
    do {                                                                                \
        T *s = h->s;                                                                    \
        l2_free##SUF(&s->cur); l2_free##SUF(&s->next); l2_free##SUF(&s->half);          \
        l2_free##SUF(&s->temp); l2_free##SUF(&s->next_local);                           \
        free(s->du); free(s->dv); free(s->dt_); free((void *)s->type); free((void *)s->bct); \
        free(s->segx); free(s->segy); free(s);                                          \
    } while (0)

void oracle2d_destroy(void *vh)
{
    oracle2d_h *h = vh;
    if (!h) return;
    if (h->precision == 8) FREE2(solver2_f64, _f64);
    else FREE2(solver2_f32, _f32);
    free(h);
}
