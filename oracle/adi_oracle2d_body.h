/* Precision-generic body of the 2D CPU restatement oracle (the reference's
 * AdiSolver2D).  Included twice by adi_oracle2d.c (REAL=float, SFX=_f32 and
 * REAL=double, SFX=_f64).  TEST INFRASTRUCTURE ONLY.
 *
 * Operation by operation, in the reference's operand order:
 *   segments            AdiSolver2D.cpp:228-277  (CreateSegments: one segment per
 *                       row/column, from the node before the first IN to the node
 *                       after the last IN; obstacles inside are ordinary rows)
 *   bc rows             AdiSolver2D.cpp:74-116   (ApplyBC0/1 by the node's BC type,
 *                       the same for every variable; FREE rows x0 - x1 = 0)
 *   matrix rows         AdiSolver2D.cpp:118-178  (BuildMatrix: 1/dt, advection by
 *                       temp_local U (X) / V (Y))
 *   Thomas              Common/Algorithms.h:21-39
 *   one direction       AdiSolver2D.cpp:203-226  (copy-then-merge on temp_local)
 *   one time step       AdiSolver2D.cpp:279-323  (global loop while it < num_global
 *                       or err > 0.1)
 *   boundaries          Solver2D.cpp:40-54, :68-80 (UpdateBoundaries, ClearOutterCells)
 *   layer copies        TimeLayer2D.h:98-176     (loops stop at dimx-1, dimy-1: the
 *                       last row and column are never copied or merged)
 *   divergence error    TimeLayer2D.h:86-100     (as written: dy*(dU) + (dU')/2,
 *                       accumulated in REAL)
 * Layers the reference allocates with new[] and never fully writes (the last row
 * and column of temp, half, next, next_local and of every temp_local) start at
 * zero here; the reference harness makes new[] return zeroed memory so that both
 * read the same values. */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

typedef struct {
    REAL *u, *v, *t;   /* [i][j], j fastest */
} FN(layer2);

typedef struct {
    int nx, ny;
    REAL dx, dy;           /* (FTYPE)grid->dx etc. */
    const uint8_t *type;   /* NodeType */
    const uint8_t *bct;    /* BCtype of the node's data */
    REAL *du, *dv, *dt_;   /* node data: vel.x, vel.y, T */
    REAL startT;
    REAL v_T, v_vis, t_vis, t_phi;
    FN(layer2) cur, next, half, temp, next_local;
    seg2_t *segx, *segy;   /* listX (columns, dir Y), listY (rows, dir X) */
    int nsegx, nsegy;
    int last_iters;
    double last_err;
} FN(solver2);

#define IX(s, i, j) ((size_t)(i) * (s)->ny + (j))

static void FN(l2_alloc)(FN(layer2) *l, size_t n)
{
    l->u = calloc(n, sizeof(REAL));
    l->v = calloc(n, sizeof(REAL));
    l->t = calloc(n, sizeof(REAL));
}

static void FN(l2_free)(FN(layer2) *l)
{
    free(l->u); free(l->v); free(l->t);
}

static REAL *FN(fld)(FN(layer2) *l, int var) { return var == 0 ? l->u : (var == 1 ? l->v : l->t); }

/* CopyAllto(grid, dest, type) / MergeAllto: i < nx-1, j < ny-1 only. */
static void FN(copy_type)(FN(solver2) *s, FN(layer2) *src, FN(layer2) *dst, int type)
{
    for (int var = 0; var < 3; var++) {
        REAL *a = FN(fld)(src, var), *b = FN(fld)(dst, var);
        for (int i = 0; i < s->nx - 1; i++)
            for (int j = 0; j < s->ny - 1; j++)
                if (s->type[IX(s, i, j)] == type) b[IX(s, i, j)] = a[IX(s, i, j)];
    }
}

static void FN(copy_all)(FN(solver2) *s, FN(layer2) *src, FN(layer2) *dst)
{
    FN(copy_type)(s, src, dst, NODE_IN_);
    FN(copy_type)(s, src, dst, NODE_OUT_);
    FN(copy_type)(s, src, dst, NODE_BOUND_);
    FN(copy_type)(s, src, dst, NODE_VALVE_);
}

static void FN(merge_in)(FN(solver2) *s, FN(layer2) *src, FN(layer2) *dst)
{
    for (int var = 0; var < 3; var++) {
        REAL *a = FN(fld)(src, var), *b = FN(fld)(dst, var);
        for (int i = 0; i < s->nx - 1; i++)
            for (int j = 0; j < s->ny - 1; j++)
                if (s->type[IX(s, i, j)] == NODE_IN_) b[IX(s, i, j)] = (b[IX(s, i, j)] + a[IX(s, i, j)]) / 2;
    }
}

static double FN(div_err2)(FN(solver2) *s, FN(layer2) *l)
{
    REAL err = 0.0;
    int count = 0;
    for (int i = 0; i < s->nx - 1; i++)
        for (int j = 0; j < s->ny - 1; j++)
            if (s->type[IX(s, i, j)] == NODE_IN_ && s->type[IX(s, i + 1, j)] == NODE_IN_ &&
                s->type[IX(s, i, j + 1)] == NODE_IN_ && s->type[IX(s, i + 1, j + 1)] == NODE_IN_) {
                REAL tx = s->dy * (l->u[IX(s, i + 1, j)] - l->u[IX(s, i, j)]) +
                          (l->u[IX(s, i + 1, j + 1)] - l->u[IX(s, i, j + 1)]) / 2;
                REAL ty = s->dx * (l->v[IX(s, i, j + 1)] - l->v[IX(s, i, j)]) +
                          (l->v[IX(s, i + 1, j + 1)] - l->v[IX(s, i + 1, j)]) / 2;
                err += (REAL)FN(absr)(tx + ty);
                count++;
            }
    return (double)(err / count);
}

static void FN(thomas2)(REAL *a, REAL *b, REAL *c, REAL *d, REAL *x, int num)
{
    c[num - 1] = 0.0;
    c[0] = c[0] / b[0];
    d[0] = d[0] / b[0];
    for (int i = 1; i < num; i++) {
        c[i] = c[i] / (b[i] - a[i] * c[i - 1]);
        d[i] = (d[i] - d[i - 1] * a[i]) / (b[i] - a[i] * c[i - 1]);
    }
    x[num - 1] = d[num - 1];
    for (int i = num - 2; i >= 0; i--)
        x[i] = d[i] - c[i] * x[i + 1];
}

static REAL FN(data_of)(FN(solver2) *s, size_t id, int var) { return var == 0 ? s->du[id] : (var == 1 ? s->dv[id] : s->dt_[id]); }

static void FN(solve_seg2)(FN(solver2) *s, REAL dt, const seg2_t *g, int var, FN(layer2) *cur, FN(layer2) *tl,
                           FN(layer2) *nl, REAL *work)
{
    int n = g->size, mx = s->nx > s->ny ? s->nx : s->ny;
    REAL *a = work, *b = a + mx, *c = b + mx, *d = c + mx, *x = d + mx;
    size_t id0 = IX(s, g->posx, g->posy), id1 = IX(s, g->endx, g->endy);
    /* ApplyBC0 */
    if (s->bct[id0] == BC_FREE_) { b[0] = 1.0; c[0] = -1.0; d[0] = 0.0; }
    else { b[0] = 1.0; c[0] = 0.0; d[0] = FN(data_of)(s, id0, var); }
    /* BuildMatrix */
    REAL vis_x = (var == 2 ? s->t_vis : s->v_vis) / (s->dx * s->dx);
    REAL vis_y = (var == 2 ? s->t_vis : s->v_vis) / (s->dy * s->dy);
    int i = g->posx, j = g->posy;
    for (int p = 1; p < n - 1; p++) {
        if (g->dir == 0) {
            size_t id = IX(s, i + p, j);
            REAL w = tl->u[id];
            a[p] = -w / (2 * s->dx) - vis_x;
            b[p] = 1 / dt + 2 * vis_x;
            c[p] = w / (2 * s->dx) - vis_x;
            if (var == 0) d[p] = cur->u[id] / dt - s->v_T * ((tl->t[IX(s, i + p + 1, j)] - tl->t[IX(s, i + p - 1, j)]) / (2 * s->dx));
            else if (var == 1) d[p] = cur->v[id] / dt;
            else {
                REAL ux = (tl->u[IX(s, i + p + 1, j)] - tl->u[IX(s, i + p - 1, j)]) / (2 * s->dx);
                REAL vx = (tl->v[IX(s, i + p + 1, j)] - tl->v[IX(s, i + p - 1, j)]) / (2 * s->dx);
                REAL uy = (tl->u[IX(s, i + p, j + 1)] - tl->u[IX(s, i + p, j - 1)]) / (2 * s->dy);
                REAL vy = (tl->v[IX(s, i + p, j + 1)] - tl->v[IX(s, i + p, j - 1)]) / (2 * s->dy);
                (void)vy;
                d[p] = cur->t[id] / dt + s->t_phi * (2 * ux * ux + vx * vx + uy * vx);
            }
        } else {
            size_t id = IX(s, i, j + p);
            REAL w = tl->v[id];
            a[p] = -w / (2 * s->dy) - vis_y;
            b[p] = 1 / dt + 2 * vis_y;
            c[p] = w / (2 * s->dy) - vis_y;
            if (var == 0) d[p] = cur->u[id] / dt;
            else if (var == 1) d[p] = cur->v[id] / dt - s->v_T * ((tl->t[IX(s, i, j + p + 1)] - tl->t[IX(s, i, j + p - 1)]) / (2 * s->dy));
            else {
                REAL ux = (tl->u[IX(s, i + 1, j + p)] - tl->u[IX(s, i - 1, j + p)]) / (2 * s->dx);
                REAL vx = (tl->v[IX(s, i + 1, j + p)] - tl->v[IX(s, i - 1, j + p)]) / (2 * s->dx);
                REAL uy = (tl->u[IX(s, i, j + p + 1)] - tl->u[IX(s, i, j + p - 1)]) / (2 * s->dy);
                REAL vy = (tl->v[IX(s, i, j + p + 1)] - tl->v[IX(s, i, j + p - 1)]) / (2 * s->dy);
                (void)ux;
                d[p] = cur->t[id] / dt + s->t_phi * (uy * uy + 2 * vy * vy + vx * uy);
            }
        }
    }
    /* ApplyBC1 */
    if (s->bct[id1] == BC_FREE_) { a[n - 1] = 1.0; b[n - 1] = -1.0; d[n - 1] = 0.0; }
    else { a[n - 1] = 0.0; b[n - 1] = 1.0; d[n - 1] = FN(data_of)(s, id1, var); }
    FN(thomas2)(a, b, c, d, x, n);
    REAL *o = FN(fld)(nl, var);
    for (int t = 0; t < n; t++) {
        if (g->dir == 0) o[IX(s, i + t, j)] = x[t];
        else o[IX(s, i, j + t)] = x[t];
    }
}

/* SolveDirection (AdiSolver2D.cpp:203-226). */
static void FN(solve_dir2)(FN(solver2) *s, REAL dt, int num_local, const seg2_t *list, int nseg, FN(layer2) *cur,
                           FN(layer2) *temp, FN(layer2) *next)
{
    size_t n = (size_t)s->nx * s->ny;
    FN(layer2) tl;
    FN(l2_alloc)(&tl, n);
    FN(copy_all)(s, temp, &tl);
    int mx = s->nx > s->ny ? s->nx : s->ny;
    REAL *work = malloc(sizeof(REAL) * 5 * mx);
    for (int it = 0; it < num_local; it++) {
        for (int q = 0; q < nseg; q++)
            for (int var = 0; var < 3; var++) FN(solve_seg2)(s, dt, &list[q], var, cur, &tl, &s->next_local, work);
        if (it == 0) FN(copy_type)(s, &s->next_local, &tl, NODE_IN_);
        else FN(merge_in)(s, &s->next_local, &tl);
    }
    FN(copy_type)(s, &tl, temp, NODE_IN_);
    FN(copy_type)(s, &s->next_local, next, NODE_IN_);
    free(work);
    FN(l2_free)(&tl);
}

/* Solver2D::UpdateBoundaries (Solver2D.cpp:40-54). */
static void FN(update_bnd2)(FN(solver2) *s)
{
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++) {
            size_t id = IX(s, i, j);
            if (s->type[id] == NODE_BOUND_ || s->type[id] == NODE_VALVE_) {
                s->cur.u[id] = s->du[id];
                s->cur.v[id] = s->dv[id];
                s->cur.t[id] = s->dt_[id];
            }
        }
    FN(copy_type)(s, &s->cur, &s->next, NODE_BOUND_);
    FN(copy_type)(s, &s->cur, &s->next, NODE_VALVE_);
}

/* AdiSolver2D::TimeStep (AdiSolver2D.cpp:279-323).  Returns the number of global
 * iterations, or -1 where the reference calls exit(1). */
static int FN(time_step2)(FN(solver2) *s, REAL dt, int num_global, int num_local)
{
    FN(copy_all)(s, &s->cur, &s->next);
    FN(copy_all)(s, &s->cur, &s->half);
    FN(copy_all)(s, &s->cur, &s->temp);
    double err = FN(div_err2)(s, &s->next);
    int it;
    for (it = 0; (it < num_global) || (err > 0.1); it++) {
        FN(solve_dir2)(s, dt, num_local, s->segy, s->nsegy, &s->cur, &s->temp, &s->half);
        FN(solve_dir2)(s, dt, num_local, s->segx, s->nsegx, &s->half, &s->temp, &s->next);
        err = FN(div_err2)(s, &s->next);
        if (it == 0) FN(copy_type)(s, &s->next, &s->temp, NODE_IN_);
        else FN(merge_in)(s, &s->next, &s->temp);
        if (it > 100 || err > 0.1 * 10) { s->last_err = err; return -1; }
    }
    /* ClearOutterCells (Solver2D.cpp:68-80) */
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            if (s->type[IX(s, i, j)] == NODE_OUT_) {
                s->next.u[IX(s, i, j)] = 0.0;
                s->next.v[IX(s, i, j)] = 0.0;
                s->next.t[IX(s, i, j)] = s->startT;
            }
    FN(copy_all)(s, &s->next, &s->cur);
    s->last_err = err;
    s->last_iters = it;
    return it;
}

/* Tolerance mode (no counterpart in the reference; restates adi2d_step_tol):
 * global iterations until r = max|next_k - next_(k-1)| / max|next_k| over NODE_IN
 * nodes and the three fields (next_0 = the state the step starts from) is <= tol,
 * at most max_global of them; the reference's guard (error above 1.0) returns -1.
 * Returns the iterations run; *res gets the last r. */
static int FN(time_step2_tol)(FN(solver2) *s, REAL dt, int max_global, int num_local, double tol, double *res)
{
    FN(copy_all)(s, &s->cur, &s->next);
    FN(copy_all)(s, &s->cur, &s->half);
    FN(copy_all)(s, &s->cur, &s->temp);
    double err = 0, r = NAN;
    size_t n = (size_t)s->nx * s->ny;
    int it = 0;
    REAL *prev = malloc(sizeof(REAL) * 3 * n);
    while (it < max_global) {
        for (size_t q = 0; q < n; q++) { prev[q] = s->next.u[q]; prev[n + q] = s->next.v[q]; prev[2 * n + q] = s->next.t[q]; }
        FN(solve_dir2)(s, dt, num_local, s->segy, s->nsegy, &s->cur, &s->temp, &s->half);
        FN(solve_dir2)(s, dt, num_local, s->segx, s->nsegx, &s->half, &s->temp, &s->next);
        err = FN(div_err2)(s, &s->next);
        REAL dm = 0, xm = 0;
        for (size_t q = 0; q < n; q++) {
            if (s->type[q] != NODE_IN_) continue;
            const REAL *xs[3] = {s->next.u, s->next.v, s->next.t}, *ts[3] = {prev, prev + n, prev + 2 * n};
            for (int v = 0; v < 3; v++) {
                REAL a = xs[v][q], d = (REAL)FN(absr)(a - ts[v][q]), ax = (REAL)FN(absr)(a);
                if (d > dm || d != d) dm = d;
                if (ax > xm || ax != ax) xm = ax;
            }
        }
        if (it == 0) FN(copy_type)(s, &s->next, &s->temp, NODE_IN_);
        else FN(merge_in)(s, &s->next, &s->temp);
        it++;
        r = xm > 0 ? (double)dm / (double)xm : (double)dm;
        if (err > 0.1 * 10) { s->last_err = err; *res = r; free(prev); return -1; }
        if (r <= tol) break;
    }
    free(prev);
    /* ClearOutterCells (Solver2D.cpp:68-80) */
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            if (s->type[IX(s, i, j)] == NODE_OUT_) {
                s->next.u[IX(s, i, j)] = 0.0;
                s->next.v[IX(s, i, j)] = 0.0;
                s->next.t[IX(s, i, j)] = s->startT;
            }
    FN(copy_all)(s, &s->next, &s->cur);
    s->last_err = err;
    s->last_iters = it;
    *res = r;
    return it;
}

#undef IX
#undef CAT_
#undef CAT
#undef FN
