/* Precision-generic body of the CPU restatement oracle.  Included twice by
 * adi_oracle.c, once with REAL=float (SFX=_f32) and once with REAL=double
 * (SFX=_f64).  TEST INFRASTRUCTURE ONLY: the product never links this.
 *
 * Every function restates the reference's CPU 3D ADI path operation by
 * operation, so that the float instantiation reproduces the reference's float
 * results bit for bit (same operand order, no fused multiply-add):
 *   bc rows            AdiSolver3D.cpp:804-852  (ApplyBC0 / ApplyBC1)
 *   matrix rows        AdiSolver3D.cpp:732-802  (BuildMatrix)
 *   Thomas             Common/Algorithms.h:21-39 (SolveTridiagonal)
 *   write-back         AdiSolver3D.cpp:707-730  (UpdateSegment)
 *   one direction      AdiSolver3D.cpp:564-666  (SolveDirection, CPU branch)
 *   one time step      AdiSolver3D.cpp:306-391  (TimeStep, CPU branch)
 *   boundaries         AdiSolver3D.cpp:286-304 + TimeLayer3D.h:926-951
 *   merge              TimeLayer3D.h:415-436,664-683
 *   stencils           TimeLayer3D.h:338-343,554-588
 *   divergence error   TimeLayer3D.h:595-641
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

typedef struct {
    REAL *f[4]; /* U, V, W, T; [i][j][k], k fastest */
} FN(layer);

typedef struct {
    int nx, ny, nz;
    REAL dx, dy, dz;
    const uint8_t *type, *bc_vel, *bc_temp;
    REAL *nv[4];                    /* node boundary values: v.x v.y v.z T */
    REAL v_T, v_vis, t_vis, t_phi;  /* FluidParams, already in REAL */
    FN(layer) L[4];                 /* storage for cur, next, half, temp */
    int cur, next, half, temp;      /* indices into L */
    seg_list segs[3];
    REAL *scratch;                  /* a b c d x, 5 * max(n) per thread */
    int nthreads;
    double diff_error;
} FN(solver);

static inline REAL *FN(el)(const FN(solver) *s, REAL *f, int i, int j, int k)
{
    return f + ((size_t)i * s->ny + j) * s->nz + k;
}
#define E(f, i, j, k) (*FN(el)(s, (f), (i), (j), (k)))

static REAL FN(d_x)(const FN(solver) *s, REAL *f, int i, int j, int k) { return (E(f, i + 1, j, k) - E(f, i - 1, j, k)) / (2 * s->dx); }
static REAL FN(d_y)(const FN(solver) *s, REAL *f, int i, int j, int k) { return (E(f, i, j + 1, k) - E(f, i, j - 1, k)) / (2 * s->dy); }
static REAL FN(d_z)(const FN(solver) *s, REAL *f, int i, int j, int k) { return (E(f, i, j, k + 1) - E(f, i, j, k - 1)) / (2 * s->dz); }

static REAL FN(diss_x)(const FN(solver) *s, FN(layer) *t, int i, int j, int k)
{
    REAL u_x = FN(d_x)(s, t->f[0], i, j, k);
    REAL v_x = FN(d_x)(s, t->f[1], i, j, k);
    REAL w_x = FN(d_x)(s, t->f[2], i, j, k);
    REAL u_y = FN(d_y)(s, t->f[0], i, j, k);
    REAL u_z = FN(d_z)(s, t->f[0], i, j, k);
    return 2 * u_x * u_x + v_x * v_x + w_x * w_x + v_x * u_y + w_x * u_z;
}
static REAL FN(diss_y)(const FN(solver) *s, FN(layer) *t, int i, int j, int k)
{
    REAL u_y = FN(d_y)(s, t->f[0], i, j, k);
    REAL v_y = FN(d_y)(s, t->f[1], i, j, k);
    REAL w_y = FN(d_y)(s, t->f[2], i, j, k);
    REAL v_x = FN(d_x)(s, t->f[1], i, j, k);
    REAL v_z = FN(d_z)(s, t->f[1], i, j, k);
    return u_y * u_y + 2 * v_y * v_y + w_y * w_y + u_y * v_x + w_y * v_z;
}
static REAL FN(diss_z)(const FN(solver) *s, FN(layer) *t, int i, int j, int k)
{
    REAL u_z = FN(d_z)(s, t->f[0], i, j, k);
    REAL v_z = FN(d_z)(s, t->f[1], i, j, k);
    REAL w_z = FN(d_z)(s, t->f[2], i, j, k);
    REAL w_x = FN(d_x)(s, t->f[2], i, j, k);
    REAL w_y = FN(d_y)(s, t->f[2], i, j, k);
    return u_z * u_z + v_z * v_z + 2 * w_z * w_z + u_z * w_x + v_z * w_y;
}

/* BC row at a segment end node (ApplyBC0 when first != 0, else ApplyBC1). */
static void FN(bc_row)(const FN(solver) *s, int i, int j, int k, int var, int first,
                       REAL *a_or_b, REAL *b_or_c, REAL *d)
{
    size_t id = ((size_t)i * s->ny + j) * s->nz + k;
    int is_free = var == 3 ? s->bc_temp[id] == BC_FREE_ : s->bc_vel[id] == BC_FREE_;
    if (is_free) {
        if (first) { *a_or_b = 2.0; *b_or_c = -1.0; }   /* b0, c0 */
        else       { *a_or_b = -1.0; *b_or_c = 2.0; }   /* a1, b1 */
        *d = 0.0;
    } else {
        if (first) { *a_or_b = 1.0; *b_or_c = 0.0; }
        else       { *a_or_b = 0.0; *b_or_c = 1.0; }
        *d = s->nv[var][id];
    }
}

static void FN(thomas)(REAL *a, REAL *b, REAL *c, REAL *d, REAL *x, int num)
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

static void FN(build_matrix)(const FN(solver) *s, REAL dt, const seg_t *g, int var, int dir,
                             REAL *a, REAL *b, REAL *c, REAL *d, FN(layer) *cur, FN(layer) *temp)
{
    REAL vis_dx2, vis_dy2, vis_dz2;
    REAL dx = s->dx, dy = s->dy, dz = s->dz;
    int n = g->size, i = g->pos[0], j = g->pos[1], k = g->pos[2];
    if (var != 3) {
        vis_dx2 = s->v_vis / (dx * dx);
        vis_dy2 = s->v_vis / (dy * dy);
        vis_dz2 = s->v_vis / (dz * dz);
    } else {
        vis_dx2 = s->t_vis / (dx * dx);
        vis_dy2 = s->t_vis / (dy * dy);
        vis_dz2 = s->t_vis / (dz * dz);
    }
    REAL *cf = cur->f[var];
    for (int p = 1; p < n - 1; p++) {
        if (dir == 0) {
            REAL w = E(temp->f[0], i + p, j, k);
            a[p] = -w / (2 * dx) - vis_dx2;
            b[p] = 3 / dt + 2 * vis_dx2;
            c[p] = w / (2 * dx) - vis_dx2;
            switch (var) {
            case 0: d[p] = E(cf, i + p, j, k) * 3 / dt - s->v_T * FN(d_x)(s, temp->f[3], i + p, j, k); break;
            case 3: d[p] = E(cf, i + p, j, k) * 3 / dt + s->t_phi * FN(diss_x)(s, temp, i + p, j, k); break;
            default: d[p] = E(cf, i + p, j, k) * 3 / dt; break;
            }
        } else if (dir == 1) {
            REAL w = E(temp->f[1], i, j + p, k);
            a[p] = -w / (2 * dy) - vis_dy2;
            b[p] = 3 / dt + 2 * vis_dy2;
            c[p] = w / (2 * dy) - vis_dy2;
            switch (var) {
            case 1: d[p] = E(cf, i, j + p, k) * 3 / dt - s->v_T * FN(d_y)(s, temp->f[3], i, j + p, k); break;
            case 3: d[p] = E(cf, i, j + p, k) * 3 / dt + s->t_phi * FN(diss_y)(s, temp, i, j + p, k); break;
            default: d[p] = E(cf, i, j + p, k) * 3 / dt; break;
            }
        } else {
            REAL w = E(temp->f[2], i, j, k + p);
            a[p] = -w / (2 * dz) - vis_dz2;
            b[p] = 3 / dt + 2 * vis_dz2;
            c[p] = w / (2 * dz) - vis_dz2;
            switch (var) {
            case 2: d[p] = E(cf, i, j, k + p) * 3 / dt - s->v_T * FN(d_z)(s, temp->f[3], i, j, k + p); break;
            case 3: d[p] = E(cf, i, j, k + p) * 3 / dt + s->t_phi * FN(diss_z)(s, temp, i, j, k + p); break;
            default: d[p] = E(cf, i, j, k + p) * 3 / dt; break;
            }
        }
    }
}

static void FN(solve_segment)(const FN(solver) *s, REAL dt, REAL *work, const seg_t *g, int var, int dir,
                              FN(layer) *cur, FN(layer) *temp, FN(layer) *next)
{
    int n = g->size, mx = s->nx > s->ny ? s->nx : s->ny;
    mx = mx > s->nz ? mx : s->nz;
    REAL *a = work, *b = a + mx, *c = b + mx, *d = c + mx, *x = d + mx;
    FN(bc_row)(s, g->pos[0], g->pos[1], g->pos[2], var, 1, &b[0], &c[0], &d[0]);
    FN(bc_row)(s, g->end[0], g->end[1], g->end[2], var, 0, &a[n - 1], &b[n - 1], &d[n - 1]);
    FN(build_matrix)(s, dt, g, var, dir, a, b, c, d, cur, temp);
    FN(thomas)(a, b, c, d, x, n);
    int i = g->pos[0], j = g->pos[1], k = g->pos[2];
    REAL *nf = next->f[var];
    for (int t = 0; t < n; t++) {
        E(nf, i, j, k) = x[t];
        if (dir == 0) i++; else if (dir == 1) j++; else k++;
    }
}

/* dest = (dest + src) / 2 where node type == IN, all four fields. */
static void FN(merge)(FN(solver) *s, FN(layer) *src, FN(layer) *dest)
{
    size_t n = (size_t)s->nx * s->ny * s->nz;
    for (int v = 0; v < 4; v++) {
        REAL *d = dest->f[v], *x = src->f[v];
        #pragma omp parallel for num_threads(s->nthreads) schedule(static)
        for (long long id = 0; id < (long long)n; id++)
            if (s->type[id] == NODE_IN_) d[id] = (d[id] + x[id]) / 2;
    }
}

/* One local iteration of SolveDirection without its merge: every segment of the
 * direction, four variables (AdiSolver3D.cpp:584-632). */
static void FN(solve_segments)(FN(solver) *s, int dir, REAL dt, FN(layer) *cur, FN(layer) *temp, FN(layer) *next)
{
    const seg_list *sl = &s->segs[dir];
    int mx = s->nx > s->ny ? s->nx : s->ny;
    mx = mx > s->nz ? mx : s->nz;
    #pragma omp parallel num_threads(s->nthreads)
    {
        REAL *work = s->scratch + (size_t)omp_get_thread_num() * 5 * mx;
        #pragma omp for schedule(static)
        for (int q = 0; q < sl->count; q++)
            for (int var = 0; var < 4; var++)
                FN(solve_segment)(s, dt, work, &sl->seg[q], var, dir, cur, temp, next);
    }
}

static void FN(solve_direction)(FN(solver) *s, int dir, REAL dt, int num_local,
                                FN(layer) *cur, FN(layer) *temp, FN(layer) *next)
{
    for (int it = 0; it < num_local; it++) {
        FN(solve_segments)(s, dir, dt, cur, temp, next);
        FN(merge)(s, next, temp);
    }
}

static void FN(copy_where)(FN(solver) *s, FN(layer) *src, FN(layer) *dest, int t1, int t2)
{
    size_t n = (size_t)s->nx * s->ny * s->nz;
    for (int v = 0; v < 4; v++)
        for (size_t id = 0; id < n; id++)
            if (s->type[id] == t1 || s->type[id] == t2) dest->f[v][id] = src->f[v][id];
}

/* Solver3D/AdiSolver3D::UpdateBoundaries (CPU): cur[BOUND|VALVE] = node values. */
static void FN(update_boundaries)(FN(solver) *s)
{
    size_t n = (size_t)s->nx * s->ny * s->nz;
    FN(layer) *cur = &s->L[s->cur];
    for (size_t id = 0; id < n; id++)
        if (s->type[id] == NODE_BOUND_ || s->type[id] == NODE_VALVE_)
            for (int v = 0; v < 4; v++) cur->f[v][id] = s->nv[v][id];
}

static double FN(div_error)(FN(solver) *s, FN(layer) *l)
{
    REAL *U = l->f[0], *V = l->f[1], *W = l->f[2];
    REAL dx = s->dx, dy = s->dy, dz = s->dz;
    double err = 0.0;
    int count = 0;
    for (int i = 0; i < s->nx - 1; i++)
        for (int j = 0; j < s->ny - 1; j++)
            for (int k = 0; k < s->nz - 1; k++)
                if (s->type[((size_t)i * s->ny + j) * s->nz + k] == NODE_IN_) {
                    double err_x = (E(U, i, j, k) + E(U, i, j - 1, k) + E(U, i, j - 1, k - 1) + E(U, i, j, k - 1) -
                                    E(U, i - 1, j, k) - E(U, i - 1, j - 1, k) - E(U, i - 1, j - 1, k - 1) - E(U, i - 1, j, k - 1)) * dz * dy / 4.0;
                    double err_y = (E(V, i, j, k) + E(V, i - 1, j, k) + E(V, i - 1, j, k - 1) + E(V, i, j, k - 1) -
                                    E(V, i, j - 1, k) - E(V, i - 1, j - 1, k) - E(V, i - 1, j - 1, k - 1) - E(V, i, j - 1, k - 1)) * dx * dz / 4.0;
                    double err_z = (E(W, i, j, k) + E(W, i, j - 1, k) + E(W, i - 1, j - 1, k) + E(W, i - 1, j, k) -
                                    E(W, i, j, k - 1) - E(W, i, j - 1, k - 1) - E(W, i - 1, j - 1, k - 1) - E(W, i - 1, j, k - 1)) * dx * dy / 4.0;
                    err += fabs(err_x + err_y + err_z);
                    count++;
                }
    return count ? err / count : 0.0;
}

/* UpdateBoundaries() (when update_bnd) followed by TimeStep(): with update_bnd
 * one pass of the reference driver loop (FluidSolver3D.cpp:241-242), without it
 * TimeStep alone.  Returns 0, or 1 if the divergence guard (> 0.01) fires, in
 * which case the layers are left unswapped exactly as the reference's throw
 * leaves them. */
static int FN(step)(FN(solver) *s, double dt_in, int num_global, int num_local, int compute_error, int update_bnd)
{
    REAL dt = (REAL)dt_in;
    if (update_bnd) FN(update_boundaries)(s);
    FN(layer) *cur = &s->L[s->cur], *next = &s->L[s->next], *half = &s->L[s->half], *temp = &s->L[s->temp];
    FN(copy_where)(s, cur, next, NODE_BOUND_, NODE_BOUND_);
    FN(copy_where)(s, cur, next, NODE_VALVE_, NODE_VALVE_);
    size_t n = (size_t)s->nx * s->ny * s->nz;
    for (int v = 0; v < 4; v++) memcpy(temp->f[v], cur->f[v], n * sizeof(REAL));
    for (int it = 0; it < num_global; it++) {
        FN(solve_direction)(s, 2, dt, num_local, cur, temp, next);
        FN(solve_direction)(s, 1, dt, num_local, next, temp, half);
        FN(solve_direction)(s, 0, dt, num_local, half, temp, next);
        FN(merge)(s, next, temp);
    }
    if (compute_error) s->diff_error = FN(div_error)(s, next);
    if (s->diff_error > 0.01) return 1;
    int t = s->next; s->next = s->cur; s->cur = t;
    return 0;
}

/* Tolerance-mode residual (the library's adi_step_tol; no reference counterpart):
 * max |x - t| and max |x| over NODE_IN cells and the four fields. */
static void FN(residual)(FN(solver) *s, FN(layer) *x, FN(layer) *t, double *dm, double *xm)
{
    size_t n = (size_t)s->nx * s->ny * s->nz;
    double a = 0.0, b = 0.0;
    for (int v = 0; v < 4; v++)
        for (size_t id = 0; id < n; id++)
            if (s->type[id] == NODE_IN_) {
                double xv = x->f[v][id], d = fabs(xv - (double)t->f[v][id]);
                if (d > a || d != d) a = d;
                if (fabs(xv) > b) b = fabs(xv);
            }
    *dm = a;
    *xm = b;
}

/* UpdateBoundaries + TimeStep in tolerance mode: global iterations until
 * max|x - t| / max|x| <= tol (t the nonlinear layer the last X sweep read, before
 * its merge), at most max_global of them. */
static int FN(step_tol)(FN(solver) *s, double dt_in, int max_global, int num_local, double tol, int compute_error,
                        int *iters, double *res)
{
    REAL dt = (REAL)dt_in;
    FN(update_boundaries)(s);
    FN(layer) *cur = &s->L[s->cur], *next = &s->L[s->next], *half = &s->L[s->half], *temp = &s->L[s->temp];
    FN(copy_where)(s, cur, next, NODE_BOUND_, NODE_BOUND_);
    FN(copy_where)(s, cur, next, NODE_VALVE_, NODE_VALVE_);
    size_t n = (size_t)s->nx * s->ny * s->nz;
    for (int v = 0; v < 4; v++) memcpy(temp->f[v], cur->f[v], n * sizeof(REAL));
    int it = 0;
    double r = NAN;
    while (it < max_global) {
        FN(solve_direction)(s, 2, dt, num_local, cur, temp, next);
        FN(solve_direction)(s, 1, dt, num_local, next, temp, half);
        FN(solve_direction)(s, 0, dt, num_local - 1, half, temp, next);
        FN(solve_segments)(s, 0, dt, half, temp, next);
        double dm, xm;
        FN(residual)(s, next, temp, &dm, &xm);
        FN(merge)(s, next, temp);
        FN(merge)(s, next, temp);
        it++;
        r = xm > 0 ? dm / xm : dm;
        if (r <= tol) break;
    }
    *iters = it;
    *res = r;
    if (compute_error) s->diff_error = FN(div_error)(s, next);
    if (s->diff_error > 0.01) return 1;
    int t = s->next; s->next = s->cur; s->cur = t;
    return 0;
}

#undef E
#undef FN
#undef CAT
#undef CAT_
