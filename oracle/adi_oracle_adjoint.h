/* FP64 discrete adjoint of the fixed-iteration step (adi_step semantics): the
 * CPU restatement the library's adjoint kernels are checked against.  TEST
 * INFRASTRUCTURE ONLY; included once by adi_oracle.c after the double
 * instantiation of adi_oracle_body.h, whose functions it reuses.
 *
 * The reference has no adjoint.  Its forward step (AdiSolver3D.cpp:306-391, CPU
 * branch) is, per sweep: x = A(t)^-1 d(s, t, nv) on every segment of the
 * direction (BuildMatrix / ApplyBC0 / ApplyBC1 rows, AdiSolver3D.cpp:732-852),
 * dst = x on the segment nodes, temp = (temp + x) / 2 on NODE_IN (twice after the
 * last X sweep of a global iteration).  Differentiating it: with xbar the adjoint
 * of x, lambda = A^-T xbar per segment, and
 *   sbar  += 3/dt lambda                      (IN rows; d = 3/dt s + ...)
 *   nvbar += lambda                           (Dirichlet rows; d = node value)
 *   tbar[dir] += lambda (x[p-1] - x[p+1])/(2h)  (a, c depend on the advecting temp)
 *   tbar[T][p+-1] -/+= v_T lambda / (2h)      (pressure term of the velocity along dir)
 *   tbar += t_phi lambda d(DissFunc)/d(temp)  (temperature rows)
 * plus the merge (tbar_in = tbar_out/2 or /4 on IN, xbar += tbar_out/2 or 3/4),
 * the step start (temp = cur, next[BOUND|VALVE] = cur) and UpdateBoundaries
 * (cur[BOUND|VALVE] = node values). */

static size_t adj_n(const solver_f64 *s) { return (size_t)s->nx * s->ny * s->nz; }

#define AE(f, i, j, k) (*el_f64(s, (f), (i), (j), (k)))

static void adj_alloc(layer_f64 *l, size_t n)
{
    for (int v = 0; v < 4; v++) l->f[v] = calloc(n, sizeof(double));
}

static void adj_free(layer_f64 *l)
{
    for (int v = 0; v < 4; v++) free(l->f[v]);
}

static void adj_copy(layer_f64 *dst, const layer_f64 *src, size_t n)
{
    for (int v = 0; v < 4; v++) memcpy(dst->f[v], src->f[v], n * sizeof(double));
}

static void adj_zero(layer_f64 *l, size_t n)
{
    for (int v = 0; v < 4; v++) memset(l->f[v], 0, n * sizeof(double));
}

/* One adi_step (UpdateBoundaries + TimeStep, no divergence guard), recording the
 * nonlinear layer each sweep read (Ti[q]) and the layer it wrote (X[q]). */
static void adj_step_with_tape(solver_f64 *s, double dt_in, int ng, int nl, layer_f64 *Ti, layer_f64 *X)
{
    double dt = dt_in;
    size_t n = adj_n(s);
    update_boundaries_f64(s);
    layer_f64 *cur = &s->L[s->cur], *next = &s->L[s->next], *half = &s->L[s->half], *temp = &s->L[s->temp];
    copy_where_f64(s, cur, next, NODE_BOUND_, NODE_BOUND_);
    copy_where_f64(s, cur, next, NODE_VALVE_, NODE_VALVE_);
    adj_copy(temp, cur, n);
    int q = 0;
    for (int it = 0; it < ng; it++)
        for (int dd = 0; dd < 3; dd++) {
            int dir = 2 - dd;
            layer_f64 *src = dir == 2 ? cur : (dir == 1 ? next : half);
            layer_f64 *dst = dir == 1 ? half : next;
            for (int l = 0; l < nl; l++, q++) {
                adj_copy(&Ti[q], temp, n);
                solve_segments_f64(s, dir, dt, src, temp, dst);
                adj_copy(&X[q], dst, n);
                merge_f64(s, dst, temp);
                if (dir == 0 && l == nl - 1) merge_f64(s, dst, temp);
            }
        }
    int t = s->next; s->next = s->cur; s->cur = t;
}

/* Adds g * d(DissFunc_dir)/d(temp) at cell (i,j,k) to tb (the adjoint of temp). */
static void adj_diss(const solver_f64 *s, layer_f64 *t, layer_f64 *tb, int dir, int i, int j, int k, double g)
{
    double hx = 2 * s->dx, hy = 2 * s->dy, hz = 2 * s->dz;
    double *U = t->f[0], *V = t->f[1], *W = t->f[2];
#define DX(F) ((AE(F, i + 1, j, k) - AE(F, i - 1, j, k)) / hx)
#define DY(F) ((AE(F, i, j + 1, k) - AE(F, i, j - 1, k)) / hy)
#define DZ(F) ((AE(F, i, j, k + 1) - AE(F, i, j, k - 1)) / hz)
#define ADDX(F, c) do { AE(F, i + 1, j, k) += (c) / hx; AE(F, i - 1, j, k) -= (c) / hx; } while (0)
#define ADDY(F, c) do { AE(F, i, j + 1, k) += (c) / hy; AE(F, i, j - 1, k) -= (c) / hy; } while (0)
#define ADDZ(F, c) do { AE(F, i, j, k + 1) += (c) / hz; AE(F, i, j, k - 1) -= (c) / hz; } while (0)
    double *Ub = tb->f[0], *Vb = tb->f[1], *Wb = tb->f[2];
    if (dir == 0) {          /* 2 u_x^2 + v_x^2 + w_x^2 + v_x u_y + w_x u_z */
        double ux = DX(U), vx = DX(V), wx = DX(W), uy = DY(U), uz = DZ(U);
        ADDX(Ub, g * 4 * ux); ADDX(Vb, g * (2 * vx + uy)); ADDX(Wb, g * (2 * wx + uz));
        ADDY(Ub, g * vx); ADDZ(Ub, g * wx);
    } else if (dir == 1) {   /* u_y^2 + 2 v_y^2 + w_y^2 + u_y v_x + w_y v_z */
        double uy = DY(U), vy = DY(V), wy = DY(W), vx = DX(V), vz = DZ(V);
        ADDY(Ub, g * (2 * uy + vx)); ADDY(Vb, g * 4 * vy); ADDY(Wb, g * (2 * wy + vz));
        ADDX(Vb, g * uy); ADDZ(Vb, g * wy);
    } else {                 /* u_z^2 + v_z^2 + 2 w_z^2 + u_z w_x + v_z w_y */
        double uz = DZ(U), vz = DZ(V), wz = DZ(W), wx = DX(W), wy = DY(W);
        ADDZ(Ub, g * (2 * uz + wx)); ADDZ(Vb, g * (2 * vz + wy)); ADDZ(Wb, g * 4 * wz);
        ADDX(Wb, g * uz); ADDY(Wb, g * vz);
    }
#undef DX
#undef DY
#undef DZ
#undef ADDX
#undef ADDY
#undef ADDZ
}

/* Adjoint of one sweep (direction dir, merges m) with its tape (Ti, X): consumes
 * dbar on the segment nodes, turns tbar from the adjoint of the temp it wrote
 * into the adjoint of the temp it read, and accumulates sbar and nvbar.  xb is a
 * full-size work layer. */
static void adj_sweep(solver_f64 *s, double dt, int dir, int m, layer_f64 *Ti, layer_f64 *X, layer_f64 *sbar,
                      layer_f64 *dbar, layer_f64 *tbar, layer_f64 *nvbar, layer_f64 *xb)
{
    const seg_list *sl = &s->segs[dir];
    size_t n = adj_n(s);
    const double mx_ = m == 2 ? 0.75 : 0.5, mt_ = m == 2 ? 0.25 : 0.5;
    double h = dir == 0 ? s->dx : (dir == 1 ? s->dy : s->dz);
    int mx = s->nx > s->ny ? s->nx : s->ny;
    mx = mx > s->nz ? mx : s->nz;
    double *a = malloc(sizeof(double) * mx), *b = malloc(sizeof(double) * mx), *c = malloc(sizeof(double) * mx);
    double *d = malloc(sizeof(double) * mx), *lam = malloc(sizeof(double) * mx), *cp = malloc(sizeof(double) * mx);
    double *xs = malloc(sizeof(double) * mx), *xbs = malloc(sizeof(double) * mx);
    /* 1. xbar of every written value, before any adjoint changes */
    adj_zero(xb, n);
    for (int q = 0; q < sl->count; q++) {
        const seg_t *g = &sl->seg[q];
        int i = g->pos[0], j = g->pos[1], k = g->pos[2];
        for (int p = 0; p < g->size; p++) {
            size_t id = ((size_t)i * s->ny + j) * s->nz + k;
            for (int v = 0; v < 4; v++) {
                double x = dbar->f[v][id];
                if (s->type[id] == NODE_IN_) x += mx_ * tbar->f[v][id];
                xb->f[v][id] = x;
            }
            if (dir == 0) i++; else if (dir == 1) j++; else k++;
        }
    }
    /* 2. the merge: temp_out = temp_in * mt_ + x * mx_ on IN, temp_in elsewhere */
    for (int v = 0; v < 4; v++)
        for (size_t id = 0; id < n; id++)
            if (s->type[id] == NODE_IN_) tbar->f[v][id] *= mt_;
    /* 3. dst values on the segment nodes were overwritten */
    for (int q = 0; q < sl->count; q++) {
        const seg_t *g = &sl->seg[q];
        int i = g->pos[0], j = g->pos[1], k = g->pos[2];
        for (int p = 0; p < g->size; p++) {
            size_t id = ((size_t)i * s->ny + j) * s->nz + k;
            for (int v = 0; v < 4; v++) dbar->f[v][id] = 0.0;
            if (dir == 0) i++; else if (dir == 1) j++; else k++;
        }
    }
    /* 4. lambda = A^-T xbar per segment and variable; a node shared by two
     *    segments gives its xbar to the first of them (either way the sum of the
     *    two Dirichlet rows' lambdas is the same) */
    for (int q = 0; q < sl->count; q++) {
        const seg_t *g = &sl->seg[q];
        int nn = g->size;
        for (int var = 0; var < 4; var++) {
            bc_row_f64(s, g->pos[0], g->pos[1], g->pos[2], var, 1, &b[0], &c[0], &d[0]);
            bc_row_f64(s, g->end[0], g->end[1], g->end[2], var, 0, &a[nn - 1], &b[nn - 1], &d[nn - 1]);
            build_matrix_f64(s, dt, g, var, dir, a, b, c, d, Ti, Ti);
            a[0] = 0.0;
            c[nn - 1] = 0.0;
            int i = g->pos[0], j = g->pos[1], k = g->pos[2];
            for (int p = 0; p < nn; p++) {
                size_t id = ((size_t)i * s->ny + j) * s->nz + k;
                xs[p] = X->f[var][id];
                xbs[p] = xb->f[var][id];
                xb->f[var][id] = 0.0;
                if (dir == 0) i++; else if (dir == 1) j++; else k++;
            }
            /* transposed Thomas: sub c[p-1], diagonal b[p], super a[p+1] */
            cp[0] = (nn > 1 ? a[1] : 0.0) / b[0];
            lam[0] = xbs[0] / b[0];
            for (int p = 1; p < nn; p++) {
                double sub = c[p - 1], sup = p + 1 < nn ? a[p + 1] : 0.0;
                double den = b[p] - sub * cp[p - 1];
                cp[p] = sup / den;
                lam[p] = (xbs[p] - sub * lam[p - 1]) / den;
            }
            for (int p = nn - 2; p >= 0; p--) lam[p] -= cp[p] * lam[p + 1];
            /* accumulate */
            i = g->pos[0]; j = g->pos[1]; k = g->pos[2];
            for (int p = 0; p < nn; p++) {
                size_t id = ((size_t)i * s->ny + j) * s->nz + k;
                if (p == 0 || p == nn - 1) {
                    int is_free = var == 3 ? s->bc_temp[id] == BC_FREE_ : s->bc_vel[id] == BC_FREE_;
                    if (!is_free) nvbar->f[var][id] += lam[p];
                } else {
                    sbar->f[var][id] += 3.0 / dt * lam[p];
                    tbar->f[dir][id] += lam[p] * (xs[p - 1] - xs[p + 1]) / (2 * h);
                    size_t step = dir == 0 ? (size_t)s->ny * s->nz : (dir == 1 ? (size_t)s->nz : 1);
                    if (var == dir) {
                        tbar->f[3][id + step] -= s->v_T * lam[p] / (2 * h);
                        tbar->f[3][id - step] += s->v_T * lam[p] / (2 * h);
                    }
                    if (var == 3) adj_diss(s, Ti, tbar, dir, i, j, k, s->t_phi * lam[p]);
                }
                if (dir == 0) i++; else if (dir == 1) j++; else k++;
            }
        }
    }
    free(a); free(b); free(c); free(d); free(lam); free(cp); free(xs); free(xbs);
}

/* Adjoint of one adi_step with its tape: cbar holds the adjoint of the step's
 * result on entry and of its input state on return; nvbar accumulates. */
static void adj_step(solver_f64 *s, double dt, int ng, int nl, layer_f64 *Ti, layer_f64 *X, layer_f64 *cbar,
                     layer_f64 *nvbar, layer_f64 *nbar, layer_f64 *hbar, layer_f64 *tbar, layer_f64 *xb)
{
    size_t n = adj_n(s);
    adj_copy(nbar, cbar, n);
    adj_zero(cbar, n);
    adj_zero(hbar, n);
    adj_zero(tbar, n);
    int q = ng * nl * 3 - 1;
    for (int it = ng - 1; it >= 0; it--)
        for (int dir = 0; dir < 3; dir++) {
            layer_f64 *sb = dir == 2 ? cbar : (dir == 1 ? nbar : hbar);
            layer_f64 *db = dir == 1 ? hbar : nbar;
            for (int l = nl - 1; l >= 0; l--, q--)
                adj_sweep(s, dt, dir, (dir == 0 && l == nl - 1) ? 2 : 1, &Ti[q], &X[q], sb, db, tbar, nvbar, xb);
        }
    for (int v = 0; v < 4; v++)
        for (size_t id = 0; id < n; id++) {
            cbar->f[v][id] += tbar->f[v][id];
            if (s->type[id] == NODE_BOUND_ || s->type[id] == NODE_VALVE_) {
                cbar->f[v][id] += nbar->f[v][id];
                nvbar->f[v][id] += cbar->f[v][id];
                cbar->f[v][id] = 0.0;
            }
        }
}

#undef AE
