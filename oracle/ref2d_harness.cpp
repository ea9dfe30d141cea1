// Test-infrastructure harness around the reference's OWN 2D ADI solver.
//
// Part of the parity oracle, not of the product.  Compiled with the reference's
// unmodified sources (FluidSolver2D/AdiSolver2D.cpp, Solver2D.cpp, Grid2D.cpp and
// the Common objects, where they lie in the reference checkout) into
// oracle/_ref/libref2d.so by oracle/Makefile.  Only tests and the CPU-baseline leg
// of the benchmark load it.
//
// What it adds:
//   * HarnessGrid2D: a Grid2D whose node data (cell type, BC type, velocity, T)
//     come from plain arrays instead of the reference's shape loaders.
//   * HarnessSolver2D: an AdiSolver2D exposing its protected cur/next layers.
//   * operator new[] returning zeroed memory.  The reference allocates its layers
//     with new[] and its copy loops stop one row and one column short
//     (TimeLayer2D.h:98-176), so those cells are read uninitialised; zeroing makes
//     the runs reproducible and equal to the restatement, which starts them at 0.
//   * A C ABI (ref2d_*) driving the solver like its driver loop:
//     UpdateBoundaries() then TimeStep() (FluidSolver2D.cpp:131-132).
//
// The reference is compiled for FTYPE=float (src/Common/Geometry.h:21), as shipped.
// Its TimeStep calls exit(1) when the divergence error exceeds 1.0 or after 100
// global iterations (AdiSolver2D.cpp:303-313); inputs given to this harness must
// stay clear of both.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "FluidSolver2D/AdiSolver2D.h"

using namespace FluidSolver2D;
using namespace Common;

void *operator new[](std::size_t n)
{
    void *p = std::calloc(n ? n : 1, 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }

namespace {

struct HarnessGrid2D : public Grid2D {
    HarnessGrid2D(int nx, int ny, double dx_, double dy_, double startT_, const uint8_t *type, const uint8_t *bct,
                  const double *vx, const double *vy, const double *T)
        : Grid2D(dx_, dy_, startT_, true, 0.0)
    {
        dimx = nx;
        dimy = ny;
        frames = NULL;
        num_frames = 0;
        curData = new CondData2D[nx * ny];
        nextData = new CondData2D[nx * ny];
        for (int q = 0; q < nx * ny; q++) {
            curData[q] = CondData2D((BCtype)bct[q], (NodeType)type[q], Vec2D((FTYPE)vx[q], (FTYPE)vy[q]), (FTYPE)T[q]);
            nextData[q] = curData[q];
        }
    }
};

struct HarnessSolver2D : public AdiSolver2D {
    TimeLayer2D *layer(int which) { return which ? next : cur; }
    int nx() const { return dimx; }
    int ny() const { return dimy; }
};

struct Ref2D {
    HarnessGrid2D *grid;
    HarnessSolver2D *solver;
    FluidParams params;
};

} // namespace

extern "C" {

// The NetCDF loader the shared Common code links against; never reached here.
int nc_open(const char *, int, int *) { return -1; }
int nc_inq_dimid(int, const char *, int *) { return -1; }
int nc_inq_dimlen(int, int, size_t *) { return -1; }
int nc_inq_varid(int, const char *, int *) { return -1; }
int nc_get_var(int, int, void *) { return -1; }

void *ref2d_create(int nx, int ny, double dx, double dy, double startT, const uint8_t *type, const uint8_t *bct,
                   const double *vx, const double *vy, const double *T, double Re, double Pr, double lambda)
{
    Ref2D *h = new Ref2D;
    h->grid = new HarnessGrid2D(nx, ny, dx, dy, startT, type, bct, vx, vy, T);
    h->params = FluidParams(Re, Pr, lambda);
    h->solver = new HarnessSolver2D();
    h->solver->Init(h->grid, h->params);
    return h;
}

void ref2d_step(void *vh, double dt, int num_global, int num_local)
{
    Ref2D *h = (Ref2D *)vh;
    h->solver->UpdateBoundaries();
    h->solver->TimeStep((FTYPE)dt, num_global, num_local);
}

void ref2d_get_fields(void *vh, int which, double *u, double *v, double *T)
{
    Ref2D *h = (Ref2D *)vh;
    TimeLayer2D *l = h->solver->layer(which);
    int nx = h->solver->nx(), ny = h->solver->ny();
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            u[i * ny + j] = l->U(i, j);
            v[i * ny + j] = l->V(i, j);
            T[i * ny + j] = l->T(i, j);
        }
}

void ref2d_destroy(void *vh)
{
    Ref2D *h = (Ref2D *)vh;
    if (!h) return;
    delete h->solver;
    delete h->grid;
    delete h;
}

} // extern "C"
