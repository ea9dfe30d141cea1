// Test-infrastructure harness: the reference's driver loop run through the
// B200AdiSolver3D adapter (cmc-fluid-solver_b200/host/B200AdiSolver3D.cpp).
//
// This file is part of the parity checking, not of the product.  oracle/Makefile
// compiles it with the adapter against the reference's own headers (Solver3D.h,
// Grid3D.h, Geometry.h: FTYPE float as shipped) into oracle/_ref/libadapter3d.so,
// linked to the reference's Grid3D code (oracle/_ref/libref3d.so) and to
// libadi_b200.so.  That the adapter compiles there is the check that its
// overrides match Solver3D (FluidSolver3D/Solver3D.h:24-49); the GPU tests run
// adapter_run and compare its GetLayer output with the reference solver's.
//
// adapter_run follows FluidSolver3D.cpp:224-262 on a synthetic grid: construct
// the solver, Init, CreateSegments, then per step UpdateBoundaries() and
// TimeStep(dt, num_global, num_local, i % 10 == 0 || last step), and GetLayer
// after the last step.

#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "FluidSolver3D/Grid3D.h"
#include "B200AdiSolver3D.h"

using namespace FluidSolver3D;
using namespace Common;

namespace
{
	// A Grid3D whose node array comes from plain arrays instead of the reference's
	// loaders (Grid3D.cpp:373-513).
	struct AdapterGrid : public Grid3D
	{
		AdapterGrid(int nx, int ny, int nz, double _dx, double _dy, double _dz)
			: Grid3D(_dx, _dy, _dz, 1.0, CPU, false, EVEN_X)
		{
			dimx = nx; dimy = ny; dimz = nz;
			nodes = new Node[(size_t)nx * ny * nz];
		}
		Node *Nodes() { return nodes; }
	};
}

extern "C" {

// Returns 0; 1 when the adapter threw (message in err); 2 on a bad argument.
// vout: 3 floats per output point, Tout: one double per output point.
int adapter_run(int nx, int ny, int nz, double dx, double dy, double dz, const unsigned char *type,
                const unsigned char *bc_vel, const unsigned char *bc_temp, const float *vx, const float *vy,
                const float *vz, const float *T, double Re, double Pr, double lambda, double dt, int num_global,
                int num_local, int steps, int solver_kind, int outdimx, int outdimy, int outdimz, float *vout,
                double *Tout, char *err, int errlen)
{
	if (nx < 3 || ny < 3 || nz < 3 || steps < 1 || !vout || !Tout) return 2;
	try
	{
		AdapterGrid g(nx, ny, nz, dx, dy, dz);
		Node *nodes = g.Nodes();
		const size_t n = (size_t)nx * ny * nz;
		for (size_t i = 0; i < n; i++)
		{
			nodes[i].type = (NodeType)type[i];
			nodes[i].bc_vel = (BCtype)bc_vel[i];
			nodes[i].bc_temp = (BCtype)bc_temp[i];
			nodes[i].v = Vec3D(vx[i], vy[i], vz[i]);
			nodes[i].T = T[i];
		}
		FluidParams params(Re, Pr, lambda);
		B200AdiSolver3D solver(solver_kind);
		Solver3D *base = &solver;   // the driver holds the solver as Solver3D*
		base->Init(GPU, false, &g, params, false, 1);
		solver.CreateSegments();
		for (int i = 0; i < steps; i++)
		{
			base->UpdateBoundaries();
			base->TimeStep((FTYPE)dt, num_global, num_local, (i % 10 == 0) || (i + 1 == steps));
		}
		const size_t m = (size_t)(outdimx ? outdimx : nx) * (outdimy ? outdimy : ny) * (outdimz ? outdimz : nz);
		std::vector<Vec3D> v(m);
		solver.GetLayerB200(v.data(), Tout, outdimx, outdimy, outdimz);
		for (size_t i = 0; i < m; i++)
		{
			vout[3 * i] = v[i].x;
			vout[3 * i + 1] = v[i].y;
			vout[3 * i + 2] = v[i].z;
		}
		return 0;
	}
	catch (std::exception &e)
	{
		if (err && errlen > 0)
		{
			strncpy(err, e.what(), (size_t)errlen - 1);
			err[errlen - 1] = 0;
		}
		return 1;
	}
}

}
