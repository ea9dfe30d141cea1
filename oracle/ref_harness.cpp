// Test-infrastructure harness around the reference's OWN CPU solver.
//
// This file is part of the parity oracle, not of the product.  It is compiled
// together with the reference's unmodified sources (AdiSolver3D.cpp, Grid3D.cpp,
// Solver3D.cpp, Grid2D.cpp, GPUplan.cpp, PARAplan.cpp, LinuxIO.cpp, taken from
// where they lie in the reference checkout) into oracle/_ref/libref3d.so by
// oracle/Makefile.  Only tests, the smoke check and the CPU-baseline leg of the
// benchmark load it.
//
// What it adds on top of the reference:
//   * HarnessGrid: a Grid3D whose node array is filled from plain SoA arrays
//     (type, bc_vel, bc_temp, v.xyz, T) instead of the reference's rasterising
//     loaders (Grid3D.cpp:373-513), so synthetic masks can be injected.
//   * HarnessSolver: an AdiSolver3D that exposes the protected cur/next layers.
//   * A C ABI (ref_*) so Python (ctypes) can drive the reference exactly like its
//     driver loop does: UpdateBoundaries() then TimeStep()
//     (FluidSolver3D/FluidSolver3D.cpp:241-242).
//   * No-op stand-ins for the GPU launchers and the four NetCDF calls the
//     reference links against; the CPU backend never reaches them.
//
// The reference is compiled for FTYPE=float (src/Common/Geometry.h:21), as shipped.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <vector>

#include "FluidSolver3D/AdiSolver3D.h"

using namespace FluidSolver3D;
using namespace Common;

// ----------------------------------------------------------------------------
// Stand-ins for symbols only the GPU backend uses (TimeLayer3D.h:29-34,
// AdiSolver3D.h:40-46) and for the NetCDF loader (Grid3D.cpp:437-486).
// ----------------------------------------------------------------------------
static void ref_gpu_unreachable(const char *what)
{
	fprintf(stderr, "ref_harness: GPU-backend entry %s reached on the CPU backend\n", what);
	abort();
}

void CopyFieldTo_GPU(int, int, int, FTYPE **, FTYPE **, NodeType **, NodeType, int) { ref_gpu_unreachable("CopyFieldTo_GPU"); }
void MergeFieldTo_GPU(int, int, int, FTYPE **, FTYPE **, NodeType **, NodeType, int) { ref_gpu_unreachable("MergeFieldTo_GPU"); }
void CopyGridBoundary_GPU(DirType, int, int, int, FTYPE **, FTYPE **, FTYPE **, FTYPE **, int *, Segment3D **, NodesBoundary3D **, int) { ref_gpu_unreachable("CopyGridBoundary_GPU"); }
void Clear_GPU(int, int, int, FTYPE **, FTYPE **, FTYPE **, FTYPE **, NodeType **, NodeType, FTYPE, FTYPE, FTYPE, FTYPE, int) { ref_gpu_unreachable("Clear_GPU"); }
void Transpose_GPU(int, int, int, FTYPE **, FTYPE **, int) { ref_gpu_unreachable("Transpose_GPU"); }

namespace FluidSolver3D
{
	void SolveSegments_GPU(FTYPE, FluidParams, int *, Segment3D **, DirType, NodesBoundary3D **, NodeType **,
	                       TimeLayer3D *, TimeLayer3D *, TimeLayer3D *, FTYPE **, FTYPE **, int, FTYPE *)
	{
		ref_gpu_unreachable("SolveSegments_GPU");
	}
	void SolveSegments_XY_GPU(FTYPE, FluidParams, int **, int **, int **, int **, Segment3D **, Segment3D **,
	                          int, int, NodesBoundary3D **, NodesBoundary3D **, NodeType **,
	                          TimeLayer3D *, TimeLayer3D *, TimeLayer3D *, TimeLayer3D *,
	                          FTYPE **, FTYPE **, FTYPE **, FTYPE **)
	{
		ref_gpu_unreachable("SolveSegments_XY_GPU");
	}
}

extern "C" {
int nc_open(const char *, int, int *) { return -1; }
int nc_inq_dimid(int, const char *, int *) { return -1; }
int nc_inq_dimlen(int, int, size_t *) { return -1; }
int nc_inq_varid(int, const char *, int *) { return -1; }
int nc_get_var(int, int, void *) { return -1; }
}

// ----------------------------------------------------------------------------
// Grid and solver with the hooks the harness needs.
// ----------------------------------------------------------------------------
struct HarnessGrid : public Grid3D
{
	HarnessGrid(int nx, int ny, int nz, double _dx, double _dy, double _dz)
		: Grid3D(_dx, _dy, _dz, 1.0, CPU, false, EVEN_X)
	{
		dimx = nx; dimy = ny; dimz = nz;
		nodes = new Node[(size_t)nx * ny * nz];
	}
	Node *Nodes() { return nodes; }
};

// A Grid3D built by the reference's own loaders and mask builders (Shape3D,
// SeaNetCDF, Shape2D), with read access to what they produced.
struct MaskGrid : public Grid3D
{
	// 3D shapes (Grid3D.h:106) or a 2D shape extruded in depth (Grid3D.h:105)
	MaskGrid(double _dx, double _dy, double _dz, double _baseT, bool netcdf)
		: Grid3D(_dx, _dy, _dz, _baseT, CPU, netcdf, EVEN_X) { }
	MaskGrid(double _dx, double _dy, double _dz, double _depth, double _depth_var, double _baseT)
		: Grid3D(_dx, _dy, _dz, _depth, _depth_var, _baseT, CPU, false, EVEN_X) { }
	Node *Nodes() { return nodes; }
	int NumFrames() { return num_frames; }
	FrameInfo3D *Frames() { return frames; }
	int ActiveDimz() { return active_dimz; }
	BBox3D &Box() { return bbox; }
	// the state LoadNetCDF leaves (Grid3D.cpp:437-486), from a depth map in memory
	void SetSea(int nx, int ny, int nz, const float *depth, int dnx, int dny, float zmin)
	{
		dimx = nx; dimy = ny; dimz = nz;
		nodes = new Node[(size_t)nx * ny * nz];
		depthInfo = new DepthInfo3D(dnx, dny);
		memcpy(depthInfo->depth, depth, sizeof(float) * (size_t)dnx * dny);
		bbox.pMin.z = zmin;
		num_frames = 1;
	}
};

struct HarnessSolver : public AdiSolver3D
{
	TimeLayer3D *Cur() { return cur; }
	TimeLayer3D *Next() { return next; }
};

struct RefHandle
{
	HarnessGrid *grid;
	HarnessSolver *solver;
	FluidParams params;
	int steps_done;
};

static int seg_capacity(HarnessGrid *g, int dir)
{
	int d1 = dir == X ? g->dimx : (dir == Y ? g->dimy : g->dimz);
	int d2 = dir == X ? g->dimy : g->dimx;
	int d3 = dir == Z ? g->dimy : g->dimz;
	return d2 * d3 * (d1 / 2 + 1);
}

static int reference_list_capacity(HarnessGrid *g, int dir)
{
	// AdiSolver3D::Init / CreateListSegments allocate lines * MAX_SEGS_PER_ROW
	// (AdiSolver3D.cpp:189-191,407-419).
	int lines = dir == X ? g->dimy * g->dimz : (dir == Y ? g->dimx * g->dimz : g->dimx * g->dimy);
	return lines * MAX_SEGS_PER_ROW;
}

static int generate(HarnessGrid *g, int dir, std::vector<Segment3D> &buf)
{
	buf.resize(seg_capacity(g, dir));
	int num = 0;
	switch (dir)
	{
	// argument order as in AdiSolver3D::CreateSegments (AdiSolver3D.cpp:557-559)
	case X: g->GenerateListSegments(num, buf.data(), g->dimx, g->dimy, g->dimz, X, 1); break;
	case Y: g->GenerateListSegments(num, buf.data(), g->dimy, g->dimx, g->dimz, Y, 1); break;
	default: g->GenerateListSegments(num, buf.data(), g->dimz, g->dimx, g->dimy, Z, 1); break;
	}
	return num;
}

extern "C" {

int ref_ftype_size() { return (int)sizeof(FTYPE); }

void *ref_create(int nx, int ny, int nz, double dx, double dy, double dz,
                 const unsigned char *type, const unsigned char *bc_vel, const unsigned char *bc_temp,
                 const float *vx, const float *vy, const float *vz, const float *T)
{
	try
	{
		PARAplan *pplan = PARAplan::Instance();
		pplan->init(CPU);
		pplan->splitEven1D(nx);
		RefHandle *h = new RefHandle();
		h->grid = new HarnessGrid(nx, ny, nz, dx, dy, dz);
		h->solver = NULL;
		h->steps_done = 0;
		Node *nodes = h->grid->Nodes();
		size_t n = (size_t)nx * ny * nz;
		for (size_t i = 0; i < n; i++)
		{
			nodes[i].type = (NodeType)type[i];
			nodes[i].bc_vel = (BCtype)bc_vel[i];
			nodes[i].bc_temp = (BCtype)bc_temp[i];
			nodes[i].v = Vec3D(vx[i], vy[i], vz[i]);
			nodes[i].T = T[i];
		}
		return h;
	}
	catch (std::exception &)
	{
		return NULL;
	}
}

// Segments exactly as Grid3D::GenerateListSegments (Grid3D.cpp:47-127) lists them,
// 7 ints each: posx posy posz endx endy endz size.  Returns the count, or -1 if
// out7 is too small.
int ref_segments(void *vh, int dir, int *out7, int cap)
{
	RefHandle *h = (RefHandle *)vh;
	std::vector<Segment3D> buf;
	int num = generate(h->grid, dir, buf);
	if (out7 == NULL) return num;
	if (num > cap) return -1;
	for (int s = 0; s < num; s++)
	{
		const Segment3D &g = buf[s];
		int *o = out7 + 7 * s;
		o[0] = g.posx; o[1] = g.posy; o[2] = g.posz;
		o[3] = g.endx; o[4] = g.endy; o[5] = g.endz;
		o[6] = g.size;
	}
	return num;
}

// params_mode 0: FluidParams(Re, Pr, lambda)           (Geometry.h:545-552)
// params_mode 1: FluidParams(vis, rho, R, k, cv)       (Geometry.h:554-561)
// Returns 0, or -3 when a direction has more segments than the reference's
// fixed lists hold (it would overrun them).
int ref_solver_init(void *vh, int params_mode, double p0, double p1, double p2, double p3, double p4)
{
	RefHandle *h = (RefHandle *)vh;
	try
	{
		for (int dir = 0; dir < 3; dir++)
		{
			std::vector<Segment3D> buf;
			if (generate(h->grid, dir, buf) > reference_list_capacity(h->grid, dir)) return -3;
		}
		if (params_mode == 0) h->params = FluidParams(p0, p1, p2);
		else h->params = FluidParams(p0, p1, p2, p3, p4);
		PARAplan::Instance()->splitEven1D(h->grid->dimx);
		h->solver = new HarnessSolver();
		h->solver->Init(CPU, false, h->grid, h->params, false, 1);
		h->solver->CreateSegments();
		return 0;
	}
	catch (std::exception &)
	{
		return -2;
	}
}

int ref_fluid_params(void *vh, float *out4)
{
	RefHandle *h = (RefHandle *)vh;
	out4[0] = h->params.v_T; out4[1] = h->params.v_vis; out4[2] = h->params.t_vis; out4[3] = h->params.t_phi;
	return 0;
}

// One pass of the reference driver loop body: UpdateBoundaries(); TimeStep().
// Returns 0, or 1 when TimeStep threw on the divergence guard (AdiSolver3D.cpp:371-374).
int ref_step(void *vh, double dt, int num_global, int num_local, int compute_error)
{
	RefHandle *h = (RefHandle *)vh;
	if (h->solver == NULL) return -2;
	try
	{
		h->solver->UpdateBoundaries();
		h->solver->TimeStep((FTYPE)dt, num_global, num_local, compute_error != 0);
		h->steps_done++;
		return 0;
	}
	catch (std::exception &)
	{
		return 1;
	}
}

// AdiSolver3D::TimeStep alone, without UpdateBoundaries.
int ref_time_step(void *vh, double dt, int num_global, int num_local, int compute_error)
{
	RefHandle *h = (RefHandle *)vh;
	if (h->solver == NULL) return -2;
	try
	{
		h->solver->TimeStep((FTYPE)dt, num_global, num_local, compute_error != 0);
		h->steps_done++;
		return 0;
	}
	catch (std::exception &)
	{
		return 1;
	}
}

// which = 0: cur (latest state after the step's swap), 1: next.
int ref_get_fields(void *vh, int which, float *u, float *v, float *w, float *T)
{
	RefHandle *h = (RefHandle *)vh;
	if (h->solver == NULL) return -2;
	TimeLayer3D *l = which == 0 ? h->solver->Cur() : h->solver->Next();
	int nx = h->grid->dimx, ny = h->grid->dimy, nz = h->grid->dimz;
	for (int i = 0; i < nx; i++)
		for (int j = 0; j < ny; j++)
			for (int k = 0; k < nz; k++)
			{
				size_t id = ((size_t)i * ny + j) * nz + k;
				u[id] = l->U->elem(i, j, k);
				v[id] = l->V->elem(i, j, k);
				w[id] = l->W->elem(i, j, k);
				T[id] = l->T->elem(i, j, k);
			}
	return 0;
}

int ref_set_state(void *vh, const float *u, const float *v, const float *w, const float *T)
{
	RefHandle *h = (RefHandle *)vh;
	if (h->solver == NULL) return -2;
	TimeLayer3D *l = h->solver->Cur();
	int nx = h->grid->dimx, ny = h->grid->dimy, nz = h->grid->dimz;
	for (int i = 0; i < nx; i++)
		for (int j = 0; j < ny; j++)
			for (int k = 0; k < nz; k++)
			{
				size_t id = ((size_t)i * ny + j) * nz + k;
				l->U->elem(i, j, k) = u[id];
				l->V->elem(i, j, k) = v[id];
				l->W->elem(i, j, k) = w[id];
				l->T->elem(i, j, k) = T[id];
			}
	return 0;
}

// Mean absolute finite-volume divergence of cur (TimeLayer3D::EvalDivError,
// TimeLayer3D.h:595-641).
// Solver3D::GetLayer (Solver3D.cpp:21-25) of the reference solver: v gets 3 floats
// per output point, T one double.
int ref_get_layer(void *vh, int outdimx, int outdimy, int outdimz, float *v, double *T)
{
	RefHandle *h = (RefHandle *)vh;
	if (h->solver == NULL) return -2;
	const size_t m = (size_t)(outdimx ? outdimx : h->grid->dimx) * (outdimy ? outdimy : h->grid->dimy) *
	                 (outdimz ? outdimz : h->grid->dimz);
	std::vector<Vec3D> vel(m);
	h->solver->GetLayer(vel.data(), T, outdimx, outdimy, outdimz);
	for (size_t i = 0; i < m; i++)
	{
		v[3 * i] = vel[i].x;
		v[3 * i + 1] = vel[i].y;
		v[3 * i + 2] = vel[i].z;
	}
	return 0;
}

double ref_div_error(void *vh)
{
	RefHandle *h = (RefHandle *)vh;
	return h->solver->Cur()->EvalDivError(h->grid);
}

void ref_destroy(void *vh)
{
	RefHandle *h = (RefHandle *)vh;
	if (h == NULL) return;
	delete h->solver;   // prints the reference Profiler table (AdiSolver3D.cpp:155)
	delete h->grid;
	delete h;
}

// ---- mask builders ----------------------------------------------------------

// Grid3D(dx, dy, dz, baseT) + LoadFromFile (Load3DShape, Grid3D.cpp:371-435) of a
// Shape3D text file; dims_out receives dimx, dimy, dimz.
void *ref_shape3d_load(const char *path, double dx, double dy, double dz, double baseT, int *dims_out)
{
	PARAplan::Instance()->init(CPU);
	MaskGrid *g = new MaskGrid(dx, dy, dz, baseT, false);
	if (!g->LoadFromFile(const_cast<char *>(path), false)) { delete g; return NULL; }
	dims_out[0] = g->dimx; dims_out[1] = g->dimy; dims_out[2] = g->dimz;
	return g;
}

// Grid3D(dx, dy, dz, depth, depth_var, baseT) + LoadFromFile of a Shape2D file
// (Grid3D.cpp:497-509); dims_out: dimx, dimy, dimz, active_dimz.
void *ref_shape2d_load(const char *path, double dx, double dy, double dz, double depth, double depth_var,
                       double baseT, int *dims_out)
{
	PARAplan::Instance()->init(CPU);
	MaskGrid *g = new MaskGrid(dx, dy, dz, depth, depth_var, baseT);
	if (!g->LoadFromFile(const_cast<char *>(path), false)) { delete g; return NULL; }
	dims_out[0] = g->dimx; dims_out[1] = g->dimy; dims_out[2] = g->dimz; dims_out[3] = g->ActiveDimz();
	return g;
}

// The state LoadNetCDF leaves, from a depth map in memory, and the inflow of
// SetBoundParams (Grid3D.cpp:316-320).
void *ref_sea_create(int nx, int ny, int nz, const float *depth, int dnx, int dny, float zmin, double baseT,
                     const float *in_vel, double in_T)
{
	PARAplan::Instance()->init(CPU);
	MaskGrid *g = new MaskGrid(1.0, 1.0, 1.0, baseT, true);
	g->SetSea(nx, ny, nz, depth, dnx, dny, zmin);
	g->SetBoundParams(Vec3D(in_vel[0], in_vel[1], in_vel[2]), in_T);
	return g;
}

// Grid3D::Prepare(time) on the CPU backend.
int ref_mask_prepare(void *vg, double time)
{
	try { ((MaskGrid *)vg)->Prepare(time); }
	catch (std::exception &) { return -1; }
	return 0;
}

// The node array as SoA.
void ref_mask_nodes(void *vg, unsigned char *type, unsigned char *bc_vel, unsigned char *bc_temp, float *vx,
                    float *vy, float *vz, float *T)
{
	MaskGrid *g = (MaskGrid *)vg;
	const Node *nd = g->Nodes();
	size_t n = (size_t)g->dimx * g->dimy * g->dimz;
	for (size_t i = 0; i < n; i++)
	{
		type[i] = (unsigned char)nd[i].type;
		bc_vel[i] = (unsigned char)nd[i].bc_vel;
		bc_temp[i] = (unsigned char)nd[i].bc_temp;
		vx[i] = nd[i].v.x; vy[i] = nd[i].v.y; vz[i] = nd[i].v.z; T[i] = nd[i].T;
	}
}

// Vertices (grid coordinates, 3 floats each) and triangles of shape 0 of frame f
// as Load3DShape left them; returns the vertex count, *ntris the triangle count.
int ref_shape3d_frame(void *vg, int f, float *verts, int *tris, int *ntris)
{
	MaskGrid *g = (MaskGrid *)vg;
	if (f < 0 || f >= g->NumFrames()) return -1;
	Shape3D &sh = g->Frames()[f].Shapes[0];
	if (verts)
		for (int k = 0; k < sh.NumVertices; k++)
		{
			verts[3 * k] = sh.Vertices[k].x; verts[3 * k + 1] = sh.Vertices[k].y; verts[3 * k + 2] = sh.Vertices[k].z;
		}
	if (tris)
		for (int k = 0; k < 3 * sh.NumIndices; k++) tris[k] = sh.Indices[k];
	*ntris = sh.NumIndices;
	return sh.NumVertices;
}

// The 2D helper grid after Prepare (types, BC, velocity and T per (i, j), i-major).
void ref_shape2d_grid(void *vg, unsigned char *type, unsigned char *bc, float *vel2, float *T)
{
	MaskGrid *g = (MaskGrid *)vg;
	FluidSolver2D::Grid2D *g2 = g->GetGrid2D();
	for (int i = 0; i < g2->dimx; i++)
		for (int j = 0; j < g2->dimy; j++)
		{
			size_t c = (size_t)i * g2->dimy + j;
			FluidSolver2D::CondData2D d = g2->GetData(i, j);
			type[c] = (unsigned char)g2->GetType(i, j);
			bc[c] = (unsigned char)d.type;
			vel2[2 * c] = d.vel.x; vel2[2 * c + 1] = d.vel.y; T[c] = d.T;
		}
}

void ref_mask_destroy(void *vg) { delete (MaskGrid *)vg; }

} // extern "C"
