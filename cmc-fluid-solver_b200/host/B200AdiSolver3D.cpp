// B200AdiSolver3D: Solver3D surface over libadi_b200.so (see the header).
#include "B200AdiSolver3D.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{
	const char *status_name(adi_status s)
	{
		switch (s) {
		case ADI_OK: return "ok";
		case ADI_ERR_BAD_ARG: return "bad argument";
		case ADI_ERR_CAPACITY: return "capacity exceeded";
		case ADI_ERR_NONFINITE: return "non-finite field value";
		case ADI_ERR_NOT_CONVERGED: return "not converged";
		case ADI_ERR_CUDA: return "CUDA error";
		case ADI_ERR_TIMEOUT: return "device wait timed out";
		case ADI_ERR_DIVERGENCE: return "divergence error above the guard";
		case ADI_ERR_STATE: return "call out of order";
		case ADI_ERR_NO_DEVICE: return "no sm_100 device";
		default: return "error";
		}
	}
}

namespace FluidSolver3D
{
	B200AdiSolver3D::B200AdiSolver3D(int kind) : h(nullptr), solver_kind(kind)
	{
		grid = nullptr;
		cur = next = nullptr;
		dimx = dimy = dimz = 0;
	}

	B200AdiSolver3D::~B200AdiSolver3D()
	{
		if (h) adi_destroy(h);
	}

	void B200AdiSolver3D::Check(adi_status s)
	{
		if (s == ADI_OK) return;
		const char *msg = h ? adi_last_error_string(h) : nullptr;
		throw std::runtime_error(std::string("libadi_b200: ") + status_name(s) + (msg && *msg ? ": " : "") +
		                         (msg ? msg : ""));
	}

	void B200AdiSolver3D::Init(BackendType, bool, Grid3D *g, FluidParams &p, bool, int)
	{
		grid = g;
		dimx = g->dimx;
		dimy = g->dimy;
		dimz = g->dimz;
		params = p;
		if (h) {
			adi_destroy(h);
			h = nullptr;
		}
		adi_grid_desc d;
		d.dimx = dimx;
		d.dimy = dimy;
		d.dimz = dimz;
		d.dx = g->dx;
		d.dy = g->dy;
		d.dz = g->dz;
		d.precision = sizeof(FTYPE) == 8 ? ADI_FP64 : ADI_FP32;
		// the FluidParams members are already rounded to FTYPE by their constructors
		adi_fluid_params fp;
		fp.v_T = p.v_T;
		fp.v_vis = p.v_vis;
		fp.t_vis = p.t_vis;
		fp.t_phi = p.t_phi;
		Check(adi_create(&d, &fp, &h));
		Check(adi_set_solver(h, solver_kind));
		// Grid3D's Node array (Grid3D.h:73-88) as the ABI's arrays of one field each
		const size_t n = (size_t)dimx * dimy * dimz;
		std::vector<uint8_t> t(n), bv(n), bt(n);
		std::vector<double> vx(n), vy(n), vz(n), T(n);
		const Node *nodes = g->GetNodesCPU();
		for (size_t i = 0; i < n; i++) {
			t[i] = (uint8_t)nodes[i].type;
			bv[i] = (uint8_t)nodes[i].bc_vel;
			bt[i] = (uint8_t)nodes[i].bc_temp;
			vx[i] = nodes[i].v.x;
			vy[i] = nodes[i].v.y;
			vz[i] = nodes[i].v.z;
			T[i] = nodes[i].T;
		}
		Check(adi_set_mask(h, t.data(), bv.data(), bt.data(), vx.data(), vy.data(), vz.data(), T.data()));
	}

	void B200AdiSolver3D::CreateSegments() { Check(adi_build_segments(h, nullptr)); }

	void B200AdiSolver3D::UpdateBoundaries() { Check(adi_update_boundaries(h)); }

	void B200AdiSolver3D::TimeStep(FTYPE dt, int num_global, int num_local, bool computeError)
	{
		Check(adi_time_step(h, (double)dt, num_global, num_local, computeError ? 1 : 0));
	}

	void B200AdiSolver3D::GetLayerB200(Vec3D *v, double *T, int outdimx, int outdimy, int outdimz)
	{
		const size_t m = (size_t)(outdimx ? outdimx : dimx) * (outdimy ? outdimy : dimy) * (outdimz ? outdimz : dimz);
		std::vector<FTYPE> vel(3 * m);
		Check(adi_get_layer(h, outdimx, outdimy, outdimz, vel.data(), T));
		for (size_t i = 0; i < m; i++) {
			v[i].x = vel[3 * i];
			v[i].y = vel[3 * i + 1];
			v[i].z = vel[3 * i + 2];
		}
	}

	double B200AdiSolver3D::sum_layer(char ch)
	{
		if (ch != 'c' && ch != 'n') return 0.0;
		const size_t n = (size_t)dimx * dimy * dimz;
		std::vector<FTYPE> f(4 * n);
		Check(adi_get_state(h, ch == 'c' ? 0 : 1, f.data(), f.data() + n, f.data() + 2 * n, f.data() + 3 * n));
		double s = 0.0;
		for (size_t i = 0; i < f.size(); i++) s += f[i];
		return s;
	}

	void B200AdiSolver3D::debug(bool) {}
}
