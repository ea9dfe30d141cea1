// B200AdiSolver3D: the reference's solver surface over the B200 library.
//
// The reference's driver (FluidSolver3D/FluidSolver3D.cpp:176-262) talks to its
// solver through the abstract Solver3D (FluidSolver3D/Solver3D.h:24-49).  This
// class implements that surface on top of the C ABI of libadi_b200.so
// (include/adi_b200.h), so a host adds this header and B200AdiSolver3D.cpp to its
// FluidSolver3D tree, constructs B200AdiSolver3D where it constructs AdiSolver3D,
// and keeps its loop: CreateSegments() once, then UpdateBoundaries() and
// TimeStep() per step.  The one call that changes is GetLayer: Solver3D::GetLayer
// is not virtual (Solver3D.h:31) and reads host time layers this class does not
// keep, so the driver calls GetLayerB200 on the adapter instead (same arguments,
// same output: Solver3D.cpp:21-25 with TimeLayer3D::FilterToArrays).
//
// Errors: every ABI status other than ADI_OK becomes std::runtime_error with the
// handle's message, as the reference's gpuSafeCall does (Common/GPUplan.cpp:173-193);
// ADI_ERR_DIVERGENCE is the reference's divergence-guard throw
// (AdiSolver3D.cpp:371-374), after which the layers are left unswapped.
//
// Build: -I<repo>/include with the reference's include paths; link
// -L<repo>/cmc-fluid-solver_b200/adi_b200 -ladi_b200 -lcudart.
#pragma once

#include "Solver3D.h"
#include "adi_b200.h"

namespace FluidSolver3D
{
	class B200AdiSolver3D : public Solver3D
	{
	public:
		// solver_kind: ADI_SOLVER_FAST (chunked sweeps, the default) or
		// ADI_SOLVER_EXACT (the reference's operation order, bit-identical results).
		explicit B200AdiSolver3D(int solver_kind = ADI_SOLVER_FAST);
		~B200AdiSolver3D() override;

		// AdiSolver3D::Init (AdiSolver3D.cpp:166-268): creates the device handle,
		// uploads the grid's node array (type, BCs, values; the values are also the
		// initial state, as TimeLayer3D(grid) copies them).  backend, csvFormat,
		// useBlocking and nblockZ select reference code paths that do not exist here.
		void Init(BackendType backend, bool csvFormat, Grid3D *grid, FluidParams &params, bool useBlocking,
		          int nblockZ) override;
		// AdiSolver3D::CreateSegments (AdiSolver3D.cpp:553-562)
		void CreateSegments();
		// AdiSolver3D::UpdateBoundaries (AdiSolver3D.cpp:286-304)
		void UpdateBoundaries() override;
		// AdiSolver3D::TimeStep (AdiSolver3D.cpp:306-391)
		void TimeStep(FTYPE dt, int num_global, int num_local, bool computeError) override;
		// Solver3D::GetLayer (Solver3D.cpp:21-25)
		void GetLayerB200(Vec3D *v, double *T, int outdimx = 0, int outdimy = 0, int outdimz = 0);
		// AdiSolver3D::sum_layer ('c' cur, 'n' next; the reference's version returns 0
		// because its summation is commented out, AdiSolver3D.cpp:30-58)
		double sum_layer(char ch) override;
		void debug(bool ifdebug) override;

		adi_handle *Handle() { return h; }

	private:
		adi_handle *h;
		int solver_kind;
		void Check(adi_status s);
	};
}
