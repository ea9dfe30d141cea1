"""The B200AdiSolver3D host adapter (cmc-fluid-solver_b200/host) on the reference's side.

oracle/Makefile compiles the adapter together with the reference's own headers
(Solver3D.h, Grid3D.h, Geometry.h) into oracle/_ref/libadapter3d.so; that it
compiles there is the check that its overrides match Solver3D
(FluidSolver3D/Solver3D.h:24-49).  The CPU test checks the built library's
symbols; the GPU test runs the reference driver loop (FluidSolver3D.cpp:224-262:
CreateSegments, then UpdateBoundaries + TimeStep per step, GetLayer) through it
and compares the output with the reference solver's own GetLayer.
"""
import ctypes as C
import subprocess

import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G


def _adapter_or_skip():
    if not O.have_adapter():
        pytest.skip("oracle/_ref/libadapter3d.so not built (needs the reference checkout)")


def test_adapter_library_exports_the_solver3d_overrides():
    _adapter_or_skip()
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", O.ADAPTER_LIB], capture_output=True, text=True,
                         check=True).stdout
    assert " adapter_run" in out
    for method in ("Init(", "TimeStep(", "UpdateBoundaries()", "GetLayerB200(", "sum_layer(", "debug(",
                   "CreateSegments()"):
        assert f"FluidSolver3D::B200AdiSolver3D::{method}" in out, method
    # the vtable: B200AdiSolver3D is a complete Solver3D (no pure virtual left)
    assert "vtable for FluidSolver3D::B200AdiSolver3D" in out
    assert C.CDLL(O.ADAPTER_LIB).adapter_run


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["exact", "fast"])
def test_reference_driver_loop_through_adapter(adi_lib, solver):
    """Three driver-loop steps through the adapter against the reference CPU solver:
    GetLayer output bit-identical with the exact solver, within 1e-5 of the flow
    scale with the fast one."""
    _adapter_or_skip()
    if not O.have_ref():
        pytest.skip("reference build missing")
    from adi_b200 import _abi
    d = G.spheres_channel(dims=(48, 40, 44), n_spheres=5, rmin=3.0, rmax=6.0, seed=7).round_values_to_float32()
    Re, Pr, lam, dt, ng, nl, steps = 200.0, 0.72, 1.4, 5e-4, 4, 2, 3
    kind = _abi.ADI_SOLVER_EXACT if solver == "exact" else _abi.ADI_SOLVER_FAST
    va, Ta = O.adapter_run(d, Re, Pr, lam, dt, ng, nl, steps, kind)
    ref = O.RefSolver(d, Re=Re, Pr=Pr, lam=lam)
    for i in range(steps):
        assert ref.step(dt, ng, nl, (i % 10 == 0) or (i + 1 == steps)) == 0
    vr, Tr = ref.get_layer()
    ref.close()
    if solver == "exact":
        assert np.array_equal(va, vr)
        assert np.array_equal(Ta, Tr)
    else:
        m = d.type != G.NODE_OUT
        vs = float(np.max(np.abs(vr[m])))
        assert float(np.max(np.abs(va[m] - vr[m]))) <= 1e-5 * vs
        assert float(np.max(np.abs(Ta[m] - Tr[m]))) <= 1e-5 * float(np.max(np.abs(Tr[m])))
        assert np.array_equal(va[~m], vr[~m]) and np.array_equal(Ta[~m], Tr[~m])   # 99999 at OUT cells
    # a coarser output grid (FilterToArrays point sampling) through both
    va2, Ta2 = O.adapter_run(d, Re, Pr, lam, dt, ng, nl, 1, _abi.ADI_SOLVER_EXACT, outdims=(24, 20, 11))
    ref = O.RefSolver(d, Re=Re, Pr=Pr, lam=lam)
    assert ref.step(dt, ng, nl, True) == 0
    vr2, Tr2 = ref.get_layer(24, 20, 11)
    ref.close()
    assert np.array_equal(va2, vr2) and np.array_equal(Ta2, Tr2)
