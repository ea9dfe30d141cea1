"""GPU checks of the graph-replayed step and of tolerance mode.

Graph replay must give the same bits as issuing the kernels directly (the same
kernels run in the same order), and the launch accounting must agree.  Tolerance
mode is compared with the oracle's restatement of the same iteration rule (FP64,
fields to 1e-11 of their scale, residuals to 1e-6 relative) and must reduce to the
fixed-iteration step when tol = 0.
"""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G
from golden_util import fluid_params_tuple, non_out

pytestmark = pytest.mark.gpu


def _solver(adi_lib, d, params, precision=None, solver=None, graphs=True):
    from adi_b200 import _abi
    fp = adi_lib.fluid_params_normalized(*params)
    s = adi_lib.AdiSolver3D(d, params=fp, precision=precision or _abi.ADI_FP32,
                            solver=_abi.ADI_SOLVER_FAST if solver is None else solver)
    s.CreateSegments()
    s.set_graphs(graphs)
    return s


@pytest.mark.parametrize("solver", ["fast", "exact"])
def test_graph_replay_matches_direct_launches(adi_lib, solver):
    from adi_b200 import _abi
    kind = _abi.ADI_SOLVER_FAST if solver == "fast" else _abi.ADI_SOLVER_EXACT
    d = G.random_domain(40, 36, 48, seed=101, shell=True, n_obstacles=8, rmax=4.5)
    params = (150.0, 0.72, 1.4)
    a = _solver(adi_lib, d, params, solver=kind, graphs=True)
    b = _solver(adi_lib, d, params, solver=kind, graphs=False)
    for s in (a, b):
        if solver == "fast":
            for sh in range(3):
                K, NL, _ = b.fast_shapes()[sh]
                s.set_fast_shape(sh, K, NL)     # same kernels in both
        s.profile(reset=True)
    for i in range(11):
        assert a.step(7e-4, 3, 2, i % 5 == 0) == b.step(7e-4, 3, 2, i % 5 == 0) == 0
    for f in range(4):
        assert np.array_equal(a.fields(0)[f], b.fields(0)[f])
        assert np.array_equal(a.fields(1)[f], b.fields(1)[f])
    pa, pb = a.profile(reset=True), b.profile(reset=True)
    for k in pa:
        assert pa[k]["launches"] == pb[k]["launches"], k
        assert pa[k]["bytes"] == pb[k]["bytes"], k
    assert a.div_error() == b.div_error()


def test_run_and_reconfiguration_keep_graphs_consistent(adi_lib):
    d = G.random_domain(32, 30, 32, seed=102, shell=True, n_obstacles=6, rmax=4.0)
    params = (120.0, 0.72, 1.4)
    a = _solver(adi_lib, d, params, graphs=True)
    b = _solver(adi_lib, d, params, graphs=False)
    for sh in range(2):
        K, NL, _ = a.fast_shapes()[sh]
        b.set_fast_shape(sh, K, NL)            # the two autotuners may pick different X/Y kernels
    a.set_fast_shape(2, 4, 8)
    b.set_fast_shape(2, 4, 8)
    a.run(8e-4, 2, 2, 7, err_every=3)
    for i in range(7):
        assert b.step(8e-4, 2, 2, i % 3 == 0 or i == 6) == 0
    for f in range(4):
        assert np.array_equal(a.fields(0)[f], b.fields(0)[f])
    # a shape change after capture must not replay the old kernels
    a.set_fast_shape(2, 8, 8)
    b.set_fast_shape(2, 8, 8)
    for i in range(3):
        assert a.step(8e-4, 2, 2, False) == b.step(8e-4, 2, 2, False) == 0
    for f in range(4):
        assert np.array_equal(a.fields(0)[f], b.fields(0)[f])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tolerance_mode_matches_oracle(adi_lib, precision):
    from adi_b200 import _abi
    d = G.random_domain(36, 32, 40, seed=103, shell=True, n_obstacles=7, rmax=4.0)
    params = (140.0, 0.72, 1.4)
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    s = _solver(adi_lib, d, params, precision=prec)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    # residuals of the first step for 1..4 iterations pick a tolerance between the 2nd and 3rd
    probe = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    r = [O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
         .step_tol(7e-4, k, 2, 0.0)[2] for k in (1, 2, 3)]
    del probe
    assert r[2] < r[1] < r[0]
    tol = float(np.sqrt(r[1] * r[2]))
    m = non_out(d)
    for step in range(3):
        rc, it, res = s.step_tol(7e-4, 6, 2, tol, step == 2)
        orc_rc, orc_it, orc_res = orc.step_tol(7e-4, 6, 2, tol, step == 2)
        assert rc == orc_rc == 0
        assert it == orc_it, (step, it, orc_it, res, orc_res)
        assert abs(res - orc_res) <= (1e-6 if precision == "fp64" else 2e-2) * orc_res
        assert res <= tol
    scale = [max(np.max(np.abs(o[m])) for o in orc.fields(0)[:3])] * 3 + [np.max(np.abs(orc.fields(0)[3][m]))]
    for f in range(4):
        err = np.max(np.abs(s.fields(0)[f][m].astype(np.float64) - orc.fields(0)[f][m])) / scale[f]
        assert err < (1e-11 if precision == "fp64" else 2e-6), (f, err)


def test_tolerance_zero_is_the_fixed_iteration_step(adi_lib):
    d = G.random_domain(30, 28, 32, seed=104, n_obstacles=5, rmax=4.0)
    params = (100.0, 0.72, 1.4)
    a = _solver(adi_lib, d, params)
    b = _solver(adi_lib, d, params)
    for sh in range(3):
        K, NL, _ = a.fast_shapes()[sh]
        b.set_fast_shape(sh, K, NL)
    for i in range(3):
        rc, it, res = a.step_tol(9e-4, 3, 2, 0.0, True)
        assert (rc, it) == (0, 3) and res > 0
        assert b.step(9e-4, 3, 2, True) == 0
    for f in range(4):
        assert np.array_equal(a.fields(0)[f], b.fields(0)[f])
    rc, it, res = a.step_tol(9e-4, 4, 2, 1.0)     # loose: one iteration
    assert (rc, it) == (0, 1)
