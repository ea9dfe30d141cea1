"""Parity at the benchmarked workloads, with the kernels the benchmark runs.

The benchmark's headline workload is spheres128: a 128^3 float box with 40 solid
spheres (seed 0), Re 200, dt 5e-4, num_global 4, num_local 2, stepped by
UpdateBoundaries + TimeStep (AdiSolver3D.cpp:286-391, FluidSolver3D.cpp:241-242).
Its autotuner picks among the TMA-fed X/Y sweep's shapes (8 or 16 lines per CTA,
chunks of K = 4 or 8 rows, so P = 32 or 16 chunks per 128-row line) and the
warp-resident Z sweep (K = 4, P = 32 or K = 8, P = 16); every such shape is a
separate template instantiation, so the tests pin each one and compare it with
the oracle on the full-size domain:

* the exact solver equals the reference's own CPU solver (oracle/_ref) bit for
  bit after two driver steps;
* the fast solver in double equals the double C restatement within 1e-11 of each
  field's scale after two steps;
* the fast solver in float stays within 1e-5 (max relative error over fluid and
  boundary cells, the metric's accuracy bound) of the double restatement after ten
  steps.

The large single domain (ellipsoids384, one step) and a member of the batched
workload (batched64) are compared the same way with the shapes their autotuners pick,
and the FP64 adjoint of two spheres128 steps against the FP64 adjoint restatement.
"""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G
from golden_util import fluid_params_tuple, non_out

pytestmark = pytest.mark.gpu

PARAMS = ("normalized", (200.0, 0.72, 1.4))
DT = 5e-4

# (K, NL) per direction as set_fast_shape takes them: NL = -8 / -16 is the TMA
# X/Y sweep with 8 / 16 lines per CTA, NL = 0 the warp-resident Z sweep.
HEADLINE_SHAPES = [
    [(4, -8), (4, -8), (4, 0)],
    [(4, -8), (8, -16), (8, 0)],
    [(8, -8), (8, -8), (4, 0)],
    [(8, -16), (8, -16), (4, 0)],
]


def _ids(s):
    return "-".join(f"K{k}NL{n}" for k, n in s)


@pytest.fixture(scope="module")
def spheres128():
    return G.spheres_channel(n=128, n_spheres=40, rmin=4.0, rmax=12.0, seed=0)


@pytest.fixture(scope="module")
def oracle64_spheres128(spheres128):
    """FP64 restatement states after 2 and 10 steps (shared by the tests below)."""
    o = O.OracleSolver(spheres128, precision=8, params=fluid_params_tuple(PARAMS))
    states = {}
    for step in range(1, 11):
        assert o.step(DT, 4, 2, step % 10 == 0) == 0
        if step in (2, 10):
            states[step] = (o.fields(0), o.fields(1))
    o.close()
    return states


def _solver(adi_lib, d, precision, solver, shapes=None, Re=200.0):
    from adi_b200 import _abi
    fp = adi_lib.fluid_params_normalized(Re, 0.72, 1.4)
    s = adi_lib.AdiSolver3D(d, params=fp, precision=precision, solver=solver)
    s.CreateSegments()
    if shapes:
        for dr, (K, NL) in enumerate(shapes):
            s.set_fast_shape(dr, K, NL)
        got = s.fast_shapes()
        for dr, (K, NL) in enumerate(shapes):
            assert got[dr][0] == K and got[dr][1] == NL, (dr, got)
    return s


def _rel(got, want, m):
    vs = max(np.max(np.abs(want[f][m])) for f in range(3))
    out = []
    for f in range(4):
        scale = vs if f < 3 else np.max(np.abs(want[3][m]))
        out.append(float(np.max(np.abs(got[f][m].astype(np.float64) - want[f][m])) / scale))
    return out


def test_exact_equals_reference_spheres128(adi_lib, spheres128):
    from adi_b200 import _abi
    if not O.have_ref():
        pytest.skip("reference build oracle/_ref/libref3d.so missing")
    d = spheres128
    s = _solver(adi_lib, d, _abi.ADI_FP32, _abi.ADI_SOLVER_EXACT)
    ref = O.RefSolver(d, Re=200.0)
    m = non_out(d)
    for step in range(2):
        assert s.step(DT, 4, 2, True) == 0
        assert ref.step(DT, 4, 2, True) == 0
    got, want = s.fields(0), ref.fields(0)
    for f in range(4):
        bad = np.flatnonzero(got[f][m] != want[f][m])
        assert bad.size == 0, ("uvwT"[f], bad.size)
    assert s.div_error() == pytest.approx(ref.div_error(), rel=1e-6)
    ref.close()


@pytest.mark.parametrize("shapes", HEADLINE_SHAPES, ids=_ids)
def test_fast_fp64_spheres128(adi_lib, spheres128, oracle64_spheres128, shapes):
    from adi_b200 import _abi
    d = spheres128
    s = _solver(adi_lib, d, _abi.ADI_FP64, _abi.ADI_SOLVER_FAST, shapes)
    for step in range(2):
        assert s.step(DT, 4, 2, False) == 0
    m = non_out(d)
    want0, want1 = oracle64_spheres128[2]
    errs = _rel(s.fields(0), want0, m)
    assert max(errs) < 1e-11, errs
    errs_n = _rel(s.fields(1), want1, m)
    assert max(errs_n) < 1e-11, errs_n


@pytest.mark.parametrize("shapes", HEADLINE_SHAPES, ids=_ids)
def test_fast_fp32_spheres128_ten_steps(adi_lib, spheres128, oracle64_spheres128, shapes):
    from adi_b200 import _abi
    d = spheres128
    s = _solver(adi_lib, d, _abi.ADI_FP32, _abi.ADI_SOLVER_FAST, shapes)
    for step in range(1, 11):
        assert s.step(DT, 4, 2, step % 10 == 0) == 0
    errs = _rel(s.fields(0), oracle64_spheres128[10][0], non_out(d))
    assert max(errs) <= 1e-5, errs


def test_autotuned_spheres128_runs_specialised_kernels(adi_lib, spheres128):
    """The autotuner's choice on the headline workload is one of the pinned shapes'
    kernel families (TMA X/Y, warp-resident Z), so the tests above cover it."""
    from adi_b200 import _abi
    s = _solver(adi_lib, spheres128, _abi.ADI_FP32, _abi.ADI_SOLVER_FAST)
    sh = s.fast_shapes()
    assert sh[0][1] < 0 and sh[1][1] < 0, sh
    assert sh[2][1] == 0, sh


def test_fast_fp64_ellipsoids384_one_step(adi_lib):
    """ellipsoids384 (384^3, 300 ellipsoids, a thin-walled tube; Re 500, dt 2e-4):
    one step of the fast solver in double with the autotuned shapes against the
    double restatement."""
    from adi_b200 import _abi
    d = G.ellipsoids_tube(n=384, n_ellipsoids=300, amin=3.0, amax=20.0, seed=1)
    s = _solver(adi_lib, d, _abi.ADI_FP64, _abi.ADI_SOLVER_FAST, Re=500.0)
    assert s.step(2e-4, 4, 2, False) == 0
    got = s.fields(0)
    s.close()
    o = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", (500.0, 0.72, 1.4))))
    assert o.step(2e-4, 4, 2, False) == 0
    want = o.fields(0)
    o.close()
    errs = _rel(got, want, non_out(d))
    assert max(errs) < 1e-11, errs


def test_batched64_member_against_oracle(adi_lib):
    """The largest member of the batched64 workload, stepped inside a batch of the
    workload's first eight domains (FP32, autotuned binning), against the double
    restatement after five steps."""
    from adi_b200 import _abi
    ds = G.batch_of_domains(n_domains=8, seed=2, size_lo=64, size_hi=160, spheres=(10, 60), rmin=4.0,
                            rmax=12.0, re=(50.0, 400.0))
    q = int(np.argmax([d.cells for d in ds]))
    members = [_solver(adi_lib, d, _abi.ADI_FP32, _abi.ADI_SOLVER_FAST, Re=d.meta["Re"]) for d in ds]
    b = adi_lib.AdiBatch(members)
    b.autotune(5e-4, 2)
    o = O.OracleSolver(ds[q], precision=8, params=fluid_params_tuple(("normalized", (ds[q].meta["Re"], 0.72, 1.4))))
    for step in range(5):
        assert b.step(5e-4, 4, 2, step == 4) == 0, b.last_error()
        assert o.step(5e-4, 4, 2, step == 4) == 0
    errs = _rel(members[q].fields(0), o.fields(0), non_out(ds[q]))
    assert max(errs) <= 1e-5, errs
    assert abs(b.div_errors()[q] - o.div_error()) < 1e-6


def test_fp64_adjoint_spheres128_against_oracle_adjoint(adi_lib, spheres128):
    """The adjoint at the adjoint workload's size: two steps of spheres128 (Re 200,
    dt 5e-4, num_global 4, num_local 2, windows of one step), J over the 32^3 box
    next to the inflow, FP64 GPU adjoint with the default (split) sweep against the
    FP64 CPU adjoint restatement.  (The fused and split sweeps agree to 1e-12 on
    small domains, test_gpu_adjoint.py.)"""
    from adi_b200 import _abi
    d = spheres128
    lo, hi = (2, 48, 48), (34, 80, 80)
    s = _solver(adi_lib, d, _abi.ADI_FP64, _abi.ADI_SOLVER_FAST)
    J, gnv, gst = s.adjoint_run(DT, 4, 2, 2, 1, lo, hi)
    o = O.OracleSolver(d, precision=8, params=fluid_params_tuple(PARAMS))
    Jo, gnvo, gsto = o.adjoint_run(DT, 4, 2, 2, lo, hi)
    o.close()
    assert abs(J - Jo) <= 1e-12 * abs(Jo)
    for a, b in ((gnv, gnvo), (gst, gsto)):
        scale = np.max(np.abs(b))
        assert scale > 0
        assert np.max(np.abs(a - b)) <= 1e-9 * scale
