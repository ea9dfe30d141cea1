"""GPU parity of the CUDA path (through the C ABI) against the reference and the oracle.

* Exact solver, float: fields equal the reference CPU solver's bit for bit
  (committed golden fixtures made by the reference itself, and the pinned C
  restatement on fresh random domains).
* Exact solver, double: equal to the double restatement bit for bit.
* Segment lists: identical to Grid3D::GenerateListSegments, edge masks included.
"""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G
from golden_util import GOLDEN, case_name, fluid_params_tuple, load_case, non_out, step_cases

pytestmark = pytest.mark.gpu


def make_solver(adi_lib, d, params, precision=None, solver=None):
    from adi_b200 import _abi
    kind, p = params
    if kind == "normalized":
        fp = adi_lib.fluid_params_normalized(*p)
    else:
        fp = adi_lib.fluid_params_dimensional(*p)
    s = adi_lib.AdiSolver3D(d, params=fp, precision=precision or _abi.ADI_FP32,
                            solver=_abi.ADI_SOLVER_EXACT if solver is None else solver)
    s.CreateSegments()
    return s


@pytest.mark.parametrize("path", step_cases(), ids=case_name)
def test_segments_match_golden(adi_lib, path):
    d, run, params, z = load_case(path)
    s = make_solver(adi_lib, d, params)
    for dr in range(3):
        np.testing.assert_array_equal(s.segments(dr), z[f"segs{dr}"])


def test_segments_edge_masks(adi_lib):
    z = np.load(f"{GOLDEN}/segments_edge.npz")
    names = sorted({k[: -len("_type")] for k in z.files if k.endswith("_type")})
    for name in names:
        t = z[f"{name}_type"]
        shape = t.shape
        zero = np.zeros(shape)
        d = G.Domain(*shape, 0.1, 0.1, 0.1, t, np.zeros(shape, np.uint8), np.zeros(shape, np.uint8),
                     zero, zero, zero, zero)
        s = make_solver(adi_lib, d, ("normalized", (100.0, 0.72, 1.4)))
        for dr in range(3):
            got = s.segments(dr)
            np.testing.assert_array_equal(got, z[f"{name}_segs{dr}"], err_msg=f"{name} dir {dr}")
        st = s.stats
        for dr in range(3):
            ref = z[f"{name}_segs{dr}"]
            assert st["num_segments"][dr] == len(ref)
            assert st["num_nodes"][dr] == int(ref[:, 6].sum()) if len(ref) else st["num_nodes"][dr] == 0


@pytest.mark.parametrize("path", step_cases(), ids=case_name)
def test_exact_fp32_equals_reference_golden(adi_lib, path):
    d, run, params, z = load_case(path)
    s = make_solver(adi_lib, d, params)
    m = non_out(d)
    keep = set(int(k) for k in z["keep"])
    for step in range(1, run["steps"] + 1):
        st = s.step(run["dt"], run["num_global"], run["num_local"], True)
        want = int(z["status"][step - 1])
        assert (st == 0) == (want == 0), (step, st, want)
        assert s.div_error() == pytest.approx(float(z["div_error"][step - 1]), rel=1e-12, abs=1e-300)
        if step in keep:
            got = s.fields(0)
            for f, name in enumerate("uvwT"):
                ref = z[f"step{step}_{name}"]
                bad = np.flatnonzero(got[f][m] != ref[m])
                assert bad.size == 0, (step, name, bad.size, got[f][m][bad[:3]], ref[m][bad[:3]])


@pytest.mark.parametrize("seed,shell", [(31, False), (32, True), (33, False)])
def test_exact_fp32_equals_oracle_random(adi_lib, seed, shell):
    d = G.random_domain(18, 15, 21, seed=seed, shell=shell, n_obstacles=7, rmax=3.5)
    assert G.validate_for_solver(d, strict_div=True) is None
    params = ("normalized", (90.0, 0.8, 1.5))
    s = make_solver(adi_lib, d, params)
    orc = O.OracleSolver(d, precision=4, params=fluid_params_tuple(params))
    m = non_out(d)
    for step in range(4):
        assert s.step(8e-4, 3, 2, step % 2 == 0) == orc.step(8e-4, 3, 2, step % 2 == 0)
        got, want = s.fields(0), orc.fields(0)
        for f in range(4):
            assert np.array_equal(got[f][m].astype(np.float64), want[f][m]), (step, f)
        # next holds the pre-step state plus this step's boundary writes
        got_n, want_n = s.fields(1), orc.fields(1)
        for f in range(4):
            assert np.array_equal(got_n[f][m].astype(np.float64), want_n[f][m]), (step, f, "next")


def test_exact_fp64_equals_oracle_fp64(adi_lib):
    from adi_b200 import _abi
    d = G.random_domain(16, 17, 14, seed=41, n_obstacles=5)
    params = ("normalized", (150.0, 0.72, 1.4))
    s = make_solver(adi_lib, d, params, precision=_abi.ADI_FP64)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(params))
    m = non_out(d)
    for step in range(3):
        assert s.step(1e-3, 4, 2, True) == orc.step(1e-3, 4, 2, True)
        got, want = s.fields(0), orc.fields(0)
        for f in range(4):
            assert np.array_equal(got[f][m], want[f][m]), (step, f)
    assert s.div_error() == pytest.approx(orc.div_error(), rel=1e-13)


def test_exact_is_deterministic(adi_lib):
    d = G.spheres_channel(dims=(40, 36, 44), n_spheres=6, rmin=2, rmax=5, seed=4).round_values_to_float32()
    out = []
    for _ in range(2):
        s = make_solver(adi_lib, d, ("normalized", (200.0, 0.72, 1.4)))
        for _ in range(3):
            assert s.step(5e-4, 4, 2, False) == 0
        out.append(s.fields(0))
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_fp32_error_vs_fp64_oracle_within_reference_drift(adi_lib):
    """Float GPU result against the double oracle, relative to each field's scale,
    is no worse than the reference's own float drift (the float restatement equals
    the reference bit for bit) and below 1e-5 of the flow scale."""
    d = G.spheres_channel(dims=(48, 40, 40), n_spheres=5, rmin=3, rmax=6, seed=7).round_values_to_float32()
    params = ("normalized", (200.0, 0.72, 1.4))
    s = make_solver(adi_lib, d, params)
    o32 = O.OracleSolver(d, precision=4, params=fluid_params_tuple(params))
    o64 = O.OracleSolver(d, precision=8, params=fluid_params_tuple(params))
    for _ in range(10):
        s.step(5e-4, 4, 2, False)
        o32.step(5e-4, 4, 2, False)
        o64.step(5e-4, 4, 2, False)
    m = non_out(d)
    g, a, b = s.fields(0), o32.fields(0), o64.fields(0)
    vscale = max(np.max(np.abs(b[f][m])) for f in range(3))
    for f in range(4):
        scale = vscale if f < 3 else np.max(np.abs(b[3][m]))
        err_gpu = np.max(np.abs(g[f][m] - b[f][m])) / scale
        err_ref = np.max(np.abs(a[f][m] - b[f][m])) / scale
        assert err_gpu <= 1e-5
        assert err_gpu <= 1.5 * err_ref + 1e-7


def test_contract_violation_is_rejected(adi_lib):
    from adi_b200 import _abi
    d = G.random_domain(10, 10, 10, seed=1)
    d.type[0, 5, 5] = G.NODE_IN  # IN on the outer frame
    s = make_solver(adi_lib, d, ("normalized", (100.0, 0.72, 1.4)))
    assert s.step(1e-3, 2, 1, False) == 1  # ADI_ERR_BAD_ARG
    d2 = G.random_domain(10, 10, 10, seed=1)
    d2.type[5, 5, 5] = G.NODE_IN
    d2.type[5, 5, 6] = G.NODE_OUT    # IN next to OUT
    s2 = make_solver(adi_lib, d2, ("normalized", (100.0, 0.72, 1.4)))
    with pytest.raises(_abi.AdiError):
        s2.TimeStep(1e-3, 2, 1)


def test_call_order_and_argument_errors(adi_lib):
    from adi_b200 import _abi
    d = G.random_domain(10, 9, 8, seed=2)
    s = adi_lib.AdiSolver3D(d, Re=100.0, solver=_abi.ADI_SOLVER_EXACT)
    assert s.step(1e-3, 2, 1, False) == 8      # ADI_ERR_STATE: segments not built
    s.CreateSegments()
    assert s.step(1e-3, 0, 1, False) == 1      # num_global < 1
    assert s.step(-1.0, 2, 1, False) == 1      # dt <= 0
    assert s.step(1e-3, 2, 1, False) == 0


def test_get_layer_semantics(adi_lib):
    """GetLayer reads `next` (the state the last step started from), with OUT cells
    set to 99999, point-sampled at x = i*dimx/outdimx."""
    d = G.random_domain(16, 14, 12, seed=5, shell=True, n_obstacles=4, rmax=4.0)
    params = ("normalized", (100.0, 0.72, 1.4))
    s = make_solver(adi_lib, d, params)
    orc = O.OracleSolver(d, precision=4, params=fluid_params_tuple(params))
    for _ in range(2):
        s.step(1e-3, 2, 1, False)
        orc.step(1e-3, 2, 1, False)
    ox, oy, oz = 7, 5, 6
    v, T = s.GetLayer(ox, oy, oz)
    nxt = orc.fields(1)
    out = d.type == G.NODE_OUT
    for f in range(4):
        nxt[f][out] = np.float32(99999.0)
    ii = np.arange(ox) * d.nx // ox
    jj = np.arange(oy) * d.ny // oy
    kk = np.arange(oz) * d.nz // oz
    sel = np.ix_(ii, jj, kk)
    for f in range(3):
        np.testing.assert_array_equal(v[..., f].astype(np.float64), nxt[f][sel])
    np.testing.assert_array_equal(T, nxt[3][sel])


def test_divergence_guard_matches_reference(adi_lib):
    """A state with divergence above 0.01 makes the step fail like the reference's
    throw, leaving the layers unswapped."""
    from adi_b200 import _abi
    d = G.random_domain(12, 12, 12, seed=9)
    d.dx = d.dy = d.dz = 0.5
    params = ("normalized", (50.0, 0.72, 1.4))
    s = make_solver(adi_lib, d, params)
    orc = O.OracleSolver(d, precision=4, params=fluid_params_tuple(params))
    rng = np.random.default_rng(0)
    st = [rng.standard_normal(d.shape).astype(np.float32) for _ in range(3)] + [np.ones(d.shape, np.float32)]
    s.set_state(*st)
    orc.set_state(*[a.astype(np.float64) for a in st])
    before = s.fields(0)
    rc = s.step(1e-3, 1, 1, True)
    assert rc == 7                              # ADI_ERR_DIVERGENCE
    assert orc.step(1e-3, 1, 1, True) == 1      # the reference's throw
    assert orc.last_div_error() > 0.01
    after = s.fields(0)
    m = d.type == G.NODE_IN
    for a, b in zip(before, after):
        assert np.array_equal(a[m], b[m])
