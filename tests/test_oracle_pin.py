"""Pins the CPU restatement oracle (oracle/adi_oracle.c) to the reference.

1. Against the committed golden fixtures made by the reference's own CPU solver
   (tests/golden/make_golden.py): segment lists and float fields must be identical
   bit for bit, divergence errors equal.
2. Against the reference build itself (oracle/_ref/libref3d.so) on fresh random
   domains, when that build is present.
"""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G
from golden_util import fluid_params_tuple, load_case, non_out, step_cases, case_name, GOLDEN


@pytest.mark.parametrize("path", step_cases(), ids=case_name)
def test_restatement_matches_golden(path):
    d, run, params, z = load_case(path)
    orc = O.OracleSolver(d, precision=4, params=fluid_params_tuple(params))
    for dr in range(3):
        np.testing.assert_array_equal(O.oracle_segments(d.type, dr), z[f"segs{dr}"])
    m = non_out(d)
    keep = set(int(k) for k in z["keep"])
    for s in range(1, run["steps"] + 1):
        st = orc.step(run["dt"], run["num_global"], run["num_local"], True)
        assert st == int(z["status"][s - 1])
        assert orc.div_error() == z["div_error"][s - 1]
        if s in keep:
            got = orc.fields(0)
            for f, name in enumerate("uvwT"):
                ref = z[f"step{s}_{name}"].astype(np.float64)
                assert np.array_equal(got[f][m], ref[m]), (s, name)
    orc.close()


def test_segments_edge_masks_golden():
    z = np.load(f"{GOLDEN}/segments_edge.npz")
    names = sorted({k[: -len("_type")] for k in z.files if k.endswith("_type")})
    assert names
    for name in names:
        t = z[f"{name}_type"]
        for dr in range(3):
            np.testing.assert_array_equal(O.oracle_segments(t, dr), z[f"{name}_segs{dr}"], err_msg=f"{name} dir {dr}")


@pytest.mark.skipif(not O.have_ref(), reason="reference build oracle/_ref/libref3d.so not present")
@pytest.mark.parametrize("seed", [21, 22, 23])
def test_restatement_matches_reference_live(seed):
    d = G.random_domain(14, 12, 16, seed=seed, shell=bool(seed % 2), n_obstacles=5)
    assert G.validate_for_solver(d) is None
    ref = O.RefSolver(d, Re=120.0, Pr=0.9, lam=1.3)
    orc = O.OracleSolver(d, precision=4, Re=120.0, Pr=0.9, lam=1.3)
    for dr in range(3):
        np.testing.assert_array_equal(ref.segments(dr), O.oracle_segments(d.type, dr))
    m = non_out(d)
    for s in range(3):
        assert ref.step(7e-4, 3, 2, True) == orc.step(7e-4, 3, 2, True)
        fr, fo = ref.fields(0), orc.fields(0)
        for f in range(4):
            assert np.array_equal(fr[f][m].astype(np.float64), fo[f][m])
        assert ref.div_error() == orc.div_error()


@pytest.mark.skipif(not O.have_ref(), reason="reference build oracle/_ref/libref3d.so not present")
def test_time_step_without_boundary_update_live():
    """TimeStep alone, from a state whose boundary cells differ from the node values:
    Dirichlet rows take the node values, every other read takes the state."""
    d = G.random_domain(14, 13, 15, seed=24, shell=True, n_obstacles=5)
    ref = O.RefSolver(d, Re=110.0, Pr=0.8, lam=1.3)
    orc = O.OracleSolver(d, precision=4, Re=110.0, Pr=0.8, lam=1.3)
    rng = np.random.default_rng(24)
    state = [(a + 0.05 * rng.standard_normal(d.shape)).astype(np.float32) for a in (d.vx, d.vy, d.vz, d.T)]
    ref.set_state(*state)
    orc.set_state(*[a.astype(np.float64) for a in state])
    m = non_out(d)
    for s in range(2):
        assert ref.time_step(6e-4, 2, 2, True) == orc.time_step(6e-4, 2, 2, True)
        fr, fo = ref.fields(0), orc.fields(0)
        for f in range(4):
            assert np.array_equal(fr[f][m].astype(np.float64), fo[f][m])


@pytest.mark.skipif(not O.have_ref(), reason="reference build oracle/_ref/libref3d.so not present")
def test_segment_lists_random_masks_live():
    rng = np.random.default_rng(5)
    for trial in range(6):
        shape = tuple(int(x) for x in rng.integers(3, 14, size=3))
        t = rng.integers(0, 4, size=shape).astype(np.uint8)
        t[rng.random(shape) < 0.5] = G.NODE_IN
        z = np.zeros(shape)
        d = G.Domain(*shape, 0.1, 0.1, 0.1, t, np.zeros(shape, np.uint8), np.zeros(shape, np.uint8), z, z, z, z)
        ref = O.RefSolver(d)
        for dr in range(3):
            np.testing.assert_array_equal(ref.segments(dr), O.oracle_segments(t, dr))
        ref.close()


def test_fp64_oracle_tracks_fp32():
    """The double instantiation solves the same equations: after a few steps the
    float run is close to it, relative to each field's scale."""
    d = G.random_domain(14, 12, 10, seed=3)
    a = O.OracleSolver(d, precision=4, Re=100.0)
    b = O.OracleSolver(d, precision=8, Re=100.0)
    for _ in range(3):
        a.step(1e-3, 4, 2, True)
        b.step(1e-3, 4, 2, True)
    m = non_out(d)
    for fa, fb in zip(a.fields(), b.fields()):
        scale = np.max(np.abs(fb[m]))
        assert np.max(np.abs(fa[m] - fb[m])) <= 1e-5 * scale


def test_oracle_tolerance_mode_consistent():
    """The oracle's tolerance-mode step: tol = 0 runs max_global iterations and equals
    the fixed-iteration step; a loose tol stops after one; residuals shrink."""
    d = G.random_domain(16, 14, 18, seed=31, shell=True, n_obstacles=5)
    a = O.OracleSolver(d, precision=8, Re=150.0, Pr=0.72, lam=1.4)
    b = O.OracleSolver(d, precision=8, Re=150.0, Pr=0.72, lam=1.4)
    rc, it, r3 = a.step_tol(6e-4, 3, 2, 0.0, True)
    assert (rc, it) == (0, 3)
    assert b.step(6e-4, 3, 2, True) == 0
    for f in range(4):
        assert np.array_equal(a.fields(0)[f], b.fields(0)[f])
    r1 = O.OracleSolver(d, precision=8, Re=150.0, Pr=0.72, lam=1.4).step_tol(6e-4, 1, 2, 0.0, False)[2]
    r2 = O.OracleSolver(d, precision=8, Re=150.0, Pr=0.72, lam=1.4).step_tol(6e-4, 2, 2, 0.0, False)[2]
    assert r3 < r2 < r1
    e = O.OracleSolver(d, precision=8, Re=150.0, Pr=0.72, lam=1.4)
    rc, it, r = e.step_tol(6e-4, 5, 2, r1 * 1.01, False)
    assert (rc, it) == (0, 1) and r == r1
