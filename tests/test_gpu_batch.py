"""GPU checks of batched stepping (adi_batch_*).

A batch runs every member through the generic chunked sweep with the batch's
chunk length K and lines-per-CTA max(1, 256 // P), or, for X and Y with K < 0, the
tile kernel with element-copied tiles of 8 lines, so each member must come out bit
for bit as the same domain stepped alone with that fast-sweep shape; one member is
also compared with the FP64 oracle at float tolerance (2e-6 of the field scale).
The member-graph schedule runs each member's own step on concurrent graph
branches, so it must equal each member's adi_step bit for bit.
"""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G
from golden_util import fluid_params_tuple, non_out

pytestmark = pytest.mark.gpu


def _domains(seed, n=5, lo=18, hi=44):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        dims = tuple(int(x) for x in rng.integers(lo, hi + 1, size=3))
        d = G.random_domain(*dims, seed=seed * 100 + q, shell=bool(q % 2), n_obstacles=4, rmax=3.5)
        d.meta["Re"] = float(rng.uniform(60.0, 300.0))
        out.append(d)
    return out


def _member(adi_lib, d, solver=None, precision=None):
    from adi_b200 import _abi
    fp = adi_lib.fluid_params_normalized(d.meta["Re"], 0.72, 1.4)
    s = adi_lib.AdiSolver3D(d, params=fp, precision=precision or _abi.ADI_FP32,
                            solver=_abi.ADI_SOLVER_EXACT if solver is None else solver)
    s.CreateSegments()
    return s


def _alone(adi_lib, d, K):
    """The same domain stepped by itself with the batch's sweep shape per direction:
    the generic kernel with chunks of K rows and max(1, 256 // P) lines per CTA, or
    for K < 0 the X/Y tile kernel with element-copied tiles and chunks of -K rows."""
    from adi_b200 import _abi
    s = _member(adi_lib, d, solver=_abi.ADI_SOLVER_FAST)
    for dr in range(3):
        if K[dr] < 0:
            s.set_fast_shape(dr, -K[dr], -1)
            continue
        P = -(-d.shape[dr] // K[dr])
        s.set_fast_shape(dr, K[dr], max(1, 256 // P))
    return s


@pytest.mark.parametrize("K", [(4, 4, 4), (8, 8, 8), (4, 8, 4), (-4, -4, 4), (-5, -5, 8)])
def test_batch_matches_members_stepped_alone(adi_lib, K):
    ds = _domains(7)
    members = [_member(adi_lib, d) for d in ds]
    b = adi_lib.AdiBatch(members)
    for dr in range(3):
        b.set_chunk(dr, K[dr])
    assert b.chunks() == list(K)
    alone = [_alone(adi_lib, d, K) for d in ds]
    for i in range(4):
        ce = i in (0, 3)           # the last step's errors are those of the final state
        assert b.step(6e-4, 2, 2, ce) == 0, b.last_error()
        for s in alone:
            assert s.step(6e-4, 2, 2, ce) == 0
    for q, (m, s) in enumerate(zip(members, alone)):
        for f in range(4):
            assert np.array_equal(m.fields(0)[f], s.fields(0)[f]), (q, f)
    errs = b.div_errors()
    for q, s in enumerate(alone):
        # same cells, summed in a different block order
        assert abs(errs[q] - s.div_error()) <= 1e-12 * max(1.0, abs(errs[q]))


def test_batch_member_against_oracle(adi_lib):
    ds = _domains(8, n=3)
    members = [_member(adi_lib, d) for d in ds]
    b = adi_lib.AdiBatch(members)
    orc = O.OracleSolver(ds[1], precision=8, params=fluid_params_tuple(("normalized", (ds[1].meta["Re"], 0.72, 1.4))))
    for i in range(3):
        assert b.step(7e-4, 3, 2, True) == 0
        assert orc.step(7e-4, 3, 2, True) == 0
    m = non_out(ds[1])
    got, want = members[1].fields(0), orc.fields(0)
    vs = max(np.max(np.abs(want[f][m])) for f in range(3))
    for f in range(4):
        scale = vs if f < 3 else np.max(np.abs(want[3][m]))
        assert np.max(np.abs(got[f][m].astype(np.float64) - want[f][m])) / scale < 2e-6, f
    assert abs(b.div_errors()[1] - orc.div_error()) < 1e-6


def test_batch_graph_replay_and_autotune(adi_lib):
    ds = _domains(9, n=4)
    ma = [_member(adi_lib, d) for d in ds]
    mb = [_member(adi_lib, d) for d in ds]
    a, b = adi_lib.AdiBatch(ma), adi_lib.AdiBatch(mb)
    a.autotune(6e-4, 2)
    assert all(k in (4, 8, -4, -5) for k in a.chunks()) and a.chunks()[2] > 0
    for dr, k in enumerate(a.chunks()):
        b.set_chunk(dr, k)
    b.set_graphs(False)
    l0a, l0b = a.launches(), b.launches()
    for i in range(5):
        assert a.step(6e-4, 2, 2, i == 4) == b.step(6e-4, 2, 2, i == 4) == 0
    for x, y in zip(ma, mb):
        for f in range(4):
            assert np.array_equal(x.fields(0)[f], y.fields(0)[f])
    assert a.launches() - l0a == b.launches() - l0b == 5 * (1 + 2 * 2 * 3) + 2


def test_batch_divergence_guard_and_lock_step(adi_lib):
    from adi_b200 import _abi
    ds = _domains(10, n=3)
    members = [_member(adi_lib, d) for d in ds]
    b = adi_lib.AdiBatch(members)
    before = [m.fields(0) for m in members]
    # a wild state in one member trips its divergence guard: nobody advances
    rng = np.random.default_rng(0)
    wild = [(a + 100.0 * rng.standard_normal(a.shape)).astype(np.float32) for a in members[2].fields(0)]
    members[2].set_state(*wild)
    assert b.step(6e-4, 1, 1, True) == _abi.ADI_ERR_DIVERGENCE
    assert b.div_errors()[2] > 0.01
    for m, f0 in zip(members[:2], before[:2]):
        for f in range(4):
            assert np.array_equal(m.fields(0)[f], f0[f])
    # a member stepped on its own leaves the batch out of lock step
    members[2].set_state(*before[2])
    members[2].step(6e-4, 1, 1, True)
    assert b.step(6e-4, 1, 1, False) == _abi.ADI_ERR_STATE
    # mixed precisions cannot form a batch
    m64 = _member(adi_lib, ds[0], precision=_abi.ADI_FP64)
    with pytest.raises(_abi.AdiError):
        adi_lib.AdiBatch([members[0], m64])


@pytest.mark.parametrize("branches", [1, 2, 3])
def test_member_graph_schedule_matches_members_stepped_alone(adi_lib, branches):
    """ADI_BATCH_MEMBER_GRAPHS runs each member's own step (its fast kernels and
    shapes) on concurrent graph branches: bit for bit the member's adi_step."""
    from adi_b200 import _abi
    ds = _domains(11, n=6)
    members = [_member(adi_lib, d, solver=_abi.ADI_SOLVER_FAST) for d in ds]
    alone = [_member(adi_lib, d, solver=_abi.ADI_SOLVER_FAST) for d in ds]
    for m, s in zip(members, alone):
        for dr, (K, NL, _) in enumerate(m.fast_shapes()):
            s.set_fast_shape(dr, K, NL)
    b = adi_lib.AdiBatch(members)
    b.set_schedule(_abi.ADI_BATCH_MEMBER_GRAPHS, branches)
    assert b.schedule() == (_abi.ADI_BATCH_MEMBER_GRAPHS, branches)
    for graphs in (True, False):
        b.set_graphs(graphs)
        for i in range(3):
            ce = i in (0, 2)
            assert b.step(6e-4, 2, 2, ce) == 0, b.last_error()
            for s in alone:
                assert s.step(6e-4, 2, 2, ce) == 0
        for q, (m, s) in enumerate(zip(members, alone)):
            for f in range(4):
                assert np.array_equal(m.fields(0)[f], s.fields(0)[f]), (graphs, q, f)
        assert np.array_equal(b.div_errors(), np.array([s.div_error() for s in alone]))


def test_member_graph_divergence_guard_and_autotune(adi_lib):
    from adi_b200 import _abi
    ds = _domains(12, n=4)
    members = [_member(adi_lib, d, solver=_abi.ADI_SOLVER_FAST) for d in ds]
    b = adi_lib.AdiBatch(members)
    b.autotune(6e-4, 2)
    sched, br = b.schedule()
    assert sched in (_abi.ADI_BATCH_PERSISTENT, _abi.ADI_BATCH_MEMBER_GRAPHS) and 1 <= br <= 4
    # timing steps did not advance anything: a step after autotune equals one without
    ref = [_member(adi_lib, d, solver=_abi.ADI_SOLVER_FAST) for d in ds]
    b.set_schedule(_abi.ADI_BATCH_MEMBER_GRAPHS, 2)
    for m, s in zip(members, ref):
        for dr, (K, NL, _) in enumerate(m.fast_shapes()):
            s.set_fast_shape(dr, K, NL)
    assert b.time_step(6e-4, 1, 2, 2) > 0
    assert b.step(6e-4, 2, 2, True) == 0
    for s in ref:
        assert s.step(6e-4, 2, 2, True) == 0
    for m, s in zip(members, ref):
        for f in range(4):
            assert np.array_equal(m.fields(0)[f], s.fields(0)[f])
    # a wild member trips the guard; nobody advances (the boundary update at the
    # step start has been applied, as a driver's UpdateBoundaries before a throwing
    # TimeStep would, so fluid cells are compared)
    before = [m.fields(0) for m in members]
    rng = np.random.default_rng(1)
    wild = [(a + 100.0 * rng.standard_normal(a.shape)).astype(np.float32) for a in members[1].fields(0)]
    members[1].set_state(*wild)
    assert b.step(6e-4, 1, 1, True) == _abi.ADI_ERR_DIVERGENCE
    assert b.div_errors()[1] > 0.01
    for q in (0, 2, 3):
        fluid = ds[q].type == G.NODE_IN
        for f in range(4):
            assert np.array_equal(members[q].fields(0)[f][fluid], before[q][f][fluid])
    with pytest.raises(_abi.AdiError):
        b.set_schedule(_abi.ADI_BATCH_MEMBER_GRAPHS, 5)


@pytest.mark.parametrize("schedule", ["member", "persistent"])
def test_batch_step_io_time_march_equals_separate_calls(adi_lib, schedule):
    """adi_batch_step_io chained through host buffers equals, member by member,
    set_state + the batch step + get_state, in both schedules."""
    import torch
    from adi_b200 import _abi
    ds = _domains(13, n=5)
    a_m = [_member(adi_lib, d, solver=_abi.ADI_SOLVER_FAST) for d in ds]
    b_m = [_member(adi_lib, d, solver=_abi.ADI_SOLVER_FAST) for d in ds]
    for m, s in zip(a_m, b_m):
        for dr, (K, NL, _) in enumerate(m.fast_shapes()):
            s.set_fast_shape(dr, K, NL)
    a, b = adi_lib.AdiBatch(a_m), adi_lib.AdiBatch(b_m)
    for bb in (a, b):
        if schedule == "member":
            bb.set_schedule(_abi.ADI_BATCH_MEMBER_GRAPHS, 2)
        for dr in range(3):
            bb.set_chunk(dr, 4)
    pin = [[[torch.empty(d.shape, dtype=torch.float32, pin_memory=True).numpy() for _ in range(4)]
            for d in ds] for _ in range(2)]
    for q, m in enumerate(a_m):
        for x, y in zip(pin[0][q], m.fields(0)):
            x[...] = y
    state = [[x.copy() for x in pin[0][q]] for q in range(len(ds))]
    src, dst = 0, 1
    for i in range(3):
        assert a.step_io(pin[src], pin[dst], 6e-4, 2, 2, i in (0, 2)) == 0, a.last_error()
        src, dst = dst, src
    a.io_wait()
    for i in range(3):
        for q, m in enumerate(b_m):
            m.set_state(*state[q])
        assert b.step(6e-4, 2, 2, i in (0, 2)) == 0, b.last_error()
        state = [[x.copy() for x in m.fields(0)] for m in b_m]
    for q in range(len(ds)):
        for f in range(4):
            assert np.array_equal(pin[src][q][f], state[q][f]), (q, f)
    assert np.array_equal(a.div_errors(), b.div_errors())
