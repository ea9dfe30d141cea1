"""The FP64 CPU adjoint (oracle) against central finite differences of the FP64
oracle forward: node-value gradients at inflow, wall and outflow nodes, initial-
state gradients at fluid cells.  Tolerance 1e-6 relative to the largest gradient
entry checked (central differences with h = 1e-5 are accurate to ~1e-9 here)."""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G

DT, NG, NL, STEPS = 1e-2, 2, 2, 4
PARAMS = dict(Re=150.0, Pr=0.72, lam=1.4)


def _domain():
    d = G.random_domain(12, 11, 13, seed=41, shell=True, n_obstacles=3, rmax=2.5)
    assert G.validate_for_solver(d) is None
    return d


def _J(d, box, nv=None, state=None):
    s = O.OracleSolver(d, precision=8, **PARAMS)
    if nv is not None:
        s.set_node_values(*nv)
    if state is not None:
        s.set_state(*state)
    for _ in range(STEPS):
        assert s.step(DT, NG, NL, False) == 0
    u = s.fields(0)
    m = np.zeros(d.shape, bool)
    m[box[0][0]:box[1][0], box[0][1]:box[1][1], box[0][2]:box[1][2]] = True
    m &= d.type == G.NODE_IN
    return 0.5 * sum(float(np.sum(u[f][m] ** 2)) for f in range(3))


def test_adjoint_matches_finite_differences():
    d = _domain()
    box = ((2, 2, 2), (10, 9, 11))
    s = O.OracleSolver(d, precision=8, **PARAMS)
    J, gnv, gst = s.adjoint_run(DT, NG, NL, STEPS, box[0], box[1])
    assert abs(J - _J(d, box)) <= 1e-12 * abs(J)
    nv0 = [a.copy() for a in (d.vx, d.vy, d.vz, d.T)]
    eps = 1e-4
    checks = []
    # node values: inflow u, a wall node's v, the temperature of an inflow node
    fluid = np.argwhere(d.type == G.NODE_IN)
    bound = np.argwhere((d.type == G.NODE_BOUND) & (np.arange(d.nx)[:, None, None] > 0))
    for (f, idx) in [(0, (0, 5, 6)), (0, (0, 3, 9)), (1, tuple(bound[len(bound) // 2])), (3, (0, 6, 4))]:
        plus = [a.copy() for a in nv0]
        minus = [a.copy() for a in nv0]
        plus[f][idx] += eps
        minus[f][idx] -= eps
        fd = (_J(d, box, nv=plus) - _J(d, box, nv=minus)) / (2 * eps)
        checks.append((gnv[f][idx], fd))
    # initial state at fluid cells
    st0 = s.fields(0)
    s2 = O.OracleSolver(d, precision=8, **PARAMS)
    init = s2.fields(0)
    for (f, q) in [(0, 3), (1, len(fluid) // 2), (3, len(fluid) - 5)]:
        idx = tuple(fluid[q])
        plus = [a.copy() for a in init]
        minus = [a.copy() for a in init]
        plus[f][idx] += eps
        minus[f][idx] -= eps
        fd = (_J(d, box, state=plus) - _J(d, box, state=minus)) / (2 * eps)
        checks.append((gst[f][idx], fd))
    scale = max(abs(fd) for _, fd in checks)
    assert scale > 0
    for ad, fd in checks:
        assert abs(ad - fd) <= 1e-6 * scale, checks
    del st0
