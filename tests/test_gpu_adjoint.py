"""GPU adjoint (adi_adjoint_run) against the FP64 CPU adjoint oracle and central
finite differences.

* FP64: J to 1e-12 relative, gradients to 1e-9 of the largest entry (the GPU
  forward is the fast sweep, equal to the oracle's to ~1e-13 here).
* FP32: gradients to 1e-4 of the largest entry.
* Checkpoint windows of any length give the same bits.
* theta-gradient of the inflow profile through torch.autograd matches FP64
  central finite differences (h = 1e-3) to 1e-4 relative.
"""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G
from golden_util import fluid_params_tuple

pytestmark = pytest.mark.gpu

DT, NG, NL, STEPS = 1e-2, 2, 2, 4
RE = (150.0, 0.72, 1.4)
BOX = ((2, 2, 2), (10, 9, 11))


def _domain():
    return G.random_domain(12, 11, 13, seed=41, shell=True, n_obstacles=3, rmax=2.5)


def _gpu(adi_lib, d, precision, solver=None):
    from adi_b200 import _abi
    s = adi_lib.AdiSolver3D(d, params=adi_lib.fluid_params_normalized(*RE), precision=precision,
                            solver=_abi.ADI_SOLVER_FAST if solver is None else solver)
    s.CreateSegments()
    return s


@pytest.mark.parametrize("solver", ["fast", "exact"])
def test_fp64_adjoint_matches_oracle(adi_lib, solver):
    from adi_b200 import _abi
    d = _domain()
    s = _gpu(adi_lib, d, _abi.ADI_FP64, _abi.ADI_SOLVER_FAST if solver == "fast" else _abi.ADI_SOLVER_EXACT)
    J, gnv, gst = s.adjoint_run(DT, NG, NL, STEPS, 2, *BOX)
    o = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", RE)))
    Jo, gnvo, gsto = o.adjoint_run(DT, NG, NL, STEPS, *BOX)
    assert abs(J - Jo) <= 1e-12 * abs(Jo)
    for a, b in ((gnv, gnvo), (gst, gsto)):
        scale = np.max(np.abs(b))
        assert np.max(np.abs(a - b)) <= 1e-9 * scale
    # the handle ends at the final state
    for f in range(4):
        assert np.max(np.abs(s.fields(0)[f] - o.fields(0)[f])) <= 1e-11 * max(1.0, np.max(np.abs(o.fields(0)[f])))


def test_fp32_adjoint_and_checkpoint_windows(adi_lib):
    from adi_b200 import _abi
    d = _domain()
    o = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", RE)))
    Jo, gnvo, gsto = o.adjoint_run(DT, NG, NL, STEPS, *BOX)
    res = []
    s = _gpu(adi_lib, d, _abi.ADI_FP32)   # one handle: the same autotuned kernels for every run
    init = [a.copy() for a in s.fields(0)]
    for ck in (1, 3, STEPS):
        s.set_state(*init)
        res.append(s.adjoint_run(DT, NG, NL, STEPS, ck, *BOX))
    for J, gnv, gst in res[1:]:
        assert J == res[0][0]
        assert np.array_equal(gnv, res[0][1]) and np.array_equal(gst, res[0][2])
    J, gnv, gst = res[0]
    assert abs(J - Jo) <= 1e-5 * abs(Jo)
    for a, b in ((gnv, gnvo), (gst, gsto)):
        scale = np.max(np.abs(b))
        assert np.max(np.abs(a.astype(np.float64) - b)) <= 1e-4 * scale


def test_inflow_gradient_through_autograd_matches_finite_differences(adi_lib):
    import torch
    from adi_b200 import _abi
    from inflow_autograd import InflowEnergy, inflow_values
    d = G.spheres_channel(dims=(28, 20, 20), n_spheres=4, rmin=2.0, rmax=4.0, seed=3)
    s = _gpu(adi_lib, d, _abi.ADI_FP64)
    init = [a.copy() for a in s.fields(0)]
    run = (5e-2, 2, 2, 6, 3, (3, 5, 5), (12, 15, 15))
    theta = torch.full((16,), 0.05, dtype=torch.float64, requires_grad=True)
    J = InflowEnergy.apply(theta, s, d, init, run)
    J.backward()
    g = theta.grad.numpy().copy()
    Jv = float(J.detach())

    def J_of(th):
        t = adi_lib.AdiSolver3D(d, params=adi_lib.fluid_params_normalized(*RE), precision=_abi.ADI_FP64)
        t.CreateSegments()
        t.set_node_values(*inflow_values(d, th))
        t.set_state(*init)
        for _ in range(run[3]):
            assert t.step(run[0], run[1], run[2], False) == 0
        u = t.fields(0)
        lo, hi = run[5], run[6]
        m = np.zeros(d.shape, bool)
        m[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = True
        m &= d.type == G.NODE_IN
        return 0.5 * sum(float(np.sum(u[f][m] ** 2)) for f in range(3))

    th0 = np.full(16, 0.05)
    assert abs(J_of(th0) - Jv) <= 1e-12 * abs(Jv)
    fd = np.zeros(16)
    for m_ in range(16):
        h = 1e-3 * max(1.0, abs(th0[m_]))
        p, q = th0.copy(), th0.copy()
        p[m_] += h
        q[m_] -= h
        fd[m_] = (J_of(p) - J_of(q)) / (2 * h)
    scale = np.max(np.abs(fd))
    assert scale > 0
    assert np.max(np.abs(g - fd)) <= 1e-4 * scale, (g, fd)


@pytest.mark.parametrize("K", [0, 8, -4, -8])
def test_adjoint_sweep_variants_agree(adi_lib, K):
    """The fused chunked adjoint sweep (K = 4, 8), the split one (solve, then one
    thread per cell for the accumulations: K = -4, -8) and the one-thread-per-line
    sweep (K = 0) solve the same transposed systems: FP64 gradients agree to 1e-12."""
    from adi_b200 import _abi
    d = _domain()
    a = _gpu(adi_lib, d, _abi.ADI_FP64)
    a.set_adjoint_chunk(4)
    b = _gpu(adi_lib, d, _abi.ADI_FP64)
    for dr, (k, nl, _) in enumerate(a.fast_shapes()):
        b.set_fast_shape(dr, k, nl)          # the same forward kernels in both
    b.set_adjoint_chunk(K)
    Ja, gnva, gsta = a.adjoint_run(DT, NG, NL, STEPS, 2, *BOX)
    Jb, gnvb, gstb = b.adjoint_run(DT, NG, NL, STEPS, 2, *BOX)
    assert Ja == Jb
    for x, y in ((gnva, gnvb), (gsta, gstb)):
        assert np.max(np.abs(x - y)) <= 1e-12 * np.max(np.abs(y))
