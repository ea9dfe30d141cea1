"""GPU 2D solver (adi2d_*) against the 2D restatement oracle: float and double
results bit for bit (the kernels use the reference's operand order without fused
multiply-add), global-iteration counts equal, and against the reference's own
float build where it is present."""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry2d as G2

pytestmark = pytest.mark.gpu


def _gpu(adi_lib, d, precision, Re=100.0):
    from adi_b200 import _abi
    return adi_lib.AdiSolver2D(d, Re=Re, precision=_abi.ADI_FP64 if precision == 8 else _abi.ADI_FP32)


@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("seed", [21, 22])
def test_random_channels_bit_exact(adi_lib, precision, seed):
    d = G2.random_domain2d(30, 20, seed=seed, n_discs=3, rmax=2.5)
    g = _gpu(adi_lib, d, precision)
    o = O.Oracle2D(d, precision=precision)
    for s in range(4):
        rc, it = g.step(1e-3, 3, 2)
        assert rc == 0
        assert it == o.step(1e-3, 3, 2)
        for which in (0, 1):
            for a, b in zip(g.fields(which), o.fields(which)):
                assert np.array_equal(a.astype(np.float64), b), (s, which)
    e, its = g.last_error()
    assert its == 3 and abs(e - o.last_err()) <= 1e-6 * max(o.last_err(), 1e-12)


def test_disc_channel_fp64_and_reference_float(adi_lib):
    d = G2.channel_disc()
    g = _gpu(adi_lib, d, 8)
    o = O.Oracle2D(d, precision=8)
    for s in range(3):
        rc, it = g.step(1e-3, 4, 1)
        assert rc == 0 and it == o.step(1e-3, 4, 1) == 4
    for a, b in zip(g.fields(0), o.fields(0)):
        assert np.array_equal(a, b)
    g32 = _gpu(adi_lib, d, 4)
    if O.have_ref2d():
        r = O.Ref2D(d)
        for s in range(2):
            assert g32.step(1e-3, 4, 1)[0] == 0
            r.step(1e-3, 4, 1)
        for a, b in zip(g32.fields(0), r.fields(0)):
            assert np.array_equal(a.astype(np.float64), b)


@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("case", ["disc", "random"])
def test_masked_segments_bit_exact(adi_lib, precision, case):
    """Segment mode 1 (masked segments, runs of IN nodes): GPU == restatement
    oracle in the same mode, bit for bit, iteration counts equal; switching back
    to mode 0 reproduces the reference segmentation's results."""
    d = (G2.channel_disc(48, 32, radius=5.0, cx=16, cy=16) if case == "disc" else
         G2.random_domain2d(30, 20, seed=24, n_discs=3, rmax=2.5))
    g = _gpu(adi_lib, d, precision)
    g.set_segment_mode(1)
    o = O.Oracle2D(d, precision=precision)
    o.set_segment_mode(1)
    for s in range(3):
        rc, it = g.step(1e-3, 3, 1)
        assert rc == 0
        assert it == o.step(1e-3, 3, 1)
        for which in (0, 1):
            for a, b in zip(g.fields(which), o.fields(which)):
                assert np.array_equal(a.astype(np.float64), b), (s, which)
    g.set_segment_mode(0)
    o.set_segment_mode(0)
    rc, it = g.step(1e-3, 3, 1)
    assert rc == 0 and it == o.step(1e-3, 3, 1)
    for a, b in zip(g.fields(0), o.fields(0)):
        assert np.array_equal(a.astype(np.float64), b)


@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("tol", [1e-6, 1e-2, 0.0])
def test_tolerance_mode_bit_exact(adi_lib, precision, tol):
    """adi2d_step_tol (up to 4 global iterations until the iterate changes by at
    most tol): iteration counts, residuals and fields equal to the restatement
    oracle's tolerance mode, bit for bit."""
    d = G2.channel_disc(48, 32, radius=5.0, cx=16, cy=16)
    g = _gpu(adi_lib, d, precision)
    o = O.Oracle2D(d, precision=precision)
    for s in range(4):
        rc, it, r = g.step_tol(1e-3, 4, 1, tol)
        ito, ro = o.step_tol(1e-3, 4, 1, tol)
        assert rc == 0 and it == ito and 1 <= it <= 4
        assert r == ro
        for which in (0, 1):
            for a, b in zip(g.fields(which), o.fields(which)):
                assert np.array_equal(a.astype(np.float64), b), (s, which)


def test_layer_io_and_exit_conditions(adi_lib):
    from adi_b200 import _abi
    d = G2.random_domain2d(24, 16, seed=23)
    g = _gpu(adi_lib, d, 8)
    assert g.step(1e-3, 2, 1)[0] == 0
    vel, T = g.GetLayer(12, 8)
    nxt = g.fields(1)
    for i in range(12):
        for j in range(8):
            x, y = i * 24 // 12, j * 16 // 8
            assert vel[i, j, 0] == nxt[0][x, y] and vel[i, j, 1] == nxt[1][x, y] and T[i, j] == nxt[2][x, y]
    # a wild state: the reference would exit(1); the library reports it
    u, v, t = g.fields(0)
    rng = np.random.default_rng(0)
    g.SetLayer(u + 5 * rng.standard_normal(u.shape), v + 5 * rng.standard_normal(v.shape), t)
    rc, _ = g.step(1e-3, 2, 1)
    assert rc in (_abi.ADI_ERR_DIVERGENCE, _abi.ADI_ERR_NOT_CONVERGED)
