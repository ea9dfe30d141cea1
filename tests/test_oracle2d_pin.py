"""The 2D restatement oracle pinned against the reference's own 2D ADI solver
(oracle/_ref/libref2d.so, compiled from its sources): float results bit for bit,
cur and next, several steps, random channels with obstacles and the configuration's
256 x 128 disc channel.  The oracle runs first and the reference only when the
oracle reports no exit condition (the reference calls exit(1) there)."""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry2d as G2

pytestmark = pytest.mark.skipif(not O.have_ref2d(), reason="reference build oracle/_ref/libref2d.so not present")


def _run_both(d, steps, dt, ng, nl, Re=100.0):
    o = O.Oracle2D(d, precision=4, Re=Re)
    r = O.Ref2D(d, Re=Re)
    for s in range(steps):
        it = o.step(dt, ng, nl)
        assert it > 0, "the reference would exit here"
        r.step(dt, ng, nl)
        for which in (0, 1):
            for a, b in zip(o.fields(which), r.fields(which)):
                assert np.array_equal(a, b), (s, which)
    return o


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_random_channels_bit_exact(seed):
    d = G2.random_domain2d(26, 18, seed=seed, n_discs=3, rmax=2.5)
    _run_both(d, 4, 1e-3, 3, 2)


def test_no_free_outflow_and_single_local_iteration():
    d = G2.random_domain2d(20, 15, seed=14, n_discs=2, rmax=2.0, outflow_free=False)
    _run_both(d, 3, 2e-3, 2, 1, Re=150.0)


def test_disc_channel_configuration():
    d = G2.channel_disc()
    o = _run_both(d, 2, 1e-3, 4, 1)
    assert o.last_err() < 0.1


def test_segments_span_obstacles():
    d = G2.channel_disc(40, 24, radius=4.0, cx=15, cy=12)
    o = O.Oracle2D(d, precision=8)
    segs = o.segments()
    cols, rows = segs[segs[:, 5] == 1], segs[segs[:, 5] == 0]
    # every interior column and row has one segment from wall to wall
    assert len(cols) == 38 and len(rows) == 22
    assert np.all(cols[:, 1] == 0) and np.all(cols[:, 3] == 23)
    assert np.all(rows[:, 0] == 0) and np.all(rows[:, 2] == 39)
