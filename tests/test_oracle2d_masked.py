"""Masked-segment mode of the 2D restatement oracle (segment mode 1): the 3D
solver's segmentation applied to the 2D grid's rows and columns.  The reference has
no such mode, so it is checked through its structure and through the reference
mode it must reduce to: with no solid cell inside the box the two modes build the
same segments and give bit-identical fields."""
import numpy as np

import oracle as O
from adi_b200 import geometry2d as G2


def _coverage(d, segs):
    """Per direction: times each node is an interior row of a segment."""
    nx, ny = d.shape
    cover = {0: np.zeros((nx, ny), int), 1: np.zeros((nx, ny), int)}
    for px, py, ex, ey, size, dr in segs:
        if dr == 0:
            assert py == ey and ex - px + 1 == size
            cover[0][px + 1:ex, py] += 1
            ends = [(px, py), (ex, ey)]
        else:
            assert px == ex and ey - py + 1 == size
            cover[1][px, py + 1:ey] += 1
            ends = [(px, py), (ex, ey)]
        for (i, j) in ends:
            assert d.type[i, j] != G2.NODE_IN
    return cover


def test_masked_segments_are_runs_of_in_nodes():
    d = G2.channel_disc(40, 24, radius=4.0, cx=15, cy=12)
    o = O.Oracle2D(d, precision=8)
    n = o.set_segment_mode(1)
    segs = o.segments()
    assert len(segs) == n
    cover = _coverage(d, segs)
    fluid = d.type == G2.NODE_IN
    for dr in (0, 1):
        # every IN node is an interior row of exactly one segment per direction,
        # and no interior row is a solid node
        assert np.array_equal(cover[dr] == 1, fluid) and cover[dr].max() == 1
    # columns through the disc hold two segments, the others one
    cols = segs[segs[:, 5] == 1]
    per_col = np.bincount(cols[:, 0], minlength=40)
    assert per_col[15] == 2 and per_col[5] == 1 and per_col[0] == 0


def test_masked_equals_reference_mode_without_obstacles():
    d = G2.random_domain2d(28, 18, seed=31, n_discs=0)
    a = O.Oracle2D(d, precision=8)
    b = O.Oracle2D(d, precision=8)
    b.set_segment_mode(1)
    assert np.array_equal(a.segments(), b.segments())
    for _ in range(3):
        assert a.step(1e-3, 3, 2) == b.step(1e-3, 3, 2) > 0
    for x, y in zip(a.fields(0), b.fields(0)):
        assert np.array_equal(x, y)


def test_masked_mode_with_obstacles_runs_and_differs():
    d = G2.channel_disc(48, 32, radius=5.0, cx=16, cy=16)
    a = O.Oracle2D(d, precision=8)
    b = O.Oracle2D(d, precision=8)
    b.set_segment_mode(1)
    for _ in range(3):
        assert a.step(1e-3, 4, 1) > 0 and b.step(1e-3, 4, 1) > 0
    fa, fb = a.fields(0), b.fields(0)
    fluid = d.type == G2.NODE_IN
    assert all(np.all(np.isfinite(f)) for f in fb)
    # solid interior rows no longer take part: the fluid solution changes
    assert max(float(np.max(np.abs(x[fluid] - y[fluid]))) for x, y in zip(fa, fb)) > 0
    # switching back restores the reference segmentation
    b.set_segment_mode(0)
    assert np.array_equal(a.segments(), b.segments())


def test_tolerance_mode_restatement():
    """Tolerance mode of the 2D restatement: tol = 0 runs max_global iterations and
    equals the reference-mode step wherever that one stops at num_global (error
    below 0.1); a huge tol stops after one iteration; the residual falls with the
    iterations."""
    d = G2.random_domain2d(26, 18, seed=33, n_discs=2, rmax=2.0)
    a = O.Oracle2D(d, precision=8)
    b = O.Oracle2D(d, precision=8)
    for _ in range(2):
        it = a.step(1e-3, 3, 1)
        assert it == 3 and a.last_err() <= 0.1
        itb, r = b.step_tol(1e-3, 3, 1, 0.0)
        assert itb == 3 and r > 0
    for x, y in zip(a.fields(0), b.fields(0)):
        assert np.array_equal(x, y)
    c = O.Oracle2D(d, precision=8)
    assert c.step_tol(1e-3, 4, 1, 1e9)[0] == 1
    rs = []
    for m in (1, 2, 3, 4):
        e = O.Oracle2D(d, precision=8)
        rs.append(e.step_tol(1e-3, m, 1, 0.0)[1])
    assert rs[-1] < rs[0]
