"""Synthetic geometry inputs for the mask-builder tests, written in the reference's
input formats: Shape3D text files (Grid3D::Load3DShape, FluidSolver3D/Grid3D.cpp:371-435),
Shape2D text files (Grid2D::LoadFromFile, FluidSolver2D/Grid2D.cpp:268-320) and
bathymetry depth maps.  Every shape here is made up for the tests; coordinates are
in the files' units (scaled by 0.001 on loading)."""
from __future__ import annotations

import math

import numpy as np


def _fmt(x: float) -> str:
    return repr(float(x))


def write_shape3d(path: str, frames) -> None:
    """frames: list of (verts [nv, 3], tris [nt, 3], vels [nv, 3] or None)."""
    lines = [str(len(frames))]
    for verts, tris, vels in frames:
        verts = np.asarray(verts, np.float64)
        vels = np.zeros_like(verts) if vels is None else np.asarray(vels, np.float64)
        lines.append(str(len(verts)))
        for p, v in zip(verts, vels):
            lines.append(" ".join(_fmt(c) for c in p) + " " + " ".join(_fmt(c) for c in v))
        lines.append(str(len(tris)))
        for t in tris:
            lines.append(" ".join(str(int(i)) for i in t))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def tetra():
    v = [(120.0, 80.0, 60.0), (880.0, 140.0, 90.0), (300.0, 760.0, 110.0), (420.0, 300.0, 690.0)]
    t = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
    return np.array(v), np.array(t)


def box(lo=(0.0, 0.0, 0.0), hi=(730.0, 510.0, 640.0), drop_faces=0):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = [(x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0), (x1, y0, z0), (x1, y0, z1), (x1, y1, z1),
         (x1, y1, z0)]
    t = [(0, 1, 2), (0, 2, 3), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (3, 2, 6), (3, 6, 7), (0, 4, 7),
         (0, 7, 3), (1, 5, 6), (1, 6, 2)]
    return np.array(v), np.array(t[:len(t) - 2 * drop_faces])


def uv_sphere(center=(500.0, 480.0, 510.0), radius=360.0, n_lat=9, n_lon=14, jitter=9.0, seed=0):
    """A closed latitude-longitude sphere with jittered vertices (triangles of every
    orientation)."""
    rng = np.random.default_rng(seed)
    cx, cy, cz = center
    verts = [(cx, cy, cz + radius)]
    for a in range(1, n_lat):
        th = math.pi * a / n_lat
        for b in range(n_lon):
            ph = 2 * math.pi * b / n_lon
            verts.append((cx + radius * math.sin(th) * math.cos(ph), cy + radius * math.sin(th) * math.sin(ph),
                          cz + radius * math.cos(th)))
    verts.append((cx, cy, cz - radius))
    verts = np.array(verts) + rng.uniform(-jitter, jitter, (len(verts), 3))
    top, bot = 0, len(verts) - 1
    ring = lambda a, b: 1 + (a - 1) * n_lon + (b % n_lon)
    tris = []
    for b in range(n_lon):
        tris.append((top, ring(1, b), ring(1, b + 1)))
        tris.append((bot, ring(n_lat - 1, b + 1), ring(n_lat - 1, b)))
    for a in range(1, n_lat - 1):
        for b in range(n_lon):
            tris.append((ring(a, b), ring(a + 1, b), ring(a + 1, b + 1)))
            tris.append((ring(a, b), ring(a + 1, b + 1), ring(a, b + 1)))
    return verts, np.array(tris)


def moved(verts, shift=(40.0, -25.0, 30.0)):
    return np.asarray(verts) + np.asarray(shift)


def depth_map(dnx=64, dny=50, seed=3, open_far=False):
    """A basin: land (positive) along the borders, water (negative) inside, smooth
    bumps on the floor and an island.  open_far: the sea reaches the far borders
    x = max and y = max (where the reference puts its inflow/outflow valves)."""
    rng = np.random.default_rng(seed)
    x = np.linspace(-1.0, 1.0, dnx)[:, None]
    y = np.linspace(-1.0, 1.0, dny)[None, :]
    d = -40.0 * (1.0 - x * x) * (1.0 - y * y) + 6.0
    if open_far:
        d -= 30.0 / (1.0 + np.exp(-(x - 0.75) / 0.06)) + 30.0 / (1.0 + np.exp(-(y - 0.75) / 0.06))
    for _ in range(5):
        cx, cy = rng.uniform(-0.6, 0.6, 2)
        d += rng.uniform(-8.0, 8.0) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / 0.05)
    d += 30.0 * np.exp(-((x - 0.25) ** 2 + (y + 0.2) ** 2) / 0.01)   # island
    return d.astype(np.float32)


def write_shape2d(path: str, shapes, duration=10.0, frames=None) -> None:
    """shapes: list of (points [np, 2], velocity or None); a velocity makes the
    shape a moving wall or valve ("Motion"), None a passive wall.  frames: a list
    of (duration, shapes) for several frames instead (the same shapes, moved)."""
    frames = frames if frames is not None else [(duration, shapes)]
    lines = [str(len(frames))]
    for dur, shp in frames:
        lines += [_fmt(dur), str(len(shp))]
        for pts, vel in shp:
            lines.append(str(len(pts)))
            for p in pts:
                lines.append(f"{_fmt(p[0])} {_fmt(p[1])}")
            if vel is None:
                lines.append("Passive")
            else:
                lines.append("Motion")
                lines.append(f"{_fmt(vel[0])} {_fmt(vel[1])}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def channel2d():
    """A channel with an inflow valve on the left, an outflow valve on the right
    and a triangular obstacle."""
    return [
        (np.array([(0.0, 0.0), (1000.0, 0.0)]), None),
        (np.array([(1000.0, 420.0), (0.0, 420.0)]), None),
        (np.array([(0.0, 0.0), (0.0, 420.0)]), (1000.0, 0.0)),
        (np.array([(1000.0, 0.0), (1000.0, 420.0)]), (0.0, 0.0)),
        (np.array([(380.0, 150.0), (470.0, 210.0), (390.0, 280.0), (380.0, 150.0)]), None),
    ]


def channel2d_moving():
    """Two frames of a channel whose obstacle moves down and to the right, with a
    moving valve segment on the lower wall."""
    f0 = channel2d()
    f1 = [(pts if i != 4 else pts + np.array([60.0, -35.0]), vel) for i, (pts, vel) in enumerate(channel2d())]
    valve = (np.array([(600.0, 0.0), (700.0, 0.0)]), (0.0, 250.0))
    return [(0.5, f0 + [valve]), (0.7, f1 + [(valve[0] + np.array([20.0, 0.0]), valve[1])])]
