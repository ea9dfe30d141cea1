"""Host side of the GPU mask builders: the reference's geometry inputs read the way
the reference reads them, turned into the grid-coordinate geometry that
``adi_mask_shape3d`` / ``adi_mask_sea`` / ``adi_mask_extrude2d`` rasterise on the GPU.

All geometry arithmetic here is the reference's FTYPE = float arithmetic, done in
numpy float32 scalars operation by operation, so the vertices handed to the GPU are
bit-identical to those the reference's ``Grid3D::Build`` receives:

* ``load_shape3d``   Grid3D::Load3DShape (FluidSolver3D/Grid3D.cpp:371-435): a text
  file of frames, each with vertices (position and velocity, 6 numbers a line, the
  reader of Common/IO.h:545-574) scaled by GRID_SCALE_FACTOR
  (FluidSolver2D/Grid2D.h:31), and triangles; the bounding box with 2 % padding
  (BBox3D::Build, Common/Geometry.h:510-529), the grid size (Grid3D::Init,
  Grid3D.cpp:353-358) and the conversion to grid coordinates (Grid3D.cpp:420-428).
* ``Shape3DFrames.subframe``   the frame in force at a time and the interpolation
  between it and the next (Grid3D::Prepare3D_Shape :947-964,
  ComputeSubframeInfo :900-945).
* ``sea_geometry``   the grid size and bbox.pMin.z that Grid3D::LoadNetCDF derives
  from the latitudes, longitudes and depths of a bathymetry file
  (Grid3D.cpp:437-486).  Reading the NetCDF-4 file itself needs libnetcdf, which
  libadi_b200 does not link; the caller passes the arrays.
* ``extrude_dims``   the depth levels of a 2D shape extruded in depth
  (Grid3D::LoadFromFile, Grid3D.cpp:497-509).
* ``load_shape2d`` / ``Shape2DFrames.subframe`` / ``build_shape2d``   a Shape2D file
  read as FluidSolver2D::Grid2D reads it (Grid2D.cpp:268-396) and its node grid built
  on the GPU (``adi_mask_shape2d``, Grid2D::Build); the grid feeds the 2D solver
  (``adi2d_set_grid``) or the extrusion of a 2D shape in depth (``adi_mask_extrude2d``).
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np

F = np.float32
GRID_SCALE_FACTOR = F(0.001)   # Grid2D.h:31, 0.001f
BBOX_PADDING = F(0.02)         # Geometry.h:24, converted to FTYPE where it is used
INF = F(1e10)                  # Geometry.h:22, stored in FTYPE fields
FRAME_DURATION = 1.0 / 75      # Grid3D.cpp:414, 75 frames per second

_NUM = re.compile(r"\s*[+-]?(?:\d+\.?\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?)")


def _atof(tok: str) -> float:
    """atof: the longest numeric prefix, 0.0 when there is none."""
    m = _NUM.match(tok)
    return float(m.group(0)) if m else 0.0


def _scan_int(tok: str) -> int:
    """fscanf %i: decimal, 0x hexadecimal or 0-prefixed octal."""
    t = tok.strip()
    sign = -1 if t.startswith("-") else 1
    t = t.lstrip("+-")
    if t[:2].lower() == "0x":
        return sign * int(t[2:], 16)
    if len(t) > 1 and t.startswith("0"):
        return sign * int(t, 8)
    return sign * int(t)


@dataclass
class GridBox:
    """A grid size and spacing without a node array: a handle created from it gets
    its mask from one of the GPU builders."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    def arrays(self):
        return None


@dataclass
class Frame3D:
    verts: np.ndarray        # float32 [nv, 3], grid coordinates
    vels: np.ndarray         # float32 [nv, 3]
    tris: np.ndarray         # int32 [nt, 3]
    active: bool = False
    duration: float = FRAME_DURATION


@dataclass
class Shape3DFrames:
    frames: list = field(default_factory=list)
    dims: tuple = (0, 0, 0)
    bbox_min: np.ndarray = None   # float32 [3]
    bbox_max: np.ndarray = None

    def subframe(self, time: float):
        """(verts, tris) of the shapes Grid3D::Build rasterises at `time`: the frame
        in force and the linear blend towards the next one, in float32."""
        nf = len(self.frames)
        a = [0.0]
        for f in self.frames:
            a.append(a[-1] + f.duration)
        r_time = math.fmod(time, a[nf])
        frame = 0
        for i in range(1, nf):
            if a[i] < r_time:
                frame = i
        substep = F((r_time - a[frame]) / (a[frame + 1] - a[frame]))
        f0, f1 = self.frames[frame % nf], self.frames[(frame % nf + 1) % nf]
        isub = F(1) - substep
        verts = (f0.verts * isub + f1.verts * substep).astype(F)
        if f0.active:
            return np.zeros((0, 3), F), np.zeros((0, 3), np.int32)
        return verts, f0.tris


def load_shape3d(path: str, dx: float, dy: float, dz: float) -> Shape3DFrames:
    """Grid3D::Load3DShape of a Shape3D text file (fields separated by spaces and
    newlines, as the reference's reader requires)."""
    with open(path, "r") as fh:
        toks = fh.read().split()
    pos = 0

    def nxt():
        nonlocal pos
        t = toks[pos]
        pos += 1
        return t

    def point():
        return np.array([F(_atof(nxt().replace(",", ".", 1))) for _ in range(3)], F)

    frames = []
    num_frames = _scan_int(nxt())
    for _ in range(num_frames):
        nv = _scan_int(nxt())
        verts = np.zeros((nv, 3), F)
        vels = np.zeros((nv, 3), F)
        for k in range(nv):
            p = point()
            verts[k] = p * GRID_SCALE_FACTOR
            vels[k] = point()
        ni = _scan_int(nxt())
        tris = np.array([_scan_int(nxt()) for _ in range(3 * ni)], np.int32).reshape(ni, 3)
        frames.append(Frame3D(verts, vels, tris))

    # BBox3D::Build with padding
    pmin = np.full(3, INF, F)
    pmax = np.full(3, -INF, F)
    for f in frames:
        for v in f.verts:
            for c in range(3):
                if v[c] < pmin[c]:
                    pmin[c] = v[c]
                if v[c] > pmax[c]:
                    pmax[c] = v[c]
    w = (pmax - pmin).astype(F)
    pmin = (pmin - w * BBOX_PADDING).astype(F)
    pmax = (pmax + w * BBOX_PADDING).astype(F)

    # Grid3D::Init: the float extent divided by the double spacing
    h = (dx, dy, dz)
    dims = tuple(int(math.ceil(float(F(pmax[c] - pmin[c])) / h[c])) + 1 for c in range(3))

    # physical -> grid coordinates, (v - pMin) / (FTYPE)dx
    hf = np.array([F(dx), F(dy), F(dz)], F)
    for f in frames:
        f.verts = ((f.verts - pmin) / hf).astype(F)
    return Shape3DFrames(frames, dims, pmin, pmax)


@dataclass
class Shape2D:
    points: np.ndarray       # float32 [np, 2]
    vels: np.ndarray         # float32 [np, 2]
    active: bool             # a moving shape (valve) rather than a wall


@dataclass
class Shape2DFrames:
    frames: list = field(default_factory=list)      # per frame: list of Shape2D
    durations: list = field(default_factory=list)
    dims: tuple = (0, 0)

    def subframe(self, time: float):
        """(segments [n, 8] float32: p1, p2, v1, v2; node types [n] uint8) that
        Grid2D::Build rasterises at `time` (Grid2D::Prepare and ComputeSubframe,
        Grid2D.cpp:411-477), moving shapes first, in the reference's order."""
        nf = len(self.frames)
        a = [0.0]
        for dur in self.durations:
            a.append(a[-1] + dur)
        r_time = math.fmod(time, a[nf])
        frame = 0
        for i in range(1, nf):
            if a[i] < r_time:
                frame = i
        substep = (r_time - a[frame]) / (a[frame + 1] - a[frame])
        f0, f1 = self.frames[frame % nf], self.frames[(frame % nf + 1) % nf]
        ti, ts = F(1.0 - substep), F(substep)
        shapes = []
        for s0, s1 in zip(f0, f1):
            pts = (s0.points * ti + s1.points * ts).astype(F)
            vel = (s0.vels * ti + s1.vels * ts).astype(F)
            shapes.append((pts, vel, s0.active))
        segs, kinds = [], []
        for want_active, kind in ((True, 3), (False, 2)):   # NODE_VALVE, then NODE_BOUND
            for pts, vel, active in shapes:
                if active != want_active:
                    continue
                for i in range(len(pts) - 1):
                    segs.append(np.concatenate([pts[i], pts[i + 1], vel[i], vel[i + 1]]))
                    kinds.append(kind)
        segs = np.array(segs, F).reshape(-1, 8)
        return segs, np.array(kinds, np.uint8)


def load_shape2d(path: str, dx: float, dy: float) -> Shape2DFrames:
    """Grid2D::LoadFromFile (Grid2D.cpp:268-373, no field file) of a Shape2D text
    file: frames of polylines, each passive (a wall) or moving ("Motion" and a
    velocity: a valve); the border velocities between frames
    (ComputeBorderVelocities :375-396), the bounding box with padding, the grid size
    and the grid coordinates (Grid2D::Init :197-229)."""
    with open(path, "r") as fh:
        toks = fh.read().split()
    pos = 0

    def nxt():
        nonlocal pos
        t = toks[pos]
        pos += 1
        return t

    def point():
        return np.array([F(_atof(nxt().replace(",", "."))) for _ in range(2)], F)

    frames, durations = [], []
    for _ in range(_scan_int(nxt())):
        durations.append(float(F(float(nxt()))))
        shapes = []
        for _ in range(_scan_int(nxt())):
            npt = _scan_int(nxt())
            pts = np.array([point() * GRID_SCALE_FACTOR for _ in range(npt)], F).reshape(npt, 2)
            word = nxt()
            v = point() if word.startswith("M") else np.zeros(2, F)
            shapes.append(Shape2D(pts, np.tile((v * GRID_SCALE_FACTOR).astype(F), (npt, 1)), word.startswith("M")))
        frames.append(shapes)
    nf = len(frames)
    for j in range(nf):
        nj = (j + 1) % nf
        m = F(1.0 / durations[j])
        for i, sh in enumerate(frames[j]):
            nxt_sh = frames[nj][i]
            if not sh.active:
                nxt_sh.vels = ((nxt_sh.points - sh.points) * m).astype(F)
            else:
                nxt_sh.vels = (nxt_sh.vels + (sh.points - nxt_sh.points) * m).astype(F)
    pmin = np.full(2, INF, F)
    pmax = np.full(2, -INF, F)
    for shapes in frames:
        for sh in shapes:
            for pt in sh.points:
                for c in range(2):
                    if pt[c] < pmin[c]:
                        pmin[c] = pt[c]
                    if pt[c] > pmax[c]:
                        pmax[c] = pt[c]
    w = (pmax - pmin).astype(F)
    pmin = (pmin - w * BBOX_PADDING).astype(F)
    pmax = (pmax + w * BBOX_PADDING).astype(F)
    h = (dx, dy)
    dims = tuple(int(math.ceil(float(F(pmax[c] - pmin[c])) / h[c])) + 1 for c in range(2))
    hf = np.array([F(dx), F(dy)], F)
    for shapes in frames:
        for sh in shapes:
            sh.points = ((sh.points - pmin) / hf).astype(F)
    return Shape2DFrames(frames, durations, dims)


def build_shape2d(segs, seg_types, nx: int, ny: int, start_T: float, stream=None):
    """adi_mask_shape2d: the 2D node grid (type, bc, velocity [nx, ny, 2], T) built
    on the GPU from the segments of Shape2DFrames.subframe."""
    import ctypes as C

    from . import _abi
    lib = _abi.load()
    sg = np.ascontiguousarray(segs, F).reshape(-1, 8)
    kt = np.ascontiguousarray(seg_types, np.uint8)
    t = np.zeros((nx, ny), np.uint8)
    bc = np.zeros((nx, ny), np.uint8)
    v = np.zeros((nx, ny, 2), F)
    T = np.zeros((nx, ny), F)
    handle = stream if (stream is None or isinstance(stream, int)) else getattr(stream, "cuda_stream", stream)
    _abi.check(lib.adi_mask_shape2d(sg.ctypes.data, kt.ctypes.data, len(sg), nx, ny, start_T, C.c_void_p(handle),
                                    t.ctypes.data, bc.ctypes.data, v.ctypes.data, T.ctypes.data))
    return t, bc, v, T


def sea_geometry(lats: np.ndarray, lons: np.ndarray, depth: np.ndarray, dx: float, dy: float, dz: float):
    """Grid size and bbox.pMin.z of Grid3D::LoadNetCDF for a bathymetry grid:
    depth[i + j * len(lats)] over latitude i and longitude j."""
    lats = np.asarray(lats, np.float64)
    lons = np.asarray(lons, np.float64)
    pmin = np.full(3, INF, F)
    pmax = np.full(3, -INF, F)
    for p in ((F(lats[0]), F(lons[0]), F(0)), (F(lats[-1]), F(lons[-1]), F(0))):
        for c in range(3):
            if p[c] < pmin[c]:
                pmin[c] = p[c]
            if p[c] > pmax[c]:
                pmax[c] = p[c]
    dmin = F(np.min(np.asarray(depth, F)))
    if dmin < pmin[2]:
        pmin[2] = dmin
    pmin[2] = F(pmin[2] - F(dz))
    h = (dx, dy, dz)
    dims = tuple(int(math.ceil(float(F(pmax[c] - pmin[c])) / h[c])) + 1 for c in range(3))
    return dims, float(pmin[2])


def extrude_dims(depth: float, dz: float, align: bool = False):
    """(active_nz, nz) of a 2D shape extruded to `depth` with level spacing dz."""
    active = int(math.ceil(depth / dz)) + 1
    nz = (active + 31) // 32 * 32 if align else active
    return active, nz
