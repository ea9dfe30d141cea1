"""Synthetic masked domains for the 3D ADI solver.

A domain is the reference's ``Grid3D`` node array flattened to structure-of-arrays
(``Grid3D.h:73-88``: ``Node{type, bc_vel, bc_temp, v, T}``), all ``[i][j][k]`` with
``k`` fastest, exactly the order ``Grid3D::GetType`` indexes (``Grid3D.cpp:242-245``).

Node types and boundary codes follow ``Common/Geometry.h:31-41``:
``NODE_IN=0, NODE_OUT=1, NODE_BOUND=2, NODE_VALVE=3``; ``BC_NOSLIP=0, BC_FREE=1``.

The reference builds its masks with rasterisers and flood fill (``Grid3D.cpp:608-1075``);
those loaders are outside the solver's hot path, so domains arrive here pre-built.
Every generator is seeded and deterministic.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NODE_IN, NODE_OUT, NODE_BOUND, NODE_VALVE = 0, 1, 2, 3
BC_NOSLIP, BC_FREE = 0, 1


@dataclass
class Domain:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    type: np.ndarray      # uint8 [nx, ny, nz]
    bc_vel: np.ndarray    # uint8
    bc_temp: np.ndarray   # uint8
    vx: np.ndarray        # float64 node values (boundary data and initial state)
    vy: np.ndarray
    vz: np.ndarray
    T: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    def arrays(self):
        """Contiguous arrays in ABI order: type, bc_vel, bc_temp, vx, vy, vz, T."""
        out = [np.ascontiguousarray(a, dtype=np.uint8) for a in (self.type, self.bc_vel, self.bc_temp)]
        out += [np.ascontiguousarray(a, dtype=np.float64) for a in (self.vx, self.vy, self.vz, self.T)]
        return out

    def round_values_to_float32(self) -> "Domain":
        """Node values are FTYPE in the reference (Grid3D.h:77-78); rounding them to
        float32 makes a float run and a double run see the same boundary data."""
        for name in ("vx", "vy", "vz", "T"):
            setattr(self, name, getattr(self, name).astype(np.float32).astype(np.float64))
        return self


def empty_domain(nx: int, ny: int, nz: int, h: float | None = None, baseT: float = 1.0) -> Domain:
    """All-fluid box with a one-cell BOUND no-slip frame at rest (v = 0, T = baseT)."""
    if h is None:
        h = 1.0 / (max(nx, ny, nz) - 1)
    shape = (nx, ny, nz)
    t = np.full(shape, NODE_IN, np.uint8)
    t[0, :, :] = t[-1, :, :] = NODE_BOUND
    t[:, 0, :] = t[:, -1, :] = NODE_BOUND
    t[:, :, 0] = t[:, :, -1] = NODE_BOUND
    return Domain(nx, ny, nz, h, h, h, t,
                  np.zeros(shape, np.uint8), np.zeros(shape, np.uint8),
                  np.zeros(shape), np.zeros(shape), np.zeros(shape), np.full(shape, baseT))


def set_channel_ends(d: Domain, inflow_u: float = 1.0, inflow_T: float = 1.0) -> Domain:
    """x = 0 plane: Dirichlet inflow u = inflow_u; x = nx-1 plane: BC_FREE outflow."""
    d.vx[0, 1:-1, 1:-1] = inflow_u
    d.T[0, :, :] = inflow_T
    d.bc_vel[-1, 1:-1, 1:-1] = BC_FREE
    d.bc_temp[-1, 1:-1, 1:-1] = BC_FREE
    return d


def _carve_solid(d: Domain, solid: np.ndarray, T_solid: float, shell: bool) -> None:
    """Turns interior cells in `solid` into no-slip walls at rest.

    shell=False: every solid cell is NODE_BOUND.  shell=True: solid cells whose 26
    neighbours are all solid become NODE_OUT, the rest NODE_BOUND, so no fluid cell
    has an OUT cell anywhere in its 3x3x3 neighbourhood.  (The sweeps read the six
    face neighbours of fluid cells; the divergence error also reads the diagonal
    corners, TimeLayer3D.h:614-621, and the reference leaves OUT values of its
    work layers uninitialised.)  The outer frame keeps its own data."""
    inner = np.zeros_like(solid)
    inner[1:-1, 1:-1, 1:-1] = solid[1:-1, 1:-1, 1:-1]
    d.type[inner] = NODE_BOUND
    d.bc_vel[inner] = BC_NOSLIP
    d.bc_temp[inner] = BC_NOSLIP
    d.vx[inner] = 0.0
    d.vy[inner] = 0.0
    d.vz[inner] = 0.0
    d.T[inner] = T_solid
    if shell:
        s = solid
        full = np.zeros_like(s)
        core = np.ones(tuple(n - 2 for n in s.shape), bool)
        for di in (0, 1, 2):
            for dj in (0, 1, 2):
                for dk in (0, 1, 2):
                    core &= s[di:di + s.shape[0] - 2, dj:dj + s.shape[1] - 2, dk:dk + s.shape[2] - 2]
        full[1:-1, 1:-1, 1:-1] = core
        d.type[full & inner] = NODE_OUT


def spheres_mask(shape, centres, radii) -> np.ndarray:
    nx, ny, nz = shape
    solid = np.zeros(shape, bool)
    for c, r in zip(centres, radii):
        lo = np.maximum(np.floor(c - r).astype(int), 0)
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, shape)
        if np.any(hi <= lo):
            continue
        i, j, k = np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]), np.arange(lo[2], hi[2]), indexing="ij")
        inside = (i - c[0]) ** 2 + (j - c[1]) ** 2 + (k - c[2]) ** 2 <= r * r
        solid[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= inside
    return solid


def ellipsoids_mask(shape, centres, semi_axes) -> np.ndarray:
    solid = np.zeros(shape, bool)
    for c, ax in zip(centres, semi_axes):
        lo = np.maximum(np.floor(c - ax).astype(int), 0)
        hi = np.minimum(np.ceil(c + ax).astype(int) + 1, shape)
        if np.any(hi <= lo):
            continue
        i, j, k = np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]), np.arange(lo[2], hi[2]), indexing="ij")
        inside = ((i - c[0]) / ax[0]) ** 2 + ((j - c[1]) / ax[1]) ** 2 + ((k - c[2]) / ax[2]) ** 2 <= 1.0
        solid[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= inside
    return solid


def spheres_channel(n: int = 128, n_spheres: int = 40, rmin: float = 4.0, rmax: float = 12.0,
                    seed: int = 0, inflow_u: float = 1.0, T_solid: float = 1.2, shell: bool = True,
                    dims=None) -> Domain:
    """Plain 3D forward workload: an n^3 box (h = 1/(n-1)) with `n_spheres` solid
    spheres, radii U[rmin, rmax] and centres U[0, n)^3 from default_rng(seed); inflow
    u = inflow_u on x = 0, BC_FREE outflow on x = n-1, no-slip walls elsewhere."""
    dims = tuple(dims) if dims is not None else (n, n, n)
    d = empty_domain(*dims, h=1.0 / (max(dims) - 1))
    set_channel_ends(d, inflow_u)
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, np.array(dims, float), size=(n_spheres, 3))
    radii = rng.uniform(rmin, rmax, size=n_spheres)
    _carve_solid(d, spheres_mask(dims, centres, radii), T_solid, shell)
    d.meta.update(kind="spheres_channel", n_spheres=n_spheres, seed=seed)
    return d


def batch_of_domains(n_domains: int = 64, seed: int = 2, size_lo: int = 64, size_hi: int = 160,
                     spheres=(10, 60), rmin: float = 4.0, rmax: float = 12.0, re=(50.0, 400.0)):
    """Batched workload: n_domains independent sphere channels, each axis uniform in
    {size_lo..size_hi}, a sphere count uniform in spheres[0]..spheres[1] (radii
    U[rmin, rmax]), Reynolds number U[re]; all drawn from default_rng(seed).  Each
    domain's Re is in its meta["Re"]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_domains):
        dims = tuple(int(x) for x in rng.integers(size_lo, size_hi + 1, size=3))
        ns = int(rng.integers(spheres[0], spheres[1] + 1))
        Re = float(rng.uniform(*re))
        sub = int(rng.integers(0, 2**31 - 1))
        d = spheres_channel(dims=dims, n_spheres=ns, rmin=rmin, rmax=rmax, seed=sub)
        d.meta.update(kind="batch_member", Re=Re)
        out.append(d)
    return out


def ellipsoids_tube(n: int = 384, n_ellipsoids: int = 300, amin: float = 3.0, amax: float = 20.0,
                    seed: int = 1, inflow_u: float = 1.0, T_solid: float = 1.2, shell: bool = True) -> Domain:
    """Large 3D workload: n^3 box with `n_ellipsoids` solid ellipsoids (semi-axes
    U[amin, amax]^3, centres U[0, n)^3, default_rng(seed)) plus a thin-walled
    internal tube along x (2-cell wall, open ends) that the ellipsoids do not enter."""
    d = empty_domain(n, n, n)
    set_channel_ends(d, inflow_u)
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, n, size=(n_ellipsoids, 3))
    axes = rng.uniform(amin, amax, size=(n_ellipsoids, 3))
    solid = ellipsoids_mask(d.shape, centres, axes)
    # tube: axis along x through (cy, cz), inner radius ri, wall thickness 2 cells
    cy = cz = (n - 1) / 2.0
    ri = n / 8.0
    j, k = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    r = np.sqrt((j - cy) ** 2 + (k - cz) ** 2)
    wall2d = (r >= ri) & (r < ri + 2.0)
    bore2d = r < ri
    x0, x1 = n // 8, n - n // 8
    solid[:, bore2d] = False
    solid[x0:x1, wall2d] = True
    _carve_solid(d, solid, T_solid, shell)
    d.meta.update(kind="ellipsoids_tube", n_ellipsoids=n_ellipsoids, seed=seed)
    return d


def random_domain(nx: int, ny: int, nz: int, seed: int, n_obstacles: int = 6, rmax: float = 3.0,
                  shell: bool = False, free_outflow: bool = True, valves: bool = True,
                  perturb: float = 0.3) -> Domain:
    """Small randomised domain for parity tests: random spheres, random wall data,
    a random smooth-ish initial state so every term of the scheme is exercised."""
    rng = np.random.default_rng(seed)
    d = empty_domain(nx, ny, nz)
    set_channel_ends(d, inflow_u=float(rng.uniform(0.5, 1.5)))
    if not free_outflow:
        d.bc_vel[-1] = BC_NOSLIP
        d.bc_temp[-1] = BC_NOSLIP
    centres = rng.uniform(0, np.array([nx, ny, nz], float), size=(n_obstacles, 3))
    radii = rng.uniform(1.0, rmax, size=n_obstacles)
    _carve_solid(d, spheres_mask(d.shape, centres, radii), float(rng.uniform(0.8, 1.5)), shell)
    if valves:
        # a few VALVE cells on the y = 0 wall with a small inflow
        jj = rng.integers(1, nz - 1, size=3)
        ii = rng.integers(1, nx - 1, size=3)
        for i, k in zip(ii, jj):
            d.type[i, 0, k] = NODE_VALVE
            d.vy[i, 0, k] = float(rng.uniform(0.1, 0.5))
    fluid = d.type == NODE_IN
    for name, scale in (("vx", perturb), ("vy", perturb), ("vz", perturb), ("T", 0.2)):
        a = getattr(d, name)
        a[fluid] += scale * rng.standard_normal(int(fluid.sum()))
    d.round_values_to_float32()
    return d


def validate_for_solver(d: Domain, strict_div: bool = False) -> str | None:
    """Returns None when the solver contract holds, else the reason.

    The contract (the reference relies on the same; its stencils read +-1 without
    bounds checks, TimeLayer3D.h:256-259,338-343):
      * no IN cell on the outer frame;
      * no IN cell has an OUT 6-neighbour;
      * a non-IN cell between two IN cells along an axis has no BC_FREE code
        (the two segments meeting there would disagree).
    strict_div additionally asks that no IN cell has an OUT cell among its 26
    neighbours, which makes the divergence error independent of OUT values."""
    t = d.type
    if strict_div:
        inn = t == NODE_IN
        out = np.pad(t == NODE_OUT, 1)
        nx, ny, nz = t.shape
        for di in (0, 1, 2):
            for dj in (0, 1, 2):
                for dk in (0, 1, 2):
                    if np.any(inn & out[di:di + nx, dj:dj + ny, dk:dk + nz]):
                        return "IN cell with an OUT cell among its 26 neighbours"
    frame = np.zeros(t.shape, bool)
    frame[0] = frame[-1] = True
    frame[:, 0] = frame[:, -1] = True
    frame[:, :, 0] = frame[:, :, -1] = True
    if np.any((t == NODE_IN) & frame):
        return "IN cell on the outer frame"
    fin = t == NODE_IN
    out = t == NODE_OUT
    for ax in range(3):
        a = np.moveaxis(fin, ax, 0)
        o = np.moveaxis(out, ax, 0)
        if np.any(a[1:] & o[:-1]) or np.any(a[:-1] & o[1:]):
            return "IN cell next to an OUT cell"
        free = np.moveaxis((d.bc_vel == BC_FREE) | (d.bc_temp == BC_FREE), ax, 0)
        if np.any(a[:-2] & a[2:] & ~np.moveaxis(fin, ax, 0)[1:-1] & free[1:-1]):
            return "BC_FREE cell shared by two segments"
    return None
