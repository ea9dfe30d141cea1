"""Synthetic 2D domains for the 2D ADI solver (the reference's Grid2D node data:
cell type, BC type, velocity, temperature per node; FluidSolver2D/Grid2D.h:31-45).

Arrays are [i][j] with j fastest (Grid2D::GetData, Grid2D.cpp:55-58)."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NODE_IN, NODE_OUT, NODE_BOUND, NODE_VALVE = 0, 1, 2, 3
BC_NOSLIP, BC_FREE = 0, 1


@dataclass
class Domain2D:
    nx: int
    ny: int
    dx: float
    dy: float
    type: np.ndarray     # uint8 NodeType
    bct: np.ndarray      # uint8 BCtype of the node data
    vx: np.ndarray       # float64 node velocity x
    vy: np.ndarray       # float64 node velocity y
    T: np.ndarray        # float64 node temperature
    startT: float = 1.0
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return (self.nx, self.ny)

    @property
    def cells(self) -> int:
        return self.nx * self.ny


def channel_disc(nx: int = 256, ny: int = 128, radius: float = 12.0, cx: float = 64.0, cy: float = 64.0,
                 u_max: float = 1.0, T0: float = 1.0) -> Domain2D:
    """Channel with a disc obstacle: walls y = 0 and y = ny-1 and the disc are
    no-slip BOUND nodes at rest; x = 0 is a Dirichlet inflow u(y) = 4 u_max y'(1-y'),
    y' = j/(ny-1); x = nx-1 is a BC_FREE outflow; T = T0 everywhere.  The spacing
    is 1/128 for the 256 x 128 channel, 1/(ny-1) otherwise."""
    h = 1.0 / 128.0 if (nx, ny) == (256, 128) else 1.0 / (ny - 1)
    t = np.full((nx, ny), NODE_IN, np.uint8)
    bct = np.zeros((nx, ny), np.uint8)
    vx = np.zeros((nx, ny))
    vy = np.zeros((nx, ny))
    T = np.full((nx, ny), T0)
    t[:, 0] = t[:, -1] = NODE_BOUND
    t[0, :] = NODE_BOUND
    t[-1, :] = NODE_BOUND
    yp = np.arange(ny) / (ny - 1)
    vx[0, :] = 4.0 * u_max * yp * (1.0 - yp)
    bct[-1, 1:-1] = BC_FREE
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    disc = (ii - cx) ** 2 + (jj - cy) ** 2 <= radius * radius
    t[disc] = NODE_BOUND
    vx[disc] = 0.0
    vy[disc] = 0.0
    return Domain2D(nx, ny, h, h, t, bct, vx, vy, T, T0, meta={"kind": "channel_disc", "radius": radius})


def random_domain2d(nx: int, ny: int, seed: int, n_discs: int = 2, rmax: float = 3.0, perturb: float = 0.02,
                    outflow_free: bool = True) -> Domain2D:
    """Small randomised channel for parity tests: random discs, a perturbed initial
    velocity in the fluid (the node data of IN nodes are the initial state)."""
    rng = np.random.default_rng(seed)
    d = channel_disc(nx, ny, radius=0.0, cx=-10, cy=-10, u_max=float(rng.uniform(0.5, 1.5)))
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    for _ in range(n_discs):
        cx, cy = rng.uniform(3, nx - 3), rng.uniform(3, ny - 3)
        r = rng.uniform(1.0, rmax)
        disc = (ii - cx) ** 2 + (jj - cy) ** 2 <= r * r
        disc[0, :] = disc[-1, :] = False
        d.type[disc] = NODE_BOUND
        d.vx[disc] = 0.0
        d.vy[disc] = 0.0
    if not outflow_free:
        d.bct[-1, :] = BC_NOSLIP
    fluid = d.type == NODE_IN
    d.vx[fluid] += perturb * rng.standard_normal(int(fluid.sum()))
    d.vy[fluid] += perturb * rng.standard_normal(int(fluid.sum()))
    d.T[fluid] += 0.1 * rng.standard_normal(int(fluid.sum()))
    for a in (d.vx, d.vy, d.T):
        a[...] = a.astype(np.float32).astype(np.float64)
    return d
