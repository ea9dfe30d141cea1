"""One domain split over several solvers: X slabs, with the X sweeps solved on Y pencils.

The reference splits a domain over GPUs into X slabs and runs a pipelined
distributed Thomas across them (``AdiSolver3D.cu:523-881``, ``TimeLayer3D.h:158-247``;
``MGPU_EMU`` in ``Common/GPUplan.h:10-15`` emulates the GPUs on one device).  Here
every tridiagonal line is solved whole on one solver, so the result equals the
single-domain step bit for bit:

* part s holds the X slab x in [x0_s, x1_s) (all y, z) plus one ghost x-plane on
  each inner side, coded NODE_BOUND so that no line there has a row.  Y and Z
  lines lie inside a slab; their sweeps read the nonlinear layer one plane beyond
  (the off-line stencil of the advecting component), so the ghost planes of that
  layer are refreshed from the neighbouring slabs after every sweep;
* for the X sweeps the layers the sweep reads and writes are moved ("transposed")
  to Y pencils -- part r holds y in [y0_r, y1_r) for every x, plus ghost y-planes --
  the X sweeps run there on complete lines, the ghost y-planes of the nonlinear
  layer refreshed between local iterations, and the results move back;
* the divergence error is the sum over the slabs' IN cells divided by their count.

A step goes through the handles' step phases (``adi_phase_*``): begin, the sweeps
one at a time, end.  The parts run either in one process on one device
(``comm=None``: the reference's emulation mode; block moves are device copies) or
one part per rank of a ``torch.distributed`` process group (block moves are
point-to-point sends; NCCL over NVLink between GPUs, gloo between CPU processes in
the tests of the move plan).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from . import geometry as G

ROLE_CUR, ROLE_NEXT, ROLE_HALF, ROLE_TEMP_IN, ROLE_TEMP_OUT = 0, 1, 2, 3, 4


def _split(n: int, parts: int):
    """Balanced split of range(n) into `parts` contiguous ranges."""
    edges = [(n * p) // parts for p in range(parts + 1)]
    return [(edges[p], edges[p + 1]) for p in range(parts)]


@dataclass(frozen=True)
class SlabPlan:
    """Owned and stored ranges of the X slabs and the Y pencils of an nx x ny x nz
    domain split into `parts` parts.  Stored ranges add one ghost plane on each
    inner side."""
    nx: int
    ny: int
    nz: int
    parts: int

    def __post_init__(self):
        if self.parts < 1 or self.parts > min(self.nx, self.ny) // 3:
            raise ValueError("each slab and pencil needs at least three planes")

    def slab(self, s: int):
        """(x0, x1, lo, hi): owned x range and stored x range of slab s."""
        x0, x1 = _split(self.nx, self.parts)[s]
        return x0, x1, max(0, x0 - 1), min(self.nx, x1 + 1)

    def pencil(self, r: int):
        """(y0, y1, lo, hi): owned y range and stored y range of pencil r."""
        y0, y1 = _split(self.ny, self.parts)[r]
        return y0, y1, max(0, y0 - 1), min(self.ny, y1 + 1)


def _local_domain(d: G.Domain, sl, ghost_mask) -> G.Domain:
    """The sub-domain d[sl] with the cells where ghost_mask is set coded NODE_BOUND
    (no line through them has a row; their values come from the owning part)."""
    t = np.ascontiguousarray(d.type[sl]).copy()
    t[ghost_mask] = G.NODE_BOUND
    sub = G.Domain(*t.shape, d.dx, d.dy, d.dz, t,
                   *[np.ascontiguousarray(getattr(d, a)[sl]) for a in ("bc_vel", "bc_temp", "vx", "vy", "vz", "T")])
    sub.meta.update(d.meta)
    return sub


def slab_domain(d: G.Domain, plan: SlabPlan, s: int) -> G.Domain:
    x0, x1, lo, hi = plan.slab(s)
    ghost = np.zeros((hi - lo, d.ny, d.nz), bool)
    if x0 > lo:
        ghost[0] = True
    if x1 < hi:
        ghost[-1] = True
    return _local_domain(d, np.s_[lo:hi], ghost)


def pencil_domain(d: G.Domain, plan: SlabPlan, r: int) -> G.Domain:
    y0, y1, lo, hi = plan.pencil(r)
    ghost = np.zeros((d.nx, hi - lo, d.nz), bool)
    if y0 > lo:
        ghost[:, 0] = True
    if y1 < hi:
        ghost[:, -1] = True
    return _local_domain(d, np.s_[:, lo:hi], ghost)


# ---------------------------------------------------------------------------
# block moves between parts
# ---------------------------------------------------------------------------

class LocalComm:
    """Every part in this process (one device): a move is a set of copies."""

    def __init__(self, parts: int):
        self.parts = parts
        self.mine = list(range(parts))

    def move(self, transfers):
        """transfers: (src_part, dst_part, src_block, dst_block) with src_block() the
        source view and dst_block() the destination view of the same shape."""
        for _, _, src, dst in transfers:
            dst().copy_(src())

    def allreduce_sum(self, values):
        return [float(v) for v in values]


class DistComm:
    """One part per rank of the default torch.distributed group: blocks whose two
    ends are on different ranks travel as one packed message per rank pair
    (batch_isend_irecv; NCCL between GPUs, gloo between CPU processes)."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist
        self.parts = dist.get_world_size()
        self.rank = dist.get_rank()
        self.mine = [self.rank]

    def move(self, transfers):
        import torch
        dist = self.dist
        out, inc = {}, {}
        for sp, dp, src, dst in transfers:
            if sp == self.rank and dp == self.rank:
                dst().copy_(src())
            elif sp == self.rank:
                out.setdefault(dp, []).append(src)
            elif dp == self.rank:
                inc.setdefault(sp, []).append(dst)
        ops, recv = [], []
        for peer, blocks in sorted(out.items()):
            buf = torch.cat([b().reshape(-1) for b in blocks])
            ops.append(dist.P2POp(dist.isend, buf, peer))
        for peer, blocks in sorted(inc.items()):
            views = [b() for b in blocks]
            buf = torch.empty(sum(v.numel() for v in views), dtype=views[0].dtype, device=views[0].device)
            ops.append(dist.P2POp(dist.irecv, buf, peer))
            recv.append((buf, views))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for buf, views in recv:
            o = 0
            for v in views:
                v.copy_(buf[o:o + v.numel()].view(v.shape))
                o += v.numel()

    def allreduce_sum(self, values):
        import torch
        t = torch.tensor(values, dtype=torch.float64)
        if self.dist.get_backend() == "nccl":
            t = t.cuda()
        self.dist.all_reduce(t)
        return [float(v) for v in t.cpu()]


class SlabMoves:
    """The block moves of the decomposition over per-part field arrays.
    slab_fields(s, role) / pencil_fields(r, role) return the four field arrays
    (U, V, W, T; shape = the part's stored dims) of a role on the part's owner."""

    def __init__(self, plan: SlabPlan, comm, slab_fields, pencil_fields):
        self.plan, self.comm = plan, comm
        self.sf, self.pf = slab_fields, pencil_fields

    def slab_halo(self, role):
        """Ghost x-planes of every slab from the neighbouring slabs' owned planes."""
        P, tr = self.plan, []
        for s in range(P.parts):
            x0, x1, lo, hi = P.slab(s)
            for v in range(4):
                if x0 > lo:
                    nlo = P.slab(s - 1)[2]
                    tr.append((s - 1, s, lambda s=s, v=v, a=x0 - 1 - nlo: self.sf(s - 1, role)[v][a],
                               lambda s=s, v=v: self.sf(s, role)[v][0]))
                if x1 < hi:
                    nlo = P.slab(s + 1)[2]
                    tr.append((s + 1, s, lambda s=s, v=v, a=x1 - nlo: self.sf(s + 1, role)[v][a],
                               lambda s=s, v=v, e=hi - lo - 1: self.sf(s, role)[v][e]))
        self.comm.move(tr)

    def pencil_halo(self, role):
        """Ghost y-planes of every pencil from the neighbouring pencils."""
        P, tr = self.plan, []
        for r in range(P.parts):
            y0, y1, lo, hi = P.pencil(r)
            for v in range(4):
                if y0 > lo:
                    nlo = P.pencil(r - 1)[2]
                    tr.append((r - 1, r, lambda r=r, v=v, a=y0 - 1 - nlo: self.pf(r - 1, role)[v][:, a],
                               lambda r=r, v=v: self.pf(r, role)[v][:, 0]))
                if y1 < hi:
                    nlo = P.pencil(r + 1)[2]
                    tr.append((r + 1, r, lambda r=r, v=v, a=y1 - nlo: self.pf(r + 1, role)[v][:, a],
                               lambda r=r, v=v, e=hi - lo - 1: self.pf(r, role)[v][:, e]))
        self.comm.move(tr)

    def to_pencils(self, roles):
        """Slab layers -> pencil layers: every pencil's stored y range (ghosts
        included) of every slab's owned x range.  roles: (slab role, pencil role)."""
        P, tr = self.plan, []
        for s in range(P.parts):
            x0, x1, slo, _ = P.slab(s)
            for r in range(P.parts):
                _, _, plo, phi = P.pencil(r)
                for rs, rp in roles:
                    for v in range(4):
                        tr.append((s, r, lambda s=s, v=v, rs=rs, a=x0 - slo, b=x1 - slo, c=plo, e=phi:
                                   self.sf(s, rs)[v][a:b, c:e],
                                   lambda r=r, v=v, rp=rp, a=x0, b=x1: self.pf(r, rp)[v][a:b]))
        self.comm.move(tr)

    def to_slabs(self, roles):
        """Pencil layers -> slab layers: every pencil's owned y range of every
        slab's owned x range.  roles: (pencil role, slab role)."""
        P, tr = self.plan, []
        for r in range(P.parts):
            y0, y1, plo, _ = P.pencil(r)
            for s in range(P.parts):
                x0, x1, slo, _ = P.slab(s)
                for rp, rs in roles:
                    for v in range(4):
                        tr.append((r, s, lambda r=r, v=v, rp=rp, a=x0, b=x1, c=y0 - plo, e=y1 - plo:
                                   self.pf(r, rp)[v][a:b, c:e],
                                   lambda s=s, v=v, rs=rs, a=x0 - slo, b=x1 - slo, c=y0, e=y1:
                                   self.sf(s, rs)[v][a:b, c:e]))
        self.comm.move(tr)


# ---------------------------------------------------------------------------
# the split solver
# ---------------------------------------------------------------------------

class _DeviceArray:
    """A device array of the library (a role's field) as a torch tensor view."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class SlabSolver:
    """A domain stepped as `parts` X slabs (Y and Z sweeps) and Y pencils (X
    sweeps), each an AdiSolver3D handle; see the module docstring.  With comm=None
    every part lives in this process on the current device; with a DistComm the
    part of this rank does.  Each step equals AdiSolver3D.step on the whole domain
    with the same sweep shapes, bit for bit."""

    def __init__(self, domain: G.Domain, parts: int, comm=None, shapes=None, **solver_kw):
        import torch
        from . import AdiSolver3D
        self.plan = SlabPlan(domain.nx, domain.ny, domain.nz, parts)
        self.comm = comm if comm is not None else LocalComm(parts)
        if self.comm.parts != parts:
            raise ValueError("one part per rank")
        self.stream = torch.cuda.current_stream()
        kw = dict(solver_kw)
        kw["stream"] = self.stream.cuda_stream
        self.slabs = {s: AdiSolver3D(slab_domain(domain, self.plan, s), **kw) for s in self.comm.mine}
        self.pencils = {r: AdiSolver3D(pencil_domain(domain, self.plan, r), **kw) for r in self.comm.mine}
        # slabs run the Y and Z sweeps, pencils the X sweeps: shapes go where they run
        for h, dirs in [(h, (1, 2)) for h in self.slabs.values()] + [(h, (0,)) for h in self.pencils.values()]:
            h.CreateSegments()
            if shapes:
                for dr in dirs:
                    h.set_fast_shape(dr, *shapes[dr])
        any_h = next(iter(self.slabs.values()))
        self.dtype = any_h.dtype
        self.lib = any_h.lib
        self.diff_error = 0.0
        self.moves = SlabMoves(self.plan, self.comm, self._slab_fields, self._pencil_fields)

    # -- device views of the handles' layers --
    def _fields(self, h, role):
        import torch
        arr = (C.c_void_p * 4)()
        _abi.check(self.lib.adi_role_pointers(h.h, role, C.byref(arr)), h.h)
        ts = "<f8" if self.dtype == np.float64 else "<f4"
        return [torch.as_tensor(_DeviceArray(arr[v], h.shape, ts), device="cuda") for v in range(4)]

    def _slab_fields(self, s, role):
        return self._fields(self.slabs[s], role)

    def _pencil_fields(self, r, role):
        return self._fields(self.pencils[r], role)

    def _each(self, parts, fn, *args):
        for h in parts.values():
            _abi.check(fn(h.h, *args), h.h)

    def step(self, dt, num_global, num_local, compute_error=False) -> int:
        """UpdateBoundaries + TimeStep over the parts; returns the status (0 = OK,
        ADI_ERR_DIVERGENCE when the divergence error exceeds 0.01, layers unswapped)."""
        lib, mv = self.lib, self.moves
        self._each(self.slabs, lib.adi_phase_begin, 1)
        mv.slab_halo(ROLE_TEMP_IN)   # the step start gave the ghost planes node values
        for _ in range(num_global):
            for dr in (2, 1):
                for _ in range(num_local):
                    self._each(self.slabs, lib.adi_phase_sweep, dr, dt, 1)
                    mv.slab_halo(ROLE_TEMP_IN)   # the layer the sweep wrote, read next
            mv.to_pencils([(ROLE_HALF, ROLE_HALF), (ROLE_TEMP_IN, ROLE_TEMP_IN), (ROLE_NEXT, ROLE_NEXT),
                           (ROLE_TEMP_OUT, ROLE_TEMP_OUT)])
            for l in range(num_local):
                self._each(self.pencils, lib.adi_phase_sweep, 0, dt, 2 if l == num_local - 1 else 1)
                if l < num_local - 1:
                    mv.pencil_halo(ROLE_TEMP_IN)
            mv.to_slabs([(ROLE_NEXT, ROLE_NEXT), (ROLE_TEMP_IN, ROLE_TEMP_IN)])
            mv.slab_halo(ROLE_TEMP_IN)
        if compute_error:
            mv.slab_halo(ROLE_NEXT)   # the divergence stencil reads the plane below
            ssum, scnt = 0.0, 0
            for h in self.slabs.values():
                a, b = C.c_double(), C.c_uint64()
                _abi.check(lib.adi_phase_div_sum(h.h, ROLE_NEXT, C.byref(a), C.byref(b)), h.h)
                ssum += a.value
                scnt += b.value
            ssum, scnt = self.comm.allreduce_sum([ssum, scnt])
            self.diff_error = ssum / scnt if scnt else 0.0
        if self.diff_error > 0.01:
            return _abi.ADI_ERR_DIVERGENCE
        self._each(self.slabs, lib.adi_phase_end)
        return 0

    def div_error(self) -> float:
        return self.diff_error

    def fields(self):
        """The state of the parts in this process, assembled as [4][nx, ny, nz]
        arrays (regions of parts elsewhere are left zero)."""
        P = self.plan
        out = [np.zeros((P.nx, P.ny, P.nz), self.dtype) for _ in range(4)]
        for s, h in self.slabs.items():
            x0, x1, lo, _ = P.slab(s)
            f = h.fields(0)
            for v in range(4):
                out[v][x0:x1] = f[v][x0 - lo:x1 - lo]
        return out

    def close(self):
        for h in list(self.slabs.values()) + list(self.pencils.values()):
            h.close()
