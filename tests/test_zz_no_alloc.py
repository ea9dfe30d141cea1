"""The allocation-free sweep entry point (adi_sweep_exact_static).

It serves callers that cannot allocate device memory while they run (their device
memory is owned by their own pool, or their time loop must not pay for cudaMalloc):
they pass device arrays they own, and the sweep's elimination scratch is a fixed
static array inside the library.  These tests drive it through the C ABI on
torch-owned device buffers and check it against the existing handle-based entry
point (adi_step with the exact solver), which runs the same arithmetic: results
must be identical, over two consecutive time steps, and a repeated call must not
see the previous call's scratch contents, in float and in double.  A caller-owned
mask is not checked the way adi_set_mask checks one, so the kernel skips any line
whose rows would read outside the arrays; a padded-buffer case checks that.  This
file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from adi_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(torch.device("cuda"), dtype=dtype)


class StaticRunner:
    """One domain's buffers on the device, stepped only with adi_sweep_exact_static."""

    def __init__(self, adi_lib, d, Re, Pr, lam, precision=None):
        import torch
        from adi_b200 import _abi
        self.abi, self.lib, self.d = _abi, _abi.load(), d
        self.precision = _abi.ADI_FP32 if precision is None else precision
        fdt = torch.float64 if self.precision == _abi.ADI_FP64 else torch.float32
        self.params = adi_lib.fluid_params_normalized(Re, Pr, lam)
        self.ntype, self.bcv, self.bct = (_dev(a, torch.uint8) for a in (d.type, d.bc_vel, d.bc_temp))
        self.nv = [_dev(a, fdt) for a in (d.vx, d.vy, d.vz, d.T)]
        self.cur = [x.clone() for x in self.nv]          # initial state = node values
        self.nxt = [torch.zeros_like(x) for x in self.nv]
        self.half = [torch.zeros_like(x) for x in self.nv]
        self.ta = [torch.zeros_like(x) for x in self.nv]
        self.tb = [torch.zeros_like(x) for x in self.nv]
        self.bv = (self.ntype == G.NODE_BOUND) | (self.ntype == G.NODE_VALVE)

    def sweep(self, direction, src, tin, dst, tout, merges, dt):
        import torch
        a = self.abi.StaticSweepArgs()
        a.dir = direction
        a.dimx, a.dimy, a.dimz = self.d.shape
        a.dx, a.dy, a.dz, a.dt = self.d.dx, self.d.dy, self.d.dz, dt
        a.params = self.params
        a.precision = self.precision
        a.merges = merges
        a.node_type, a.bc_vel, a.bc_temp = self.ntype.data_ptr(), self.bcv.data_ptr(), self.bct.data_ptr()
        for v in range(4):
            a.node_value[v] = self.nv[v].data_ptr()
            a.cur[v] = src[v].data_ptr()
            a.temp_in[v] = tin[v].data_ptr()
            a.next[v] = dst[v].data_ptr()
            a.temp_out[v] = tout[v].data_ptr()
        a.stream = torch.cuda.current_stream().cuda_stream
        return self.lib.adi_sweep_exact_static(C.byref(a))

    def step(self, dt, num_global, num_local):
        """UpdateBoundaries + TimeStep with the exact path's schedule."""
        for v in range(4):
            self.cur[v][self.bv] = self.nv[v][self.bv]
            self.nxt[v][self.bv] = self.cur[v][self.bv]
            self.ta[v].copy_(self.cur[v])
            self.tb[v].copy_(self.cur[v])
        for _ in range(num_global):
            for direction, src, dst in ((2, self.cur, self.nxt), (1, self.nxt, self.half), (0, self.half, self.nxt)):
                for l in range(num_local):
                    merges = 2 if (direction == 0 and l == num_local - 1) else 1
                    assert self.sweep(direction, src, self.ta, dst, self.tb, merges, dt) == 0
                    self.ta, self.tb = self.tb, self.ta
        self.cur, self.nxt = self.nxt, self.cur

    def fields(self):
        import torch
        torch.cuda.synchronize()
        return [x.cpu().numpy() for x in self.cur]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_static_sweep_matches_handle_path_two_steps(adi_lib, precision):
    from adi_b200 import _abi
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    d = G.random_domain(30, 26, 34, seed=91, shell=True, n_obstacles=6, rmax=4.0)
    Re, Pr, lam, dt, ng, nl = 140.0, 0.72, 1.4, 8e-4, 3, 2
    ref = adi_lib.AdiSolver3D(d, Re=Re, Pr=Pr, lam=lam, precision=prec, solver=_abi.ADI_SOLVER_EXACT)
    ref.CreateSegments()
    run = StaticRunner(adi_lib, d, Re, Pr, lam, precision=prec)
    m = d.type != G.NODE_OUT
    for step in range(2):
        assert ref.step(dt, ng, nl, False) == 0
        run.step(dt, ng, nl)
        want, got = ref.fields(0), run.fields()
        for f in range(4):
            assert np.array_equal(got[f][m], want[f][m]), (step, f)   # same arithmetic: bit for bit


def test_static_sweep_repeat_ignores_previous_scratch(adi_lib):
    import torch
    d = G.random_domain(28, 24, 20, seed=92, n_obstacles=5, rmax=3.5)
    run = StaticRunner(adi_lib, d, 120.0, 0.72, 1.4)
    for v in range(4):
        run.ta[v].copy_(run.cur[v])
    outs = []
    for rep in range(2):
        for v in range(4):
            run.nxt[v].zero_()
            run.tb[v].zero_()
        assert run.sweep(0, run.cur, run.ta, run.nxt, run.tb, 1, 1e-3) == 0
        torch.cuda.synchronize()
        outs.append([x.cpu().numpy().copy() for x in run.nxt + run.tb])
        # another domain in between leaves different contents in the shared scratch
        other = StaticRunner(adi_lib, G.random_domain(40, 18, 22, seed=93), 90.0, 0.72, 1.4)
        for v in range(4):
            other.ta[v].copy_(other.cur[v])
        assert other.sweep(1, other.cur, other.ta, other.nxt, other.tb, 2, 2e-3) == 0
        torch.cuda.synchronize()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_static_sweep_rejects_lines_beyond_scratch(adi_lib, precision):
    from adi_b200 import _abi
    lib = _abi.load()
    prec, es = (_abi.ADI_FP64, 8) if precision == "fp64" else (_abi.ADI_FP32, 4)
    limit = lib.adi_static_scratch_bytes() // (6 * 128 * es)   # longest line: 5461 float, 2730 double
    d = G.empty_domain(limit + 8, 3, 3)
    run = StaticRunner(adi_lib, d, 100.0, 0.72, 1.4, precision=prec)
    assert run.sweep(0, run.cur, run.ta, run.nxt, run.tb, 1, 1e-3) == 2   # ADI_ERR_CAPACITY
    small = StaticRunner(adi_lib, G.empty_domain(limit, 3, 3), 100.0, 0.72, 1.4, precision=prec)
    assert small.sweep(0, small.cur, small.ta, small.nxt, small.tb, 1, 1e-3) == 0


def test_static_sweep_skips_lines_that_break_the_contract(adi_lib):
    """NODE_IN cells where the solver contract forbids them (at the end of a line, on
    the outer frame) would make rows read outside the arrays; the kernel skips those
    lines.  Every array sits inside a larger allocation padded with sentinels, so a
    stray read would stay in bounds and show up, and a stray write would change the
    padding."""
    import torch
    d = G.random_domain(24, 20, 22, seed=94, shell=True, n_obstacles=4, rmax=3.0)
    nx, ny, nz = d.shape
    j0, k0 = 9, 11               # X line (j0, k0): NODE_IN at its first node
    i1, k1 = 12, 7               # cell (i1, 0, k1) on the face y = 0: NODE_IN
    bad = G.Domain(nx, ny, nz, d.dx, d.dy, d.dz, d.type.copy(), d.bc_vel, d.bc_temp, d.vx, d.vy, d.vz, d.T)
    bad.type[0, j0, k0] = G.NODE_IN
    bad.type[i1, 0, k1] = G.NODE_IN
    n, pad = nx * ny * nz, 2 * ny * nz + 64
    sentinel = 7.0

    def padded(a, dtype, fill):
        buf = torch.full((n + 2 * pad,), fill, dtype=dtype, device="cuda")
        buf[pad:pad + n] = torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda", dtype)
        return buf, buf[pad:pad + n].view(nx, ny, nz)

    run = StaticRunner(adi_lib, bad, 120.0, 0.72, 1.4)
    bufs = {}
    run.ntype = padded(bad.type, torch.uint8, G.NODE_OUT)[1]
    run.bcv = padded(bad.bc_vel, torch.uint8, G.BC_NOSLIP)[1]
    run.bct = padded(bad.bc_temp, torch.uint8, G.BC_NOSLIP)[1]
    for name in ("nv", "cur", "ta", "nxt", "tb"):
        pairs = [padded(x.cpu().numpy() if name in ("nv", "cur", "ta") else np.full(bad.shape, sentinel),
                        torch.float32, float("nan") if name in ("nv", "cur", "ta") else sentinel)
                 for x in (run.cur if name == "ta" else getattr(run, name))]
        bufs[name] = [p[0] for p in pairs]
        setattr(run, name, [p[1] for p in pairs])
    for direction in range(3):
        for v in range(4):
            run.nxt[v].fill_(sentinel)
            run.tb[v].fill_(sentinel)
        assert run.sweep(direction, run.cur, run.ta, run.nxt, run.tb, 1, 1e-3) == 0
        torch.cuda.synchronize()
        for v in range(4):
            out = run.nxt[v].cpu().numpy()
            assert np.all(np.isfinite(out)), (direction, v)           # nothing read the NaN padding
            for name in ("nxt", "tb"):
                whole = bufs[name][v].cpu().numpy()
                assert np.all(whole[:pad] == sentinel) and np.all(whole[pad + n:] == sentinel)
            if direction == 0:
                assert np.all(out[:, j0, k0] == sentinel)               # first node NODE_IN: skipped
                assert np.all(out[:, 0, k1] == sentinel)                # line on the face y = 0: skipped
            elif direction == 1:
                assert np.all(out[i1, :, k1] == sentinel)               # first node NODE_IN: skipped
            else:
                assert np.all(out[i1, 0, :] == sentinel)                # line on the face y = 0: skipped
        # the sweep did run elsewhere
        assert np.any(run.nxt[0].cpu().numpy() != sentinel)
