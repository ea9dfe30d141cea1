"""The allocation-free sweep entry point (adi_sweep_exact_static).

It serves callers that cannot allocate device memory while they run (their device
memory is owned by their own pool, or their time loop must not pay for cudaMalloc):
they pass device arrays they own, and the sweep's elimination scratch is a fixed
static array inside the library.  These tests drive it through the C ABI on
torch-owned device buffers and check it against the existing handle-based entry
point (adi_step with the exact solver), which runs the same arithmetic: results
must be identical, over two consecutive time steps, and a repeated call must not
see the previous call's scratch contents.  This file is collected last on purpose.
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

    def __init__(self, adi_lib, d, Re, Pr, lam):
        import torch
        from adi_b200 import _abi
        self.abi, self.lib, self.d = _abi, _abi.load(), d
        self.params = adi_lib.fluid_params_normalized(Re, Pr, lam)
        self.ntype, self.bcv, self.bct = (_dev(a, torch.uint8) for a in (d.type, d.bc_vel, d.bc_temp))
        self.nv = [_dev(a, torch.float32) for a in (d.vx, d.vy, d.vz, d.T)]
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
        a.precision = self.abi.ADI_FP32
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


def test_static_sweep_matches_handle_path_two_steps(adi_lib):
    from adi_b200 import _abi
    d = G.random_domain(30, 26, 34, seed=91, shell=True, n_obstacles=6, rmax=4.0)
    Re, Pr, lam, dt, ng, nl = 140.0, 0.72, 1.4, 8e-4, 3, 2
    ref = adi_lib.AdiSolver3D(d, Re=Re, Pr=Pr, lam=lam, solver=_abi.ADI_SOLVER_EXACT)
    ref.CreateSegments()
    run = StaticRunner(adi_lib, d, Re, Pr, lam)
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


def test_static_sweep_rejects_lines_beyond_scratch(adi_lib):
    from adi_b200 import _abi
    lib = _abi.load()
    limit = lib.adi_static_scratch_bytes() // (6 * 128 * 4)   # longest float line
    d = G.empty_domain(limit + 8, 3, 3)
    run = StaticRunner(adi_lib, d, 100.0, 0.72, 1.4)
    assert run.sweep(0, run.cur, run.ta, run.nxt, run.tb, 1, 1e-3) == 2   # ADI_ERR_CAPACITY
    small = StaticRunner(adi_lib, G.empty_domain(limit, 3, 3), 100.0, 0.72, 1.4)
    assert small.sweep(0, small.cur, small.ta, small.nxt, small.tb, 1, 1e-3) == 0
