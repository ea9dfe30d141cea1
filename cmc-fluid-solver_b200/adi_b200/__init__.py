"""Python front end of the B200 3D ADI step (ctypes over include/adi_b200.h).

``AdiSolver3D`` mirrors the reference's ``Solver3D``/``AdiSolver3D`` surface
(``FluidSolver3D/Solver3D.h:24-49``, ``AdiSolver3D.h:49-61``): ``Init``, ``CreateSegments``,
``UpdateBoundaries``, ``TimeStep``, ``GetLayer``, plus state access.  Every call goes
through the C ABI of ``libadi_b200.so``; there is no Python or CPU compute path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import (ADI_FP32, ADI_FP64, ADI_SOLVER_EXACT, ADI_SOLVER_FAST, ADI_BATCH_PERSISTENT,  # noqa: F401
                   ADI_BATCH_MEMBER_GRAPHS, AdiError)

__all__ = ["AdiSolver3D", "AdiError", "fluid_params_normalized", "ADI_FP32", "ADI_FP64",
           "ADI_SOLVER_EXACT", "ADI_SOLVER_FAST", "library_path", "AdiBatch", "AdiSolver2D"]


def library_path() -> str:
    return _abi.LIB_PATH


def fluid_params_normalized(Re: float, Pr: float, lam: float) -> _abi.FluidParams:
    p = _abi.FluidParams()
    _abi.check(_abi.load().adi_fluid_params_normalized(Re, Pr, lam, C.byref(p)))
    return p


def fluid_params_dimensional(vis, rho, R, k, cv) -> _abi.FluidParams:
    p = _abi.FluidParams()
    _abi.check(_abi.load().adi_fluid_params_dimensional(vis, rho, R, k, cv, C.byref(p)))
    return p


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class AdiSolver3D:
    """One masked 3D domain resident on the current CUDA device."""

    def __init__(self, domain, params=None, Re: float = 200.0, Pr: float = 0.72, lam: float = 1.4,
                 precision: int = ADI_FP32, solver: int = ADI_SOLVER_FAST, stream=None):
        self.lib = _abi.load()
        self.domain = domain
        self.precision = precision
        self.dtype = np.float64 if precision == ADI_FP64 else np.float32
        self.shape = domain.shape
        self.h = C.c_void_p()
        self.params = params if params is not None else fluid_params_normalized(Re, Pr, lam)
        g = _abi.GridDesc(domain.nx, domain.ny, domain.nz, domain.dx, domain.dy, domain.dz, precision)
        _abi.check(self.lib.adi_create(C.byref(g), C.byref(self.params), C.byref(self.h)))
        if stream is not None:
            self.set_stream(stream)
        self._check(self.lib.adi_set_solver(self.h, solver))
        arrs = domain.arrays()
        if arrs is not None:   # a masks.GridBox leaves the mask to a GPU builder
            self._check(self.lib.adi_set_mask(self.h, *[_ptr(a) for a in arrs]))
        self.stats = None

    # -- plumbing --
    def _check(self, status):
        _abi.check(status, self.h)

    def set_stream(self, stream):
        handle = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", stream)
        self._check(self.lib.adi_set_stream(self.h, C.c_void_p(handle)))

    def set_solver(self, kind: int):
        self._check(self.lib.adi_set_solver(self.h, kind))

    def set_fault_injection(self, what: int):
        """adi_set_fault_injection: test-only failure modes (ADI_FAULT_*)."""
        self._check(self.lib.adi_set_fault_injection(self.h, what))

    def close(self):
        if self.h:
            self.lib.adi_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- mask builders (Grid3D::Prepare on the GPU) --
    def mask_shape3d(self, verts, tris, base_T: float) -> int:
        """Grid3D::Build of the triangles (grid-coordinate float32 vertices [nv, 3],
        vertex indices [nt, 3]); returns the flood-fill passes run."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        passes = C.c_int(0)
        self._check(self.lib.adi_mask_shape3d(self.h, _ptr(v), len(v), _ptr(t), len(t), base_T, C.byref(passes)))
        self.stats = None
        return passes.value

    def mask_sea(self, depth, zmin: float, base_T: float, in_vel=(0.0, 0.0, 0.0), in_T: float = 0.0):
        """Grid3D::Prepare3D_NetCDF from a depth map depth[di, dj] (negative under water)."""
        dmap = np.ascontiguousarray(depth, np.float32)
        vel = np.ascontiguousarray(in_vel, np.float32)
        self._check(self.lib.adi_mask_sea(self.h, _ptr(dmap), dmap.shape[0], dmap.shape[1], float(np.float32(zmin)),
                                          base_T, _ptr(vel), in_T))
        self.stats = None

    def mask_extrude2d(self, type2d, vel2d, T2d, active_nz: int, depth_var: float, base_T: float):
        """Grid3D::Prepare2D: the 2D node grid [nx, ny] (types, velocities [nx, ny, 2], T)
        extruded in depth."""
        t = np.ascontiguousarray(type2d, np.uint8)
        v = np.ascontiguousarray(vel2d, np.float32)
        T = np.ascontiguousarray(T2d, np.float32)
        self._check(self.lib.adi_mask_extrude2d(self.h, _ptr(t), _ptr(v), _ptr(T), active_nz, depth_var, base_T))
        self.stats = None

    def get_mask(self):
        """(type, bc_vel, bc_temp, vx, vy, vz, T) of the node grid, each [nx, ny, nz]."""
        shp = tuple(self.shape)
        out = [np.zeros(shp, np.uint8) for _ in range(3)] + [np.zeros(shp, np.float64) for _ in range(4)]
        self._check(self.lib.adi_get_mask(self.h, *[_ptr(a) for a in out]))
        return out

    # -- reference surface --
    def CreateSegments(self):
        st = _abi.SegStats()
        self._check(self.lib.adi_build_segments(self.h, C.byref(st)))
        self.stats = {
            "num_segments": list(st.num_segments), "num_nodes": list(st.num_nodes),
            "max_size": list(st.max_size), "max_per_line": list(st.max_per_line), "num_in": st.num_in,
        }
        return self.stats

    def UpdateBoundaries(self):
        self._check(self.lib.adi_update_boundaries(self.h))

    def TimeStep(self, dt, num_global, num_local, computeError=False):
        self._check(self.lib.adi_time_step(self.h, dt, num_global, num_local, int(computeError)))

    def step(self, dt, num_global, num_local, compute_error=False) -> int:
        """UpdateBoundaries + TimeStep; returns the raw status (0 = OK)."""
        return self.lib.adi_step(self.h, dt, num_global, num_local, int(compute_error))

    def run(self, dt, num_global, num_local, n_steps, err_every=10):
        self._check(self.lib.adi_run(self.h, dt, num_global, num_local, n_steps, err_every))

    def adjoint_run(self, dt, num_global, num_local, n_steps, ckpt_every, box_lo, box_hi):
        """Discrete adjoint of n_steps steps for J = 1/2 sum_{IN in box} |u|^2 at the end.
        Returns (J, dJ/d node values [4, nx, ny, nz], dJ/d initial state)."""
        lo = (C.c_int * 3)(*box_lo)
        hi = (C.c_int * 3)(*box_hi)
        J = C.c_double(0.0)
        gnv = np.zeros((4,) + tuple(self.shape), self.dtype)
        gst = np.zeros((4,) + tuple(self.shape), self.dtype)
        self._check(self.lib.adi_adjoint_run(self.h, dt, num_global, num_local, n_steps, ckpt_every, lo, hi,
                                             C.byref(J), _ptr(gnv), _ptr(gst)))
        return J.value, gnv, gst

    def set_node_values(self, vx, vy, vz, T):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (vx, vy, vz, T)]
        self._check(self.lib.adi_set_node_values(self.h, *[_ptr(a) for a in arrs]))

    def set_adjoint_chunk(self, K: int):
        self._check(self.lib.adi_set_adjoint_chunk(self.h, K))

    def step_tol(self, dt, max_global, num_local, tol, compute_error=False):
        """UpdateBoundaries + TimeStep in tolerance mode; returns (status, iterations, residual)."""
        it, res = C.c_int(0), C.c_double(0.0)
        rc = self.lib.adi_step_tol(self.h, dt, max_global, num_local, tol, int(compute_error), C.byref(it),
                                   C.byref(res))
        return rc, it.value, res.value

    def set_graphs(self, on: bool):
        self._check(self.lib.adi_set_graphs(self.h, int(on)))

    def GetLayer(self, outdimx=0, outdimy=0, outdimz=0):
        ox, oy, oz = outdimx or self.shape[0], outdimy or self.shape[1], outdimz or self.shape[2]
        v = np.zeros((ox, oy, oz, 3), self.dtype)
        T = np.zeros((ox, oy, oz), np.float64)
        self._check(self.lib.adi_get_layer(self.h, outdimx, outdimy, outdimz, _ptr(v), _ptr(T)))
        return v, T

    # -- state --
    def segments(self, direction: int) -> np.ndarray:
        n = C.c_int64()
        self._check(self.lib.adi_get_segments(self.h, direction, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 7), np.int32)
        self._check(self.lib.adi_get_segments(self.h, direction, _ptr(out), out.shape[0], C.byref(n)))
        return out[: n.value]

    def fields(self, which: int = 0):
        out = [np.zeros(self.shape, self.dtype) for _ in range(4)]
        self._check(self.lib.adi_get_state(self.h, which, *[_ptr(a) for a in out]))
        return out

    def set_state(self, u, v, w, T):
        arrs = [np.ascontiguousarray(a, self.dtype) for a in (u, v, w, T)]
        self._check(self.lib.adi_set_state(self.h, *[_ptr(a) for a in arrs]))

    def step_io(self, inputs, outputs, dt, num_global, num_local, compute_error=False) -> int:
        """adi_step_io: upload `inputs` (u, v, w, T host arrays of the handle's dtype),
        step, download into `outputs`; asynchronous until io_wait().  Returns the status."""
        for a in list(inputs) + list(outputs):
            if not (isinstance(a, np.ndarray) and a.dtype == self.dtype and a.flags.c_contiguous
                    and a.shape == tuple(self.shape)):
                raise ValueError("step_io takes C-contiguous arrays of the handle's shape and dtype")
        ins = (C.c_void_p * 4)(*[a.ctypes.data for a in inputs])
        outs = (C.c_void_p * 4)(*[a.ctypes.data for a in outputs])
        return self.lib.adi_step_io(self.h, ins, outs, dt, num_global, num_local, int(compute_error))

    def io_wait(self):
        self._check(self.lib.adi_io_wait(self.h))

    def div_error(self) -> float:
        out = C.c_double()
        self._check(self.lib.adi_div_error(self.h, C.byref(out)))
        return out.value

    def set_profiling(self, on: bool = True):
        self._check(self.lib.adi_set_profiling(self.h, int(on)))

    def profile(self, reset: bool = False) -> dict:
        """Per kernel class: launches, summed CUDA-event ms, algorithmic bytes."""
        p = _abi.Profile()
        self._check(self.lib.adi_get_profile(self.h, C.byref(p), int(reset)))
        return {name: {"launches": p.launches[c], "ms": p.ms[c], "bytes": p.bytes[c]}
                for c, name in enumerate(_abi.KERNEL_CLASSES)}

    def fast_shapes(self):
        """(K, NL, P) of the fast sweep per direction X, Y, Z."""
        out = []
        for dr in range(3):
            K, NL, P = C.c_int(), C.c_int(), C.c_int()
            self._check(self.lib.adi_get_fast_shape(self.h, dr, C.byref(K), C.byref(NL), C.byref(P)))
            out.append((K.value, NL.value, P.value))
        return out

    def set_fast_shape(self, direction: int, K: int, NL: int):
        self._check(self.lib.adi_set_fast_shape(self.h, direction, K, NL))

    def autotune(self, reps: int = 3):
        self._check(self.lib.adi_autotune(self.h, reps))

    def device_pointers(self):
        arr = (C.c_void_p * 8)()
        self._check(self.lib.adi_device_pointers(self.h, C.byref(arr)))
        return [arr[i] for i in range(8)]


class AdiBatch:
    """Many domains stepped together (adi_batch_*): one launch per sweep over all
    members, the step replayed as a CUDA graph.  Keeps its member solvers alive."""

    def __init__(self, solvers, stream=None):
        self.lib = _abi.load()
        self.members = list(solvers)
        n = len(self.members)
        arr = (C.c_void_p * n)(*[s.h.value for s in self.members])
        self.b = C.c_void_p()
        rc = self.lib.adi_batch_create(arr, n, C.byref(self.b))
        if rc != _abi.ADI_OK:
            msgs = [self.lib.adi_last_error_string(s.h) for s in self.members]
            raise _abi.AdiError(rc, "; ".join(m.decode() for m in msgs if m))
        if stream is not None:
            handle = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", stream)
            self._check(self.lib.adi_batch_set_stream(self.b, C.c_void_p(handle)))

    def _check(self, status):
        if status != _abi.ADI_OK:
            raw = self.lib.adi_batch_last_error_string(self.b) if self.b else b""
            raise _abi.AdiError(status, raw.decode() if raw else "")

    def step(self, dt, num_global, num_local, compute_error=False) -> int:
        """One step of every member; returns the raw status (0 = OK)."""
        return self.lib.adi_batch_step(self.b, dt, num_global, num_local, int(compute_error))

    def last_error(self) -> str:
        raw = self.lib.adi_batch_last_error_string(self.b)
        return raw.decode() if raw else ""

    def div_errors(self) -> np.ndarray:
        out = np.zeros(len(self.members), np.float64)
        self._check(self.lib.adi_batch_div_errors(self.b, out.ctypes.data))
        return out

    def set_chunk(self, direction: int, K: int):
        self._check(self.lib.adi_batch_set_chunk(self.b, direction, K))

    def chunks(self):
        out = []
        for dr in range(3):
            k = C.c_int()
            self._check(self.lib.adi_batch_get_chunk(self.b, dr, C.byref(k)))
            out.append(k.value)
        return out

    def autotune(self, dt: float, reps: int = 3):
        self._check(self.lib.adi_batch_autotune(self.b, dt, reps))

    def set_graphs(self, on: bool):
        self._check(self.lib.adi_batch_set_graphs(self.b, int(on)))

    def launches(self) -> int:
        v = C.c_int64()
        self._check(self.lib.adi_batch_launches(self.b, C.byref(v)))
        return v.value

    def step_io(self, inputs, outputs, dt, num_global, num_local, compute_error=False) -> int:
        """adi_batch_step_io: inputs / outputs hold, per member, its (u, v, w, T) host
        arrays (the member's shape and dtype); asynchronous until io_wait()."""
        n = len(self.members)
        flat_in = [a for m in inputs for a in m]
        flat_out = [a for m in outputs for a in m]
        if len(flat_in) != 4 * n or len(flat_out) != 4 * n:
            raise ValueError("four arrays per member in and out")
        for q, m in enumerate(self.members):
            for a in list(inputs[q]) + list(outputs[q]):
                if not (isinstance(a, np.ndarray) and a.dtype == m.dtype and a.flags.c_contiguous
                        and a.shape == tuple(m.shape)):
                    raise ValueError("step_io takes C-contiguous arrays of each member's shape and dtype")
        ins = (C.c_void_p * (4 * n))(*[a.ctypes.data for a in flat_in])
        outs = (C.c_void_p * (4 * n))(*[a.ctypes.data for a in flat_out])
        return self.lib.adi_batch_step_io(self.b, ins, outs, dt, num_global, num_local, int(compute_error))

    def io_wait(self):
        self._check(self.lib.adi_batch_io_wait(self.b))

    def set_schedule(self, schedule: int, branches: int = 1):
        """ADI_BATCH_PERSISTENT (one multi-domain launch per sweep) or
        ADI_BATCH_MEMBER_GRAPHS (each member's own step on `branches` graph branches)."""
        self._check(self.lib.adi_batch_set_schedule(self.b, schedule, branches))

    def schedule(self):
        """(schedule, branches)."""
        s, br = C.c_int(), C.c_int()
        self._check(self.lib.adi_batch_get_schedule(self.b, C.byref(s), C.byref(br)))
        return s.value, br.value

    def time_step(self, dt: float, num_global: int, num_local: int, reps: int = 3) -> float:
        """Mean ms of one whole batch step with the current schedule (graph replays)."""
        ms = C.c_float()
        self._check(self.lib.adi_batch_time_step(self.b, dt, num_global, num_local, reps, C.byref(ms)))
        return ms.value

    def time_sweeps(self, dt: float, reps: int = 3):
        """Mean ms of one batched sweep launch per direction X, Y, Z."""
        out = np.zeros(3, np.float32)
        self._check(self.lib.adi_batch_time_sweeps(self.b, dt, reps, out.ctypes.data))
        return [float(x) for x in out]

    @property
    def cells(self) -> int:
        return int(sum(int(np.prod(s.shape)) for s in self.members))

    def close(self):
        if self.b:
            self.lib.adi_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AdiSolver2D:
    """The reference's 2D ADI solver on the GPU (adi2d_*), Solver2D surface:
    Init (constructor), UpdateBoundaries, TimeStep, GetLayer, SetLayer."""

    def __init__(self, domain, Re: float = 100.0, Pr: float = 0.72, lam: float = 1.4,
                 precision: int = _abi.ADI_FP64, stream=None, params=None):
        self.lib = _abi.load()
        self.shape = domain.shape
        self.dtype = np.float64 if precision == _abi.ADI_FP64 else np.float32
        self.params = params if params is not None else fluid_params_normalized(Re, Pr, lam)
        self.h = C.c_void_p()
        _abi.check(self.lib.adi2d_create(domain.nx, domain.ny, domain.dx, domain.dy, precision,
                                         C.byref(self.params), C.byref(self.h)))
        if stream is not None:
            handle = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", stream)
            self._check(self.lib.adi2d_set_stream(self.h, C.c_void_p(handle)))
        arrs = [np.ascontiguousarray(domain.type, np.uint8), np.ascontiguousarray(domain.bct, np.uint8)]
        f = [np.ascontiguousarray(a, np.float64) for a in (domain.vx, domain.vy, domain.T)]
        self._check(self.lib.adi2d_set_grid(self.h, *[_ptr(a) for a in arrs + f], float(domain.startT)))

    def _check(self, status):
        if status != _abi.ADI_OK:
            raw = self.lib.adi2d_last_error_string(self.h) if self.h else b""
            raise _abi.AdiError(status, raw.decode() if raw else "")

    def set_segment_mode(self, mode: int):
        """0: the reference's row-spanning segments (default); 1: masked segments
        (runs of IN nodes, the 3D solver's segmentation)."""
        self._check(self.lib.adi2d_set_segments(self.h, mode))

    def UpdateBoundaries(self):
        self._check(self.lib.adi2d_update_boundaries(self.h))

    def TimeStep(self, dt, num_global, num_local) -> int:
        it = C.c_int(0)
        self._check(self.lib.adi2d_time_step(self.h, dt, num_global, num_local, C.byref(it)))
        return it.value

    def step(self, dt, num_global, num_local):
        """UpdateBoundaries + TimeStep; returns (status, global iterations)."""
        it = C.c_int(0)
        rc = self.lib.adi2d_step(self.h, dt, num_global, num_local, C.byref(it))
        return rc, it.value

    def step_tol(self, dt, max_global, num_local, tol):
        """UpdateBoundaries + tolerance-mode step; returns (status, iterations, residual)."""
        it, r = C.c_int(0), C.c_double(0)
        rc = self.lib.adi2d_step_tol(self.h, dt, max_global, num_local, tol, C.byref(it), C.byref(r))
        return rc, it.value, r.value

    def fields(self, which: int = 0):
        out = [np.zeros(self.shape, self.dtype) for _ in range(3)]
        self._check(self.lib.adi2d_get_state(self.h, which, *[_ptr(a) for a in out]))
        return out

    def SetLayer(self, u, v, T):
        arrs = [np.ascontiguousarray(a, self.dtype) for a in (u, v, T)]
        self._check(self.lib.adi2d_set_state(self.h, *[_ptr(a) for a in arrs]))

    def GetLayer(self, outdimx=0, outdimy=0):
        ox, oy = outdimx or self.shape[0], outdimy or self.shape[1]
        vel = np.zeros((ox, oy, 2))
        T = np.zeros((ox, oy))
        self._check(self.lib.adi2d_get_layer(self.h, outdimx, outdimy, _ptr(vel), _ptr(T)))
        return vel, T

    def last_error(self):
        e, it = C.c_double(), C.c_int()
        self._check(self.lib.adi2d_last_error(self.h, C.byref(e), C.byref(it)))
        return e.value, it.value

    def close(self):
        if self.h:
            self.lib.adi2d_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
