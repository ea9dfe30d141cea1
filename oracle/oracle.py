"""ctypes front ends for the two CPU oracles.  TEST INFRASTRUCTURE ONLY.

* ``RefSolver``    — the reference's own CPU solver compiled from its sources
                     (``_ref/libref3d.so``, float as shipped).
* ``OracleSolver`` — the C restatement (``liboracle_adi.so``) in float or double.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg import
this module, and only to check or to time the CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref3d.so")
ORACLE_LIB = os.path.join(HERE, "liboracle_adi.so")

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build(quiet: bool = True) -> None:
    """Builds liboracle_adi.so and, when the reference checkout is present,
    _ref/libref3d.so (oracle/Makefile)."""
    subprocess.run(["make", "-C", HERE, "all"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


_ref = None
_orc = None


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_LIB)
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [_u8p] * 3 + [_f32p] * 4
        lib.ref_segments.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        lib.ref_solver_init.argtypes = [C.c_void_p, C.c_int] + [C.c_double] * 5
        lib.ref_fluid_params.argtypes = [C.c_void_p, _f32p]
        lib.ref_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int]
        lib.ref_time_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int]
        lib.ref_get_fields.argtypes = [C.c_void_p, C.c_int] + [_f32p] * 4
        lib.ref_set_state.argtypes = [C.c_void_p] + [_f32p] * 4
        lib.ref_div_error.restype = C.c_double
        lib.ref_div_error.argtypes = [C.c_void_p]
        lib.ref_get_layer.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _f32p, _f64p]
        lib.ref_destroy.argtypes = [C.c_void_p]
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        lib.ref_shape3d_load.restype = vp
        lib.ref_shape3d_load.argtypes = [C.c_char_p, d, d, d, d, _i32p]
        lib.ref_shape2d_load.restype = vp
        lib.ref_shape2d_load.argtypes = [C.c_char_p, d, d, d, d, d, d, _i32p]
        lib.ref_sea_create.restype = vp
        lib.ref_sea_create.argtypes = [i, i, i, _f32p, i, i, C.c_float, d, _f32p, d]
        lib.ref_mask_prepare.argtypes = [vp, d]
        lib.ref_mask_nodes.argtypes = [vp] + [_u8p] * 3 + [_f32p] * 4
        lib.ref_shape3d_frame.argtypes = [vp, i, vp, vp, C.POINTER(i)]
        lib.ref_shape2d_grid.argtypes = [vp, _u8p, _u8p, _f32p, _f32p]
        lib.ref_mask_destroy.argtypes = [vp]
        _ref = lib
    return _ref


def _load_oracle():
    global _orc
    if _orc is None:
        lib = C.CDLL(ORACLE_LIB)
        lib.oracle_segments.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int]
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.c_int, C.c_int] + [C.c_int] * 3 + [C.c_double] * 3 + [_u8p] * 3 + [_f64p] * 4
        lib.oracle_set_params.argtypes = [C.c_void_p] + [C.c_double] * 4
        lib.oracle_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int]
        lib.oracle_time_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int]
        lib.oracle_step_tol.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                        C.POINTER(C.c_int), C.POINTER(C.c_double)]
        lib.oracle_get_fields.argtypes = [C.c_void_p, C.c_int] + [_f64p] * 4
        lib.oracle_adjoint_run.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                           C.c_void_p, C.POINTER(C.c_double), _f64p, _f64p]
        lib.oracle_set_node_values.argtypes = [C.c_void_p] + [_f64p] * 4
        lib.oracle_set_state.argtypes = [C.c_void_p] + [_f64p] * 4
        lib.oracle_div_error.restype = C.c_double
        lib.oracle_div_error.argtypes = [C.c_void_p]
        lib.oracle_last_div_error.restype = C.c_double
        lib.oracle_last_div_error.argtypes = [C.c_void_p]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        _orc = lib
    return _orc


def fluid_params_normalized(Re: float, Pr: float, lam: float):
    """FluidParams(Re, Pr, lambda) in double (Common/Geometry.h:545-552)."""
    return (1.0, 1.0 / Re, 1.0 / (Re * Pr), (lam - 1.0) / (lam * Re))


def oracle_segments(type_arr: np.ndarray, direction: int) -> np.ndarray:
    lib = _load_oracle()
    t = np.ascontiguousarray(type_arr, np.uint8)
    nx, ny, nz = t.shape
    n = lib.oracle_segments(t, nx, ny, nz, direction, None, 0)
    out = np.zeros((max(n, 1), 7), np.int32)
    lib.oracle_segments(t, nx, ny, nz, direction, out.ctypes.data, n)
    return out[:n]


class RefSolver:
    """The reference AdiSolver3D (CPU backend, float) on a synthetic Grid3D."""

    def __init__(self, d, Re=None, Pr=0.72, lam=1.4, dimensional=None):
        lib = _load_ref()
        self.lib = lib
        self.shape = d.shape
        t, bv, bt, vx, vy, vz, T = d.arrays()
        f = [np.ascontiguousarray(a, np.float32) for a in (vx, vy, vz, T)]
        self.h = lib.ref_create(d.nx, d.ny, d.nz, d.dx, d.dy, d.dz, t, bv, bt, *f)
        if not self.h:
            raise RuntimeError("ref_create failed")
        self._keep = (t, bv, bt, f)
        self.initialised = False
        if Re is not None or dimensional is not None:
            self.init_solver(Re, Pr, lam, dimensional)

    def init_solver(self, Re=None, Pr=0.72, lam=1.4, dimensional=None):
        if dimensional is not None:
            rc = self.lib.ref_solver_init(self.h, 1, *dimensional)
        else:
            rc = self.lib.ref_solver_init(self.h, 0, Re, Pr, lam, 0.0, 0.0)
        if rc == -3:
            raise ValueError("mask has more segments than the reference's fixed lists hold")
        if rc != 0:
            raise RuntimeError(f"ref_solver_init failed ({rc})")
        self.initialised = True

    def segments(self, direction: int) -> np.ndarray:
        n = self.lib.ref_segments(self.h, direction, None, 0)
        out = np.zeros((max(n, 1), 7), np.int32)
        self.lib.ref_segments(self.h, direction, out.ctypes.data, n)
        return out[:n]

    def step(self, dt, num_global, num_local, compute_error=True) -> int:
        return self.lib.ref_step(self.h, dt, num_global, num_local, int(compute_error))

    def time_step(self, dt, num_global, num_local, compute_error=True) -> int:
        """TimeStep without UpdateBoundaries."""
        return self.lib.ref_time_step(self.h, dt, num_global, num_local, int(compute_error))

    def fields(self, which=0):
        out = [np.zeros(self.shape, np.float32) for _ in range(4)]
        self.lib.ref_get_fields(self.h, which, *out)
        return out

    def set_state(self, u, v, w, T):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, T)]
        self.lib.ref_set_state(self.h, *arrs)

    def div_error(self) -> float:
        return self.lib.ref_div_error(self.h)

    def get_layer(self, outdimx=0, outdimy=0, outdimz=0):
        """Solver3D::GetLayer (Solver3D.cpp:21-25): velocities [ox, oy, oz, 3] (float)
        and T [ox, oy, oz] (double); it also sets the OUT cells of next to 99999."""
        ox, oy, oz = outdimx or self.shape[0], outdimy or self.shape[1], outdimz or self.shape[2]
        v = np.zeros((ox, oy, oz, 3), np.float32)
        T = np.zeros((ox, oy, oz), np.float64)
        rc = self.lib.ref_get_layer(self.h, outdimx, outdimy, outdimz, v, T)
        if rc != 0:
            raise RuntimeError(f"ref_get_layer failed ({rc})")
        return v, T

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


ADAPTER_LIB = os.path.join(HERE, "_ref", "libadapter3d.so")


def have_adapter() -> bool:
    return os.path.exists(ADAPTER_LIB)


def adapter_run(d, Re, Pr, lam, dt, num_global, num_local, steps, solver_kind, outdims=(0, 0, 0)):
    """The reference driver loop through the B200AdiSolver3D host adapter
    (oracle/adapter_harness.cpp, built against the reference's headers): returns
    GetLayer's velocities [ox, oy, oz, 3] (float) and T [ox, oy, oz] (double) after
    `steps` steps."""
    lib = C.CDLL(ADAPTER_LIB)
    lib.adapter_run.argtypes = ([C.c_int] * 3 + [C.c_double] * 3 + [_u8p] * 3 + [_f32p] * 4 + [C.c_double] * 4 +
                                [C.c_int] * 7 + [_f32p, _f64p, C.c_char_p, C.c_int])
    t, bv, bt, vx, vy, vz, T = d.arrays()
    f = [np.ascontiguousarray(a, np.float32) for a in (vx, vy, vz, T)]
    ox, oy, oz = (o or s for o, s in zip(outdims, d.shape))
    vout = np.zeros((ox, oy, oz, 3), np.float32)
    Tout = np.zeros((ox, oy, oz), np.float64)
    err = C.create_string_buffer(512)
    rc = lib.adapter_run(d.nx, d.ny, d.nz, d.dx, d.dy, d.dz, t, bv, bt, *f, Re, Pr, lam, dt, num_global, num_local,
                         steps, solver_kind, outdims[0], outdims[1], outdims[2], vout, Tout, err, len(err))
    if rc != 0:
        raise RuntimeError(f"adapter_run failed ({rc}): {err.value.decode(errors='replace')}")
    return vout, Tout


class OracleSolver:
    """The C restatement, precision 4 (float) or 8 (double)."""

    def __init__(self, d, precision=8, Re=200.0, Pr=0.72, lam=1.4, params=None, nthreads=0):
        lib = _load_oracle()
        self.lib = lib
        self.shape = d.shape
        arrs = d.arrays()
        self.h = lib.oracle_create(precision, nthreads, d.nx, d.ny, d.nz, d.dx, d.dy, d.dz, *arrs)
        self._keep = arrs
        p = params if params is not None else fluid_params_normalized(Re, Pr, lam)
        lib.oracle_set_params(self.h, *p)

    def step(self, dt, num_global, num_local, compute_error=True) -> int:
        return self.lib.oracle_step(self.h, dt, num_global, num_local, int(compute_error))

    def time_step(self, dt, num_global, num_local, compute_error=True) -> int:
        """TimeStep without UpdateBoundaries."""
        return self.lib.oracle_time_step(self.h, dt, num_global, num_local, int(compute_error))

    def adjoint_run(self, dt, num_global, num_local, n_steps, box_lo, box_hi):
        """FP64 discrete adjoint of n_steps steps for J = 1/2 sum_{IN in box} |u|^2 at the
        end; returns (J, dJ/d node values [4, nx, ny, nz], dJ/d initial state)."""
        lo = (C.c_int * 3)(*box_lo)
        hi = (C.c_int * 3)(*box_hi)
        J = C.c_double(0.0)
        gnv = np.zeros((4,) + tuple(self.shape), np.float64)
        gst = np.zeros((4,) + tuple(self.shape), np.float64)
        rc = self.lib.oracle_adjoint_run(self.h, dt, num_global, num_local, n_steps, lo, hi, C.byref(J), gnv, gst)
        if rc != 0:
            raise ValueError("the oracle adjoint needs a double-precision handle")
        return J.value, gnv, gst

    def set_node_values(self, vx, vy, vz, T):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (vx, vy, vz, T)]
        self.lib.oracle_set_node_values(self.h, *arrs)

    def step_tol(self, dt, max_global, num_local, tol, compute_error=False):
        """Tolerance-mode step; returns (status, iterations, residual)."""
        it, res = C.c_int(0), C.c_double(0.0)
        rc = self.lib.oracle_step_tol(self.h, dt, max_global, num_local, tol, int(compute_error), C.byref(it),
                                      C.byref(res))
        return rc, it.value, res.value

    def fields(self, which=0):
        out = [np.zeros(self.shape, np.float64) for _ in range(4)]
        self.lib.oracle_get_fields(self.h, which, *out)
        return out

    def set_state(self, u, v, w, T):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, T)]
        self.lib.oracle_set_state(self.h, *arrs)

    def div_error(self) -> float:
        return self.lib.oracle_div_error(self.h)

    def last_div_error(self) -> float:
        return self.lib.oracle_last_div_error(self.h)

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# 2D: the restatement (liboracle_adi2d.so) and the reference's own 2D solver
# (_ref/libref2d.so)
# ---------------------------------------------------------------------------
ORACLE2D_LIB = os.path.join(HERE, "liboracle_adi2d.so")
REF2D_LIB = os.path.join(HERE, "_ref", "libref2d.so")
_orc2d = None
_ref2d = None


def have_ref2d() -> bool:
    return os.path.exists(REF2D_LIB)


def _load_oracle2d():
    global _orc2d
    if _orc2d is None:
        lib = C.CDLL(ORACLE2D_LIB)
        lib.oracle2d_create.restype = C.c_void_p
        lib.oracle2d_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                        _u8p, _u8p, _f64p, _f64p, _f64p]
        lib.oracle2d_set_params.argtypes = [C.c_void_p] + [C.c_double] * 4
        lib.oracle2d_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
        lib.oracle2d_get_fields.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p]
        lib.oracle2d_last_err.restype = C.c_double
        lib.oracle2d_last_err.argtypes = [C.c_void_p]
        lib.oracle2d_segments.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.oracle2d_set_segments.argtypes = [C.c_void_p, C.c_int]
        lib.oracle2d_step_tol.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_double,
                                          C.POINTER(C.c_double)]
        lib.oracle2d_destroy.argtypes = [C.c_void_p]
        _orc2d = lib
    return _orc2d


def _load_ref2d():
    global _ref2d
    if _ref2d is None:
        lib = C.CDLL(REF2D_LIB)
        lib.ref2d_create.restype = C.c_void_p
        lib.ref2d_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _u8p, _u8p,
                                     _f64p, _f64p, _f64p, C.c_double, C.c_double, C.c_double]
        lib.ref2d_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
        lib.ref2d_get_fields.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p]
        lib.ref2d_destroy.argtypes = [C.c_void_p]
        _ref2d = lib
    return _ref2d


def fluid_params2d(Re, Pr, lam, precision):
    """FluidParams(Re, Pr, lambda) rounded to the working precision (Geometry.h:545-552)."""
    vals = [1.0, 1.0 / Re, 1.0 / (Re * Pr), (lam - 1) / (lam * Re)]
    if precision == 4:
        vals = [float(np.float32(v)) for v in vals]
    return vals


class Oracle2D:
    """The 2D restatement; precision 4 reproduces the reference float build."""

    def __init__(self, d, precision=8, Re=100.0, Pr=0.72, lam=1.4):
        self.lib = _load_oracle2d()
        self.shape = d.shape
        arrs = [np.ascontiguousarray(a) for a in (d.type.astype(np.uint8), d.bct.astype(np.uint8))]
        f = [np.ascontiguousarray(a, np.float64) for a in (d.vx, d.vy, d.T)]
        self.h = self.lib.oracle2d_create(precision, d.nx, d.ny, d.dx, d.dy, d.startT, *arrs, *f)
        self.lib.oracle2d_set_params(self.h, *fluid_params2d(Re, Pr, lam, precision))

    def set_segment_mode(self, mode: int) -> int:
        """0: the reference's row-spanning segments; 1: masked segments.  Returns
        the segment count."""
        n = self.lib.oracle2d_set_segments(self.h, mode)
        if n < 0:
            raise ValueError(f"bad segment mode {mode}")
        return n

    def step(self, dt, num_global, num_local) -> int:
        return self.lib.oracle2d_step(self.h, dt, num_global, num_local)

    def step_tol(self, dt, max_global, num_local, tol):
        """Tolerance-mode step: (iterations or -1, last residual)."""
        r = C.c_double()
        it = self.lib.oracle2d_step_tol(self.h, dt, max_global, num_local, tol, C.byref(r))
        return it, r.value

    def fields(self, which=0):
        out = [np.zeros(self.shape) for _ in range(3)]
        self.lib.oracle2d_get_fields(self.h, which, *out)
        return out

    def last_err(self) -> float:
        return self.lib.oracle2d_last_err(self.h)

    def segments(self) -> np.ndarray:
        n = self.lib.oracle2d_segments(self.h, None, 0)
        out = np.zeros((max(n, 1), 6), np.int32)
        self.lib.oracle2d_segments(self.h, out.ctypes.data, n)
        return out[:n]

    def close(self):
        if self.h:
            self.lib.oracle2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ref2D:
    """The reference's own AdiSolver2D (float), driven like its driver loop."""

    def __init__(self, d, Re=100.0, Pr=0.72, lam=1.4):
        self.lib = _load_ref2d()
        self.shape = d.shape
        arrs = [np.ascontiguousarray(a) for a in (d.type.astype(np.uint8), d.bct.astype(np.uint8))]
        f = [np.ascontiguousarray(a, np.float64) for a in (d.vx, d.vy, d.T)]
        self._keep = (arrs, f)
        self.h = self.lib.ref2d_create(d.nx, d.ny, d.dx, d.dy, d.startT, *arrs, *f, Re, Pr, lam)

    def step(self, dt, num_global, num_local):
        self.lib.ref2d_step(self.h, dt, num_global, num_local)

    def fields(self, which=0):
        out = [np.zeros(self.shape) for _ in range(3)]
        self.lib.ref2d_get_fields(self.h, which, *out)
        return out

    def close(self):
        if self.h:
            self.lib.ref2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefMask:
    """A reference Grid3D built by its own loaders and Prepare (Shape3D from a file,
    Shape2D from a file, SeaNetCDF from a depth map in memory)."""

    def __init__(self, handle, dims, lib, active_nz=None):
        if not handle:
            raise RuntimeError("the reference could not load the grid")
        self.h, self.dims, self.lib, self.active_nz = handle, tuple(dims), lib, active_nz

    @classmethod
    def shape3d(cls, path, dx, dy, dz, base_T):
        lib = _load_ref()
        dims = np.zeros(4, np.int32)
        return cls(lib.ref_shape3d_load(path.encode(), dx, dy, dz, base_T, dims), dims[:3], lib)

    @classmethod
    def shape2d(cls, path, dx, dy, dz, depth, depth_var, base_T):
        lib = _load_ref()
        dims = np.zeros(4, np.int32)
        h = lib.ref_shape2d_load(path.encode(), dx, dy, dz, depth, depth_var, base_T, dims)
        return cls(h, dims[:3], lib, int(dims[3]))

    @classmethod
    def sea(cls, dims, depth, zmin, base_T, in_vel, in_T):
        lib = _load_ref()
        dmap = np.ascontiguousarray(depth, np.float32)
        vel = np.ascontiguousarray(in_vel, np.float32)
        h = lib.ref_sea_create(dims[0], dims[1], dims[2], dmap, dmap.shape[0], dmap.shape[1], zmin, base_T, vel,
                               in_T)
        return cls(h, dims, lib)

    def prepare(self, time=0.0):
        if self.lib.ref_mask_prepare(self.h, time) != 0:
            raise RuntimeError("Grid3D::Prepare threw")

    def nodes(self):
        out = [np.zeros(self.dims, np.uint8) for _ in range(3)] + [np.zeros(self.dims, np.float32) for _ in range(4)]
        self.lib.ref_mask_nodes(self.h, *out)
        return out

    def frame(self, f):
        nt = C.c_int(0)
        nv = self.lib.ref_shape3d_frame(self.h, f, None, None, C.byref(nt))
        if nv < 0:
            raise IndexError(f)
        verts = np.zeros((nv, 3), np.float32)
        tris = np.zeros((nt.value, 3), np.int32)
        self.lib.ref_shape3d_frame(self.h, f, verts.ctypes.data, tris.ctypes.data, C.byref(nt))
        return verts, tris

    def grid2d(self):
        nx, ny = self.dims[0], self.dims[1]
        t = np.zeros((nx, ny), np.uint8)
        bc = np.zeros((nx, ny), np.uint8)
        v = np.zeros((nx, ny, 2), np.float32)
        T = np.zeros((nx, ny), np.float32)
        self.lib.ref_shape2d_grid(self.h, t, bc, v, T)
        self.last_bc2d = bc
        return t, v, T

    def close(self):
        if self.h:
            self.lib.ref_mask_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
