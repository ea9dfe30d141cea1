"""The reference's result file (Common/IO.h OutputNetCDF3D_header / _layer) through
adi_nc_write_header / adi_nc_write_layer: NetCDF classic (64-bit offset) files with
the reference's dimensions, variables, attributes and values."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi


class BBox3D(C.Structure):
    _fields_ = [("pmin", C.c_float * 3), ("pmax", C.c_float * 3)]


def write_header(path: str, pmin, pmax, timestep: float, time: float, outdims, out_vars, depth=None,
                 xy_degree_units: bool = False) -> None:
    """OutputNetCDF3D_header(path, bbox, depths, timestep, time, outdimx, outdimy, outdimz,
    out_vars, xy_degree_units); depth: [nx][ny] float array (needed when "d" is asked for)."""
    lib = _abi.load()
    bb = BBox3D((C.c_float * 3)(*pmin), (C.c_float * 3)(*pmax))
    dp, dnx, dny = None, 0, 0
    if depth is not None:
        depth = np.ascontiguousarray(depth, np.float32)
        dp, (dnx, dny) = depth.ctypes.data, depth.shape
    rc = lib.adi_nc_write_header(path.encode(), C.byref(bb), dp, dnx, dny, timestep, time, *outdims,
                                 ",".join(out_vars).encode(), int(xy_degree_units))
    if rc != 0:
        raise _abi.AdiError(rc, f"adi_nc_write_header({path})")


def write_layer(path: str, vel, T, layer: int, out_vars) -> None:
    """OutputNetCDF3D_layer(path, vel, T, layer, outdimx, outdimy, outdimz, out_vars):
    vel [x][y][z][3] float32 or float64 (GetLayer's Vec3D), T [x][y][z] float64."""
    lib = _abi.load()
    vel = np.ascontiguousarray(vel)
    if vel.dtype not in (np.float32, np.float64) or vel.ndim != 4 or vel.shape[3] != 3:
        raise ValueError("vel must be [x][y][z][3] float32 or float64")
    T = np.ascontiguousarray(T, np.float64)
    nx, ny, nz = vel.shape[:3]
    if T.shape != (nx, ny, nz):
        raise ValueError(f"T must be [x][y][z] like vel, got {T.shape} for {vel.shape[:3]}")
    rc = lib.adi_nc_write_layer(path.encode(), vel.ctypes.data, vel.itemsize, T.ctypes.data, layer, nx, ny, nz,
                                ",".join(out_vars).encode())
    if rc != 0:
        raise _abi.AdiError(rc, f"adi_nc_write_layer({path})")
