"""Helpers to load the golden fixtures (tests/golden/*.npz) as domains."""
from __future__ import annotations

import glob
import os

import numpy as np

from adi_b200 import geometry as G

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def step_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "step_*.npz")))


def case_name(path: str) -> str:
    return os.path.basename(path)[5:-4]


def load_case(path: str):
    z = np.load(path)
    t = z["type"]
    h = z["h"]
    d = G.Domain(*t.shape, float(h[0]), float(h[1]), float(h[2]), t, z["bc_vel"], z["bc_temp"],
                 z["vx"], z["vy"], z["vz"], z["T"])
    dt, ng, nl, steps = z["run"]
    run = dict(dt=float(dt), num_global=int(ng), num_local=int(nl), steps=int(steps))
    if "dimensional" in z:
        params = ("dimensional", tuple(float(x) for x in z["dimensional"]))
    else:
        Re, Pr, lam = (float(x) for x in z["normalized"])
        params = ("normalized", (Re, Pr, lam))
    return d, run, params, z


def fluid_params_tuple(params):
    """(v_T, v_vis, t_vis, t_phi) in double, as FluidParams' constructors compute them
    before their (FTYPE) casts (Common/Geometry.h:545-561)."""
    kind, p = params
    if kind == "normalized":
        Re, Pr, lam = p
        return (1.0, 1.0 / Re, 1.0 / (Re * Pr), (lam - 1.0) / (lam * Re))
    vis, rho, R, k, cv = p
    return (R, vis / rho, k / (rho * cv), vis / (rho * cv))


def non_out(d):
    return d.type != G.NODE_OUT
