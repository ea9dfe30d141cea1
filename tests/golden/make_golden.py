"""Generates the golden fixtures in this directory from the reference's own CPU
solver (oracle/_ref/libref3d.so, compiled from the reference sources by
oracle/Makefile).  Run on a machine that has the reference checkout:

    make -C oracle REF=<reference checkout>/src && python tests/golden/make_golden.py

Each case stores the synthetic inputs (node arrays), the reference's segment lists
for X, Y, Z, and its fields after selected steps of the driver loop
(UpdateBoundaries + TimeStep), with the status and divergence error of every step.
Edge-case masks (IN cell at index 0, runs that reach the last cell, many segments
per line, empty lines) store segment lists only: the solver cannot step them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cmc-fluid-solver_b200"))

import oracle as O  # noqa: E402
from adi_b200 import geometry as G  # noqa: E402

STEP_CASES = {
    # name: (domain factory, params, dt, num_global, num_local, steps, keep)
    "rand_a": (lambda: G.random_domain(16, 14, 12, seed=11), dict(Re=150.0), 1e-3, 4, 2, 6, (1, 6)),
    "rand_shell": (lambda: G.random_domain(13, 17, 15, seed=12, shell=True, n_obstacles=4, rmax=4.0),
                   dict(Re=80.0, Pr=1.0, lam=1.6), 2e-3, 2, 1, 5, (1, 5)),
    "spheres": (lambda: G.spheres_channel(dims=(24, 20, 18), n_spheres=4, rmin=2.0, rmax=4.0, seed=3)
                .round_values_to_float32(), dict(Re=200.0), 5e-4, 4, 2, 4, (4,)),
    "dimensional": (lambda: G.random_domain(12, 12, 12, seed=13, free_outflow=False),
                    dict(dimensional=(0.05, 1000.0, 461.495, 0.6, 4200.0)), 1e-3, 3, 1, 3, (3,)),
}


def edge_masks():
    rng = np.random.default_rng(99)
    out = {}
    t = np.full((9, 7, 8), G.NODE_IN, np.uint8)          # all IN: runs reach both ends
    out["all_in"] = t
    t = np.full((9, 7, 8), G.NODE_OUT, np.uint8)         # no fluid at all
    out["no_fluid"] = t
    t = (rng.random((11, 10, 9)) < 0.55).astype(np.uint8)  # IN(0)/OUT(1) noise, many segments per line
    out["noise"] = t
    t = rng.integers(0, 4, size=(7, 12, 10)).astype(np.uint8)  # all four node types mixed
    out["mixed_types"] = t
    t = np.full((6, 5, 40), G.NODE_BOUND, np.uint8)      # alternating single-cell runs along z
    t[:, :, 1::2] = G.NODE_IN
    out["alternating"] = t
    return out


def main():
    O.build()
    if not O.have_ref():
        raise SystemExit("reference build missing (oracle/_ref/libref3d.so)")
    for name, (make, params, dt, ng, nl, steps, keep) in STEP_CASES.items():
        d = make()
        assert G.validate_for_solver(d) is None, name
        ref = O.RefSolver(d, **params)
        rec = {"type": d.type, "bc_vel": d.bc_vel, "bc_temp": d.bc_temp,
               "vx": d.vx, "vy": d.vy, "vz": d.vz, "T": d.T,
               "h": np.array([d.dx, d.dy, d.dz]),
               "run": np.array([dt, ng, nl, steps], np.float64)}
        if "dimensional" in params:
            rec["dimensional"] = np.array(params["dimensional"])
        else:
            rec["normalized"] = np.array([params["Re"], params.get("Pr", 0.72), params.get("lam", 1.4)])
        for dr in range(3):
            rec[f"segs{dr}"] = ref.segments(dr)
        status, errs = [], []
        for s in range(1, steps + 1):
            status.append(ref.step(dt, ng, nl, True))
            errs.append(ref.div_error())
            if s in keep:
                u, v, w, T = ref.fields(0)
                rec[f"step{s}_u"], rec[f"step{s}_v"], rec[f"step{s}_w"], rec[f"step{s}_T"] = u, v, w, T
        rec["status"] = np.array(status, np.int32)
        rec["div_error"] = np.array(errs)
        rec["keep"] = np.array(keep, np.int32)
        ref.close()
        np.savez_compressed(os.path.join(HERE, f"step_{name}.npz"), **rec)
        print("wrote", name)
    segrec = {}
    for name, t in edge_masks().items():
        shape = t.shape
        z = np.zeros(shape)
        d = G.Domain(*shape, 0.1, 0.1, 0.1, t, np.zeros(shape, np.uint8), np.zeros(shape, np.uint8), z, z, z, z)
        ref = O.RefSolver(d)
        segrec[f"{name}_type"] = t
        for dr in range(3):
            segrec[f"{name}_segs{dr}"] = ref.segments(dr)
        ref.close()
    np.savez_compressed(os.path.join(HERE, "segments_edge.npz"), **segrec)
    print("wrote segments_edge")


if __name__ == "__main__":
    main()
