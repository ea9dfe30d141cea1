"""Generates tests/golden/masks.npz: node grids built by the reference's own
Grid3D loaders and mask builders (oracle/_ref/libref3d.so, compiled from the
reference's sources by oracle/Makefile) on the synthetic inputs of
adi_b200/shapes.py, together with the inputs the GPU builders take.

Run from the repository root on a machine with the reference checkout:
    python tests/golden/make_masks.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "cmc-fluid-solver_b200"))

from adi_b200 import shapes as ms  # noqa: E402
from adi_b200 import masks  # noqa: E402
from oracle.oracle import RefMask  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "masks.npz")

# (name, frames, dx, time)
SHAPE3D = [
    ("tetra", [ms.tetra() + (None,)], 0.01, 0.0),
    ("box_frame", [ms.box() + (None,)], 0.02, 0.0),
    ("box", [ms.box() + (None,)], 0.01, 0.0),
    ("sphere", [ms.uv_sphere() + (None,)], 0.01, 0.0),
    ("moving", [ms.tetra() + (None,), (ms.moved(ms.tetra()[0]), ms.tetra()[1], None)], 0.01, 0.005),
    ("leaky", [ms.box(drop_faces=1) + (None,)], 0.01, 0.0),
]
BASE_T = 1.0


def nodes_dict(prefix, r):
    t, bv, bt, vx, vy, vz, T = r.nodes()
    return {f"{prefix}_type": t, f"{prefix}_bcv": bv, f"{prefix}_bct": bt,
            f"{prefix}_val": np.stack([vx, vy, vz, T])}


def main():
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, frames, dx, time in SHAPE3D:
            path = os.path.join(tmp, name + ".txt")
            ms.write_shape3d(path, frames)
            r = RefMask.shape3d(path, dx, dx, dx, BASE_T)
            sf = masks.load_shape3d(path, dx, dx, dx)
            assert tuple(int(d) for d in r.dims) == sf.dims
            verts, tris = sf.subframe(time)
            r.prepare(time)
            out.update(nodes_dict("s3_" + name, r))
            out[f"s3_{name}_verts"] = verts
            out[f"s3_{name}_tris"] = tris
            out[f"s3_{name}_dims"] = np.array(sf.dims, np.int32)
            r.close()

        for name, dvar in (("ch_bump", 0.4), ("ch_flat", 0.0)):
            path = os.path.join(tmp, "channel2d.txt")
            ms.write_shape2d(path, ms.channel2d())
            r = RefMask.shape2d(path, 0.01, 0.01, 0.02, 0.3, dvar, BASE_T)
            r.prepare(0.0)
            t2, v2, T2 = r.grid2d()
            out.update(nodes_dict("e2_" + name, r))
            out[f"e2_{name}_t2"], out[f"e2_{name}_v2"], out[f"e2_{name}_T2"] = t2, v2, T2
            out[f"e2_{name}_dims"] = np.array(list(r.dims) + [r.active_nz], np.int32)
            out[f"e2_{name}_depth_var"] = np.array(dvar)
            r.close()

    with tempfile.TemporaryDirectory() as tmp:
        # Shape2D node grids (Grid2D::Build) of the 2D grid of Grid3D's Shape2D path
        for name, frames, time, d in (("channel", [(10.0, ms.channel2d())], 0.0, 0.01),
                                      ("moving", ms.channel2d_moving(), 0.8, 0.008)):
            path = os.path.join(tmp, name + ".txt")
            ms.write_shape2d(path, None, frames=frames)
            r = RefMask.shape2d(path, d, d, 0.02, 0.3, 0.4, BASE_T)
            r.prepare(time)
            t2, v2, T2 = r.grid2d()
            sf = masks.load_shape2d(path, d, d)
            assert sf.dims == (int(r.dims[0]), int(r.dims[1]))
            segs, kinds = sf.subframe(time)
            out[f"s2_{name}_segs"], out[f"s2_{name}_kinds"] = segs, kinds
            out[f"s2_{name}_dims"] = np.array(sf.dims, np.int32)
            out[f"s2_{name}_type"], out[f"s2_{name}_bc"] = t2, r.last_bc2d
            out[f"s2_{name}_vel"], out[f"s2_{name}_T"] = v2, T2
            r.close()

    for name, open_far, vel, tin in (("basin", False, (0.0, 0.0, 0.0), 1.0), ("open", True, (0.1, -0.2, 0.05), 1.5)):
        lats = np.linspace(64.0, 67.0, 64)
        lons = np.linspace(32.0, 37.0, 50)
        dep = ms.depth_map(64, 50, open_far=open_far)
        dims, zmin = masks.sea_geometry(lats, lons, dep, 0.05, 0.1, 2.0)
        r = RefMask.sea(dims, dep, zmin, BASE_T, vel, tin)
        r.prepare(0.0)
        out.update(nodes_dict("sea_" + name, r))
        out[f"sea_{name}_depth"] = dep
        out[f"sea_{name}_dims"] = np.array(dims, np.int32)
        out[f"sea_{name}_zmin"] = np.array(zmin, np.float32)
        out[f"sea_{name}_vel"] = np.array(vel, np.float32)
        out[f"sea_{name}_tin"] = np.array(tin)
        r.close()
    # the reference's own pipeline from a Shape3D file: its Grid3D::Prepare node grid
    # stepped by its CPU solver (the GPU test builds the grid with adi_mask_shape3d
    # from the same vertices and steps it with the exact solver)
    from adi_b200.geometry import Domain
    from oracle.oracle import RefSolver
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "sphere.txt")
        ms.write_shape3d(path, [ms.uv_sphere() + (None,)])
        dx = 0.025
        r = RefMask.shape3d(path, dx, dx, dx, BASE_T)
        r.prepare(0.0)
        t, bv, bt, vx, vy, vz, T = r.nodes()
        # the reference leaves the BCs of Shape3D walls unset (whatever the heap held);
        # they are given the no-slip value that fresh memory holds and the GPU builder
        # gives a handle without a mask
        wall = t == 2
        bv[wall] = 0
        bt[wall] = 0
        assert not bv.any() and not bt.any()
        sf = masks.load_shape3d(path, dx, dx, dx)
        verts, tris = sf.subframe(0.0)
        d = Domain(*sf.dims, dx, dx, dx, t, bv, bt, *[a.astype(np.float64) for a in (vx, vy, vz, T)])
        ref = RefSolver(d, Re=200.0)
        status, errs = [], []
        for _ in range(3):
            status.append(ref.step(2e-4, 4, 2, True))
            errs.append(ref.div_error())
        u, v, w, TT = ref.fields(0)
        ref.close()
        r.close()
        out.update({"run_s25_verts": verts, "run_s25_tris": tris, "run_s25_dims": np.array(sf.dims, np.int32),
                    "run_s25_fields": np.stack([u, v, w, TT]), "run_s25_status": np.array(status, np.int32),
                    "run_s25_div": np.array(errs), "run_s25_h": np.array([dx, dx, dx])})
    # the reference's 2D pipeline from a Shape2D file: its Grid2D::Build node grid
    # stepped by its own 2D solver (float, as shipped)
    from adi_b200.geometry2d import Domain2D
    from oracle.oracle import Ref2D
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "moving.txt")
        ms.write_shape2d(path, None, frames=ms.channel2d_moving())
        d2 = 0.008
        r = RefMask.shape2d(path, d2, d2, 0.02, 0.3, 0.4, BASE_T)
        r.prepare(0.8)
        t2, v2, T2 = r.grid2d()
        dom = Domain2D(int(r.dims[0]), int(r.dims[1]), d2, d2, t2, r.last_bc2d, v2[..., 0].astype(np.float64),
                       v2[..., 1].astype(np.float64), T2.astype(np.float64), startT=BASE_T)
        ref2 = Ref2D(dom, Re=100.0)
        for _ in range(3):
            ref2.step(1e-3, 2, 1)
        out["run2d_fields"] = np.stack(ref2.fields(0))
        ref2.close()
        r.close()
    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
