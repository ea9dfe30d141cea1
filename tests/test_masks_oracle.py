"""Host side of the mask builders against the reference's own loaders (no GPU).

* adi_b200.masks.load_shape3d reads a Shape3D file exactly as Grid3D::Load3DShape
  does: the same grid size and the same grid-coordinate vertices, bit for bit.
* Shape3DFrames.subframe gives the vertices recorded in the golden fixtures
  (the frame blend of Grid3D::ComputeSubframeInfo).
* sea_geometry / extrude_dims give the reference's grid sizes.
* The committed fixtures are what the reference builds today (when its compiled
  harness is present).
"""
import os
import tempfile

import numpy as np
import pytest

from adi_b200 import shapes as ms
import oracle as O
from adi_b200 import masks
from golden_util import GOLDEN

Z = np.load(os.path.join(GOLDEN, "masks.npz"))
need_ref = pytest.mark.skipif(not O.have_ref(), reason="the reference harness (oracle/_ref) is not built here")

SHAPES = {
    "tetra": [ms.tetra() + (None,)],
    "box": [ms.box() + (None,)],
    "sphere": [ms.uv_sphere() + (None,)],
    "moving": [ms.tetra() + (None,), (ms.moved(ms.tetra()[0]), ms.tetra()[1], None)],
    "leaky": [ms.box(drop_faces=1) + (None,)],
}


@need_ref
@pytest.mark.parametrize("name", sorted(SHAPES))
@pytest.mark.parametrize("dx", [0.02, 0.01, 0.013])
def test_shape3d_loader_matches_reference(name, dx):
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, name + ".txt")
        ms.write_shape3d(path, SHAPES[name])
        ref = O.RefMask.shape3d(path, dx, dx, dx, 1.0)
        ours = masks.load_shape3d(path, dx, dx, dx)
        assert tuple(int(d) for d in ref.dims) == ours.dims
        for f, fr in enumerate(ours.frames):
            rv, rt = ref.frame(f)
            np.testing.assert_array_equal(rv.view(np.uint32), fr.verts.view(np.uint32))
            np.testing.assert_array_equal(rt, fr.tris)


def test_shape3d_subframe_matches_fixture():
    times = {"moving": 0.005}
    with tempfile.TemporaryDirectory() as tmp:
        for name in ("tetra", "box", "sphere", "moving", "leaky"):
            path = os.path.join(tmp, name + ".txt")
            ms.write_shape3d(path, SHAPES[name])
            ours = masks.load_shape3d(path, 0.01, 0.01, 0.01)
            v, t = ours.subframe(times.get(name, 0.0))
            np.testing.assert_array_equal(v.view(np.uint32), Z[f"s3_{name}_verts"].view(np.uint32))
            np.testing.assert_array_equal(t, Z[f"s3_{name}_tris"])
            assert ours.dims == tuple(Z[f"s3_{name}_dims"])


def test_shape3d_reader_number_forms(tmp_path):
    """Commas as decimal points and %i integer forms, as the reference's reader takes them."""
    p = tmp_path / "t.txt"
    p.write_text("1\n3\n0,5 0 0 0 0 0\n1000 0 0 0 0 0\n0 700 250,25 0 0 0\n0x1\n0 1 02\n")
    s = masks.load_shape3d(str(p), 0.02, 0.02, 0.02)
    assert s.frames[0].tris.tolist() == [[0, 1, 2]]
    assert s.frames[0].verts.shape == (3, 3)


def test_sea_geometry_matches_fixture():
    lats = np.linspace(64.0, 67.0, 64)
    lons = np.linspace(32.0, 37.0, 50)
    for name, open_far in (("basin", False), ("open", True)):
        dims, zmin = masks.sea_geometry(lats, lons, ms.depth_map(64, 50, open_far=open_far), 0.05, 0.1, 2.0)
        assert dims == tuple(Z[f"sea_{name}_dims"])
        assert np.float32(zmin) == Z[f"sea_{name}_zmin"]


def test_extrude_dims_match_fixture():
    active, nz = masks.extrude_dims(0.3, 0.02)
    assert (active, nz) == (int(Z["e2_ch_bump_dims"][3]), int(Z["e2_ch_bump_dims"][2]))
    assert masks.extrude_dims(0.3, 0.02, align=True) == (16, 32)


@need_ref
def test_fixtures_are_what_the_reference_builds():
    """Rebuilds two fixture cases with the reference and compares (so a change in
    the generator or the harness cannot leave stale fixtures behind)."""
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "sphere.txt")
        ms.write_shape3d(path, SHAPES["sphere"])
        r = O.RefMask.shape3d(path, 0.01, 0.01, 0.01, 1.0)
        r.prepare(0.0)
        t = r.nodes()[0]
        np.testing.assert_array_equal(t, Z["s3_sphere_type"])
    dep = ms.depth_map(64, 50, open_far=True)
    r = O.RefMask.sea(tuple(Z["sea_open_dims"]), dep, float(Z["sea_open_zmin"]), 1.0, Z["sea_open_vel"],
                      float(Z["sea_open_tin"]))
    r.prepare(0.0)
    got = r.nodes()
    np.testing.assert_array_equal(got[0], Z["sea_open_type"])
    np.testing.assert_array_equal(np.stack(got[3:]), Z["sea_open_val"])


def test_shape2d_subframe_matches_fixture(tmp_path):
    """load_shape2d + subframe give the segments recorded with the fixtures (the grid
    they build is compared with the reference's on the GPU)."""
    for name, frames, time, d in (("channel", [(10.0, ms.channel2d())], 0.0, 0.01),
                                  ("moving", ms.channel2d_moving(), 0.8, 0.008)):
        path = str(tmp_path / (name + ".txt"))
        ms.write_shape2d(path, None, frames=frames)
        sf = masks.load_shape2d(path, d, d)
        segs, kinds = sf.subframe(time)
        assert sf.dims == tuple(Z[f"s2_{name}_dims"])
        np.testing.assert_array_equal(segs.view(np.uint32), Z[f"s2_{name}_segs"].view(np.uint32))
        np.testing.assert_array_equal(kinds, Z[f"s2_{name}_kinds"])


@need_ref
@pytest.mark.parametrize("d", [0.01, 0.008, 0.013])
def test_shape2d_grid_size_matches_reference(tmp_path, d):
    path = str(tmp_path / "moving.txt")
    ms.write_shape2d(path, None, frames=ms.channel2d_moving())
    r = O.RefMask.shape2d(path, d, d, 0.02, 0.3, 0.4, 1.0)
    assert masks.load_shape2d(path, d, d).dims == (int(r.dims[0]), int(r.dims[1]))
