"""GPU mask builders (adi_mask_shape3d / adi_mask_sea / adi_mask_extrude2d) against
the reference's own Grid3D::Prepare.

The node grids in tests/golden/masks.npz were built by the reference's compiled
loaders and mask builders (tests/golden/make_masks.py); the GPU builders must give
the same grid bit for bit: node types everywhere, BCs and node values everywhere
the reference defines them.  (The reference leaves the BCs of the NODE_BOUND cells
of a Shape3D grid unset: Grid3D::Init, Grid3D.cpp:353-370, allocates the nodes
without initialising bc_vel/bc_temp and Build never writes them there.)
"""
import os

import numpy as np
import pytest

from adi_b200 import masks
from golden_util import GOLDEN

pytestmark = pytest.mark.gpu

Z = np.load(os.path.join(GOLDEN, "masks.npz"))
S3 = sorted({k[3:-5] for k in Z.files if k.startswith("s3_") and k.endswith("_type")})
E2 = sorted({k[3:-5] for k in Z.files if k.startswith("e2_") and k.endswith("_type")})
SEA = sorted({k[4:-5] for k in Z.files if k.startswith("sea_") and k.endswith("_type")})


def _solver(adi_lib, dims, precision=None, solver=None):
    from adi_b200 import _abi
    box = masks.GridBox(int(dims[0]), int(dims[1]), int(dims[2]), 0.01, 0.01, 0.01)
    return adi_lib.AdiSolver3D(box, precision=precision or _abi.ADI_FP32,
                               solver=_abi.ADI_SOLVER_EXACT if solver is None else solver)


def _compare(got, prefix, bc_at_bound=True):
    t, bv, bt, vx, vy, vz, T = got
    rt = Z[prefix + "_type"]
    np.testing.assert_array_equal(t, rt)
    keep = np.ones(rt.shape, bool) if bc_at_bound else rt != 2
    np.testing.assert_array_equal(bv[keep], Z[prefix + "_bcv"][keep])
    np.testing.assert_array_equal(bt[keep], Z[prefix + "_bct"][keep])
    val = Z[prefix + "_val"].astype(np.float64)
    for q, a in enumerate((vx, vy, vz, T)):
        np.testing.assert_array_equal(a, val[q])


@pytest.mark.parametrize("name", S3)
def test_shape3d_matches_reference(adi_lib, name):
    p = "s3_" + name
    s = _solver(adi_lib, Z[p + "_dims"])
    passes = s.mask_shape3d(Z[p + "_verts"], Z[p + "_tris"], 1.0)
    assert passes >= 1
    _compare(s.get_mask(), p, bc_at_bound=False)


def test_shape3d_fp64_handle(adi_lib):
    from adi_b200 import _abi
    p = "s3_sphere"
    s = _solver(adi_lib, Z[p + "_dims"], precision=_abi.ADI_FP64)
    s.mask_shape3d(Z[p + "_verts"], Z[p + "_tris"], 1.0)
    _compare(s.get_mask(), p, bc_at_bound=False)


def test_shape3d_keeps_wall_data(adi_lib):
    """A rebuild over an existing grid keeps the BCs and values of the cells that
    end up NODE_BOUND (the reference's node array persists between Prepare calls)
    and resets NODE_IN / NODE_OUT cells to no-slip, v = 0, T = baseT."""
    from adi_b200.geometry import Domain
    p = "s3_tetra"
    dims = tuple(int(d) for d in Z[p + "_dims"])
    rng = np.random.default_rng(5)
    prev = Domain(*dims, 0.01, 0.01, 0.01, np.full(dims, 1, np.uint8), rng.integers(0, 2, dims).astype(np.uint8),
                  rng.integers(0, 2, dims).astype(np.uint8), *[rng.standard_normal(dims).astype(np.float32)
                                                                 .astype(np.float64) for _ in range(4)])
    s = adi_lib.AdiSolver3D(prev)
    s.mask_shape3d(Z[p + "_verts"], Z[p + "_tris"], 2.5)
    t, bv, bt, vx, vy, vz, T = s.get_mask()
    np.testing.assert_array_equal(t, Z[p + "_type"])
    wall = t == 2
    np.testing.assert_array_equal(bv[wall], prev.bc_vel[wall])
    np.testing.assert_array_equal(bt[wall], prev.bc_temp[wall])
    for a, b in ((vx, prev.vx), (vy, prev.vy), (vz, prev.vz), (T, prev.T)):
        np.testing.assert_array_equal(a[wall], b[wall])
    assert not bv[~wall].any() and not bt[~wall].any()
    assert not vx[~wall].any() and not vy[~wall].any() and not vz[~wall].any()
    assert (T[~wall] == 2.5).all()


@pytest.mark.parametrize("name", SEA)
def test_sea_matches_reference(adi_lib, name):
    p = "sea_" + name
    s = _solver(adi_lib, Z[p + "_dims"])
    s.mask_sea(Z[p + "_depth"], float(Z[p + "_zmin"]), 1.0, Z[p + "_vel"], float(Z[p + "_tin"]))
    _compare(s.get_mask(), p)


@pytest.mark.parametrize("name", E2)
def test_extrude2d_matches_reference(adi_lib, name):
    p = "e2_" + name
    nx, ny, nz, active = (int(v) for v in Z[p + "_dims"])
    s = _solver(adi_lib, (nx, ny, nz))
    s.mask_extrude2d(Z[p + "_t2"], Z[p + "_v2"], Z[p + "_T2"], active, float(Z[p + "_depth_var"]), 1.0)
    _compare(s.get_mask(), p)


def test_built_mask_steps_like_uploaded(adi_lib):
    """A grid built on the GPU steps exactly like the same grid uploaded with
    adi_set_mask (exact solver, bit for bit)."""
    from adi_b200 import _abi
    from adi_b200.geometry import Domain
    p = "s3_sphere"
    dims = tuple(int(d) for d in Z[p + "_dims"])
    a = _solver(adi_lib, dims)
    a.mask_shape3d(Z[p + "_verts"], Z[p + "_tris"], 1.0)
    t, bv, bt, vx, vy, vz, T = a.get_mask()
    # inflow on the walls of the sphere's upstream half
    vel = np.where((t == 2) & (np.arange(dims[0])[:, None, None] < dims[0] // 2), 0.5, 0.0)
    d = Domain(*dims, 0.01, 0.01, 0.01, t, bv, bt, vel, vy, vz, T)
    a.set_node_values(vel, vy, vz, T)
    b = adi_lib.AdiSolver3D(d, solver=_abi.ADI_SOLVER_EXACT)
    assert a.CreateSegments() == b.CreateSegments()   # includes the NODE_IN count
    # set_node_values changes the boundary data only; give both the same start state
    b.set_state(*a.fields())
    for s in (a, b):
        for _ in range(3):
            assert s.step(1e-3, 2, 1) == 0
    for x, y in zip(a.fields(), b.fields()):
        np.testing.assert_array_equal(x, y)


def test_shape_outside_grid_is_rejected(adi_lib):
    from adi_b200._abi import AdiError
    p = "s3_tetra"
    s = _solver(adi_lib, Z[p + "_dims"])
    with pytest.raises(AdiError, match="outside the node grid"):
        s.mask_shape3d(Z[p + "_verts"] * 3.0, Z[p + "_tris"], 1.0)
    with pytest.raises(AdiError):
        s.mask_shape3d(Z[p + "_verts"], Z[p + "_tris"] + 100, 1.0)


def test_extrude_bottom_past_column_is_rejected(adi_lib):
    """depth_var large enough that the reference's bottom loop runs past the column
    (into the next columns' nodes) is refused."""
    from adi_b200._abi import AdiError
    p = "e2_ch_bump"
    nx, ny, nz, active = (int(v) for v in Z[p + "_dims"])
    s = _solver(adi_lib, (nx, ny, nz))
    with pytest.raises(AdiError, match="outside the node grid"):
        s.mask_extrude2d(Z[p + "_t2"], Z[p + "_v2"], Z[p + "_T2"], active, 1.5, 1.0)


def test_contract_check_of_built_mask_matches_upload(adi_lib):
    """The device-side contract check of a built grid reports what the host check
    of the same grid uploaded with adi_set_mask reports (here: water reaching the
    near borders puts NODE_IN cells on the outer frame)."""
    from adi_b200 import _abi
    from adi_b200.geometry import Domain
    p = "sea_open"
    dims = tuple(int(d) for d in Z[p + "_dims"])
    dep = Z[p + "_depth"][::-1, ::-1].copy()
    a = _solver(adi_lib, dims)
    a.mask_sea(dep, float(Z[p + "_zmin"]), 1.0, Z[p + "_vel"], float(Z[p + "_tin"]))
    t, bv, bt, vx, vy, vz, T = a.get_mask()
    b = adi_lib.AdiSolver3D(Domain(*dims, 0.01, 0.01, 0.01, t, bv, bt, vx, vy, vz, T), solver=_abi.ADI_SOLVER_EXACT)
    msgs = []
    for s in (a, b):
        s.CreateSegments()
        assert s.step(1e-3, 1, 1) == _abi.ADI_ERR_BAD_ARG
        msgs.append(s.lib.adi_last_error_string(s.h))
    assert msgs[0] == msgs[1] and b"outer frame" in msgs[0]


S2 = sorted({k[3:-5] for k in Z.files if k.startswith("s2_") and k.endswith("_type")})


@pytest.mark.parametrize("name", S2)
def test_shape2d_matches_reference(adi_lib, name):
    """adi_mask_shape2d == the reference's Grid2D::Build (node type, BC, velocity, T)."""
    p = "s2_" + name
    nx, ny = (int(v) for v in Z[p + "_dims"])
    t, bc, v, T = masks.build_shape2d(Z[p + "_segs"], Z[p + "_kinds"], nx, ny, 1.0)
    np.testing.assert_array_equal(t, Z[p + "_type"])
    np.testing.assert_array_equal(bc, Z[p + "_bc"])
    np.testing.assert_array_equal(v.view(np.uint32), Z[p + "_vel"].view(np.uint32))
    np.testing.assert_array_equal(T.view(np.uint32), Z[p + "_T"].view(np.uint32))


def test_shape2d_then_extrusion_matches_reference(adi_lib):
    """A Shape2D file to a 3D node grid entirely on the GPU: the 2D grid built by
    adi_mask_shape2d, extruded by adi_mask_extrude2d, equals the reference's
    Grid3D::Prepare of the same file."""
    p2, p3 = "s2_channel", "e2_ch_bump"
    nx, ny = (int(v) for v in Z[p2 + "_dims"])
    t, bc, v, T = masks.build_shape2d(Z[p2 + "_segs"], Z[p2 + "_kinds"], nx, ny, 1.0)
    _, _, nz, active = (int(x) for x in Z[p3 + "_dims"])
    s = _solver(adi_lib, (nx, ny, nz))
    s.mask_extrude2d(t, v, T, active, float(Z[p3 + "_depth_var"]), 1.0)
    _compare(s.get_mask(), p3)


def test_shape3d_file_to_steps_matches_reference_pipeline(adi_lib):
    """The reference's own pipeline from a Shape3D file -- Grid3D::Prepare then its
    CPU solver, 3 steps -- against the GPU's: adi_mask_shape3d from the same
    vertices, then the exact solver.  Fields equal bit for bit on every cell the
    reference defines (not NODE_OUT; its layers leave those unset, which also makes
    its divergence error -- whose 8-corner stencil reaches NODE_OUT cells diagonal to
    the fluid -- depend on leftover memory, so that is not compared here)."""
    from adi_b200 import _abi
    nx, ny, nz = (int(v) for v in Z["run_s25_dims"])
    h = float(Z["run_s25_h"][0])
    box = masks.GridBox(nx, ny, nz, h, h, h)
    s = adi_lib.AdiSolver3D(box, Re=200.0, solver=_abi.ADI_SOLVER_EXACT)
    s.mask_shape3d(Z["run_s25_verts"], Z["run_s25_tris"], 1.0)
    t = s.get_mask()[0]
    s.CreateSegments()
    for q in range(3):
        assert s.step(2e-4, 4, 2, True) == int(Z["run_s25_status"][q])
    m = t != 1
    for f, want in zip(s.fields(0), Z["run_s25_fields"]):
        np.testing.assert_array_equal(f[m].view(np.uint32), want[m].view(np.uint32))


def test_shape2d_file_to_steps_matches_reference_pipeline(adi_lib):
    """The reference's 2D pipeline from a Shape2D file -- Grid2D::Build, then its own
    2D solver (float, as shipped), 3 steps -- against adi_mask_shape2d and the GPU
    2D solver in float: fields equal bit for bit."""
    from adi_b200 import _abi
    from adi_b200.geometry2d import Domain2D
    p = "s2_moving"
    nx, ny = (int(v) for v in Z[p + "_dims"])
    t, bc, v, T = masks.build_shape2d(Z[p + "_segs"], Z[p + "_kinds"], nx, ny, 1.0)
    d = Domain2D(nx, ny, 0.008, 0.008, t, bc, v[..., 0].astype(np.float64), v[..., 1].astype(np.float64),
                 T.astype(np.float64), startT=1.0)
    g = adi_lib.AdiSolver2D(d, Re=100.0, precision=_abi.ADI_FP32)
    for _ in range(3):
        assert g.step(1e-3, 2, 1)[0] == 0
    for a, b in zip(g.fields(0), Z["run2d_fields"]):
        assert np.array_equal(a.astype(np.float64), b)
