"""GPU checks of the fast (chunked) sweep against the oracle.

Tolerances: the fast sweep solves the same equations with a different elimination
order, so it is compared (a) in double against the double oracle at 1e-11 of each
field's scale, and (b) in float against the double oracle, where its error must
stay within the reference's own float drift (the float oracle equals the reference
bit for bit) and below 1e-5 of the flow scale.
"""
import numpy as np
import pytest

import oracle as O
from adi_b200 import geometry as G
from golden_util import fluid_params_tuple, non_out

pytestmark = pytest.mark.gpu


def solver(adi_lib, d, params, precision=None, shapes=None):
    from adi_b200 import _abi
    fp = adi_lib.fluid_params_normalized(*params)
    s = adi_lib.AdiSolver3D(d, params=fp, precision=precision or _abi.ADI_FP32, solver=_abi.ADI_SOLVER_FAST)
    s.CreateSegments()
    if shapes:
        for dr, (K, NL) in enumerate(shapes):
            s.set_fast_shape(dr, K, NL)
    return s


def rel_errors(got, want, m):
    vs = max(np.max(np.abs(want[f][m])) for f in range(3))
    out = []
    for f in range(4):
        scale = vs if f < 3 else np.max(np.abs(want[3][m]))
        out.append(float(np.max(np.abs(got[f][m].astype(np.float64) - want[f][m])) / scale))
    return out


# (K, NL) per direction for a 34 x 30 x 40 domain; 32 <= NL * ceil(len/K) <= 256
SHAPES = [
    [(4, 8), (4, 8), (4, 4)],
    [(8, 16), (8, 8), (8, 8)],
    [(12, 16), (12, 16), (12, 8)],
    [(16, 32), (16, 16), (16, 16)],
    [(8, 8), (16, 16), (4, 4)],
]


@pytest.mark.parametrize("shapes", SHAPES, ids=lambda s: "-".join(f"K{k}NL{n}" for k, n in s))
def test_fast_fp64_matches_oracle(adi_lib, shapes):
    from adi_b200 import _abi
    d = G.random_domain(34, 30, 40, seed=51, shell=True, n_obstacles=9, rmax=5.0)
    params = (120.0, 0.72, 1.4)
    s = solver(adi_lib, d, params, precision=_abi.ADI_FP64, shapes=shapes)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(8e-4, 4, 2, True) == 0
        assert orc.step(8e-4, 4, 2, True) == 0
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < 1e-11, errs
    # next layer (boundary writes of the last step) as well
    errs_n = rel_errors(s.fields(1), orc.fields(1), m)
    assert max(errs_n) < 1e-11, errs_n


@pytest.mark.parametrize("shapes", [[(4, 8), (4, 8), (4, 4)], [(8, 16), (8, 8), (8, 8)], [(12, 16), (12, 16), (12, 8)]],
                         ids=lambda s: "-".join(f"K{k}NL{n}" for k, n in s))
def test_fast_fp32_within_reference_drift(adi_lib, shapes):
    d = G.spheres_channel(dims=(48, 40, 44), n_spheres=5, rmin=3, rmax=6, seed=7).round_values_to_float32()
    params = (200.0, 0.72, 1.4)
    s = solver(adi_lib, d, params, shapes=shapes)
    o32 = O.OracleSolver(d, precision=4, params=fluid_params_tuple(("normalized", params)))
    o64 = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    for _ in range(10):
        assert s.step(5e-4, 4, 2, False) == 0
        o32.step(5e-4, 4, 2, False)
        o64.step(5e-4, 4, 2, False)
    m = non_out(d)
    e_gpu = rel_errors(s.fields(0), o64.fields(0), m)
    e_ref = rel_errors(o32.fields(0), o64.fields(0), m)
    for f in range(4):
        assert e_gpu[f] <= 1e-5, (f, e_gpu, e_ref)
        assert e_gpu[f] <= 2.0 * e_ref[f] + 2e-7, (f, e_gpu, e_ref)


def test_autotuner_picks_supported_shapes(adi_lib):
    from adi_b200 import _abi
    d = G.spheres_channel(dims=(64, 48, 80), n_spheres=8, rmin=3, rmax=7, seed=3)
    s = solver(adi_lib, d, (200.0, 0.72, 1.4))
    shapes = s.fast_shapes()
    for dr, (K, NL, P) in enumerate(shapes):
        assert K in (4, 5, 8, 12, 16)
        assert P * K >= d.shape[dr]
        if NL == 0:
            assert dr == 2 and P == -(-d.shape[2] // K)      # warp-resident Z lines
        elif NL < 0:
            assert dr < 2 and NL in (-8, -16, -32) and P * K == d.shape[dr]   # TMA-fed X/Y tiles
        else:
            assert 32 <= NL * P <= 256
    with pytest.raises(_abi.AdiError):
        s.set_fast_shape(0, 5, 8)
    with pytest.raises(_abi.AdiError):
        s.set_fast_shape(2, 4, 64)   # 64 lines x 20 chunks > 256 threads
    s.autotune(2)
    assert s.step(5e-4, 2, 1, True) == 0


def test_fast_matches_exact_closely(adi_lib):
    """Fast and exact sweeps agree to float rounding after a few steps."""
    from adi_b200 import _abi
    d = G.random_domain(24, 22, 26, seed=61, n_obstacles=6, rmax=4.0)
    fp = adi_lib.fluid_params_normalized(150.0, 0.72, 1.4)
    a = adi_lib.AdiSolver3D(d, params=fp, solver=_abi.ADI_SOLVER_FAST)
    b = adi_lib.AdiSolver3D(d, params=fp, solver=_abi.ADI_SOLVER_EXACT)
    a.CreateSegments()
    b.CreateSegments()
    for _ in range(3):
        assert a.step(1e-3, 4, 2, True) == 0
        assert b.step(1e-3, 4, 2, True) == 0
    m = non_out(d)
    errs = rel_errors(a.fields(0), [x.astype(np.float64) for x in b.fields(0)], m)
    assert max(errs) < 2e-6, errs


@pytest.mark.parametrize("zK", [4, 8])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_zwarp_kernel(adi_lib, zK, precision):
    """Warp-resident Z kernel (NL = 0): dimz = P*K with P a power of two <= 32."""
    from adi_b200 import _abi
    d = G.random_domain(30, 26, 32, seed=71, shell=True, n_obstacles=7, rmax=4.0)
    params = (110.0, 0.72, 1.4)
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    s = solver(adi_lib, d, params, precision=prec, shapes=[(8, 8), (8, 8), (zK, 0)])
    assert s.fast_shapes()[2][1] == 0
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(8e-4, 4, 2, True) == 0
        assert orc.step(8e-4, 4, 2, True) == 0
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < (1e-11 if precision == "fp64" else 2e-6), errs
    errs_n = rel_errors(s.fields(1), orc.fields(1), m)
    assert max(errs_n) < (1e-11 if precision == "fp64" else 2e-6), errs_n


@pytest.mark.parametrize("xK,nl", [(8, -16), (16, -16), (8, -8), (4, -8), (4, -16)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_xytma_kernel(adi_lib, xK, nl, precision):
    """TMA-fed X/Y kernel with 16 (NL = -16) or 8 (NL = -8) lines per CTA and
    chunk-major tiles: dimz a multiple of 16, lines of 4, 8 or 16 chunks of K rows
    (X: 64 rows, Y: 32 rows)."""
    from adi_b200 import _abi
    d = G.random_domain(64, 32, 32, seed=81, shell=True, n_obstacles=8, rmax=4.5)
    params = (130.0, 0.72, 1.4)
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    s = solver(adi_lib, d, params, precision=prec, shapes=[(xK, nl), (min(xK, 8), nl), (4, 0)])
    assert s.fast_shapes()[0][1] == nl and s.fast_shapes()[1][1] == nl
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(8e-4, 4, 2, True) == 0
        assert orc.step(8e-4, 4, 2, True) == 0
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < (1e-11 if precision == "fp64" else 2e-6), errs
    errs_n = rel_errors(s.fields(1), orc.fields(1), m)
    assert max(errs_n) < (1e-11 if precision == "fp64" else 2e-6), errs_n


@pytest.mark.parametrize("nx", [256, 384])
def test_xytma_lines_over_several_warps(adi_lib, nx):
    """TMA-fed X sweep with X lines of 64 and 96 chunks (K = 4, 8 lines per CTA): a
    line spans two or three warps, whose reduced system goes through shared memory
    with a named barrier per line; against the FP64 oracle."""
    d = G.random_domain(nx, 32, 32, seed=83, shell=True, n_obstacles=12, rmax=5.0)
    params = (140.0, 0.72, 1.4)
    s = solver(adi_lib, d, params, shapes=[(4, -8), (4, -8), (4, 0)])
    assert s.fast_shapes()[0] == (4, -8, nx // 4)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(8e-4, 4, 2, True) == 0
        assert orc.step(8e-4, 4, 2, True) == 0
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < 2e-6, errs
    errs_n = rel_errors(s.fields(1), orc.fields(1), m)
    assert max(errs_n) < 2e-6, errs_n


@pytest.mark.parametrize("dims,xK", [((61, 45, 37), 4), ((150, 37, 29), 5), ((100, 120, 33), 4)],
                         ids=["61x45x37-K4", "150x37x29-K5", "100x120x33-K4"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_xy_tiles_copied_elementwise_any_dims(adi_lib, dims, xK, precision):
    """The X/Y tile kernel with tiles copied element by element (NL = -1): dimz not a
    multiple of the 8-line tile (the last tile of each plane is partly padding) and
    line lengths that are not P K (rows past the line end are padding rows)."""
    from adi_b200 import _abi
    d = G.random_domain(*dims, seed=85, shell=True, n_obstacles=9, rmax=5.0)
    params = (125.0, 0.72, 1.4)
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    s = solver(adi_lib, d, params, precision=prec, shapes=[(xK, -1), (xK, -1), (4, 8)])
    assert s.fast_shapes()[0][:2] == (xK, -1) and s.fast_shapes()[1][:2] == (xK, -1)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(8e-4, 4, 2, True) == 0
        assert orc.step(8e-4, 4, 2, True) == 0
    tol = 1e-11 if precision == "fp64" else 2e-6
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < tol, errs
    errs_n = rel_errors(s.fields(1), orc.fields(1), m)
    assert max(errs_n) < tol, errs_n


@pytest.mark.parametrize("nz,zK", [(50, 4), (52, 4), (50, 5), (77, 8), (160, 5), (36, 8)],
                         ids=["nz50-K4-scalar", "nz52-K4-vector-ragged", "nz50-K5", "nz77-K8", "nz160-K5-full",
                              "nz36-K8-vector-ragged"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_zwarp_any_dimz(adi_lib, nz, zK, precision):
    """The warp-resident Z sweep on lines that are not P K long: the smallest P in
    {4, 8, 16, 32} with P K >= dimz, rows past the line end as padding, chunks moved
    as vectors where dimz keeps them aligned and row by row elsewhere."""
    from adi_b200 import _abi
    d = G.random_domain(30, 26, nz, seed=86 + nz, shell=True, n_obstacles=7, rmax=4.5)
    params = (140.0, 0.72, 1.4)
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    s = solver(adi_lib, d, params, precision=prec)
    s.set_fast_shape(2, zK, 0)
    assert s.fast_shapes()[2][:2] == (zK, 0)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(8e-4, 4, 2, True) == 0
        assert orc.step(8e-4, 4, 2, True) == 0
    tol = 1e-11 if precision == "fp64" else 2e-6
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < tol, errs
    errs_n = rel_errors(s.fields(1), orc.fields(1), m)
    assert max(errs_n) < tol, errs_n


@pytest.mark.parametrize("nz", [384, 300], ids=["nz384-K12-full", "nz300-K12-ragged"])
def test_zwarp_twelve_row_chunks(adi_lib, nz):
    """The warp-resident Z sweep with 12-row chunks (float only): lines of up to 384
    rows in one warp; FP64 rejects the shape."""
    from adi_b200 import _abi
    d = G.random_domain(12, 10, nz, seed=90 + nz, shell=True, n_obstacles=6, rmax=4.0)
    params = (140.0, 0.72, 1.4)
    s = solver(adi_lib, d, params, precision=_abi.ADI_FP32)
    s.set_fast_shape(2, 12, 0)
    assert s.fast_shapes()[2][:2] == (12, 0)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(8e-4, 4, 2, True) == 0
        assert orc.step(8e-4, 4, 2, True) == 0
    assert max(rel_errors(s.fields(0), orc.fields(0), m)) < 2e-6
    assert max(rel_errors(s.fields(1), orc.fields(1), m)) < 2e-6
    s64 = solver(adi_lib, d, params, precision=_abi.ADI_FP64)
    with pytest.raises(_abi.AdiError):
        s64.set_fast_shape(2, 12, 0)


def _slab_domain(nx, ny, nz, seed):
    """Random shell domain plus a wall slab at k = 1..16, so that the first 16-line
    tile of every X and Y plane holds no segment (the persistent kernel skips it)."""
    d = G.random_domain(nx, ny, nz, seed=seed, shell=True, n_obstacles=10, rmax=6.0)
    slab = np.zeros(d.shape, bool)
    slab[:, :, 1:17] = True
    slab &= d.type != G.NODE_BOUND
    d.type[slab] = G.NODE_BOUND
    d.bc_vel[slab] = G.BC_NOSLIP
    d.bc_temp[slab] = G.BC_NOSLIP
    for name in ("vx", "vy", "vz"):
        getattr(d, name)[slab] = 0.0
    assert G.validate_for_solver(d) is None
    return d


@pytest.mark.parametrize("xK", [4, 8])
@pytest.mark.parametrize("slab", [False, True], ids=["plain", "empty-tiles"])
def test_xypair_kernel(adi_lib, xK, slab):
    """Persistent double-buffered X/Y kernel (NL = -32, FP32): more tiles than CTAs,
    so every CTA cycles both tile buffers; with the slab, tiles without segments
    are skipped without a load."""
    d = (_slab_domain(128, 96, 48, seed=85) if slab else
         G.random_domain(128, 96, 48, seed=84, shell=True, n_obstacles=12, rmax=7.0))
    params = (160.0, 0.72, 1.4)
    s = solver(adi_lib, d, params, shapes=[(xK, -32), (xK, -32), (8, 8)])
    assert s.fast_shapes()[0][1] == -32 and s.fast_shapes()[1][1] == -32
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(3):
        assert s.step(6e-4, 4, 2, True) == 0
        assert orc.step(6e-4, 4, 2, True) == 0
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < 2e-6, errs
    errs_n = rel_errors(s.fields(1), orc.fields(1), m)
    assert max(errs_n) < 2e-6, errs_n


@pytest.mark.parametrize("nl", [-16, -8])
def test_xytma_empty_tiles(adi_lib, nl):
    """TMA-fed X/Y kernel on a domain whose first tiles of every X and Y plane hold
    no segment: those CTAs leave before any load; the rest match the FP64 oracle."""
    d = _slab_domain(128, 64, 48, seed=88)
    params = (150.0, 0.72, 1.4)
    s = solver(adi_lib, d, params, shapes=[(8, nl), (8, nl), (8, 8)])
    assert s.fast_shapes()[0][1] == nl and s.fast_shapes()[1][1] == nl
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    m = non_out(d)
    for _ in range(2):
        assert s.step(6e-4, 4, 2, True) == 0
        assert orc.step(6e-4, 4, 2, True) == 0
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < 2e-6, errs


def test_xypair_rejects_fp64_and_bad_shapes(adi_lib):
    from adi_b200 import _abi
    d = G.random_domain(64, 48, 32, seed=86, n_obstacles=4)
    s = solver(adi_lib, d, (100.0, 0.72, 1.4), precision=_abi.ADI_FP64)
    with pytest.raises(_abi.AdiError):
        s.set_fast_shape(0, 4, -32)          # FP32 only
    s32 = solver(adi_lib, d, (100.0, 0.72, 1.4))
    s32.set_fast_shape(0, 4, -32)
    with pytest.raises(_abi.AdiError):
        s32.set_fast_shape(2, 4, -32)        # X and Y only
    with pytest.raises(_abi.AdiError):
        s32.set_fast_shape(0, 16, -32)       # K in {4, 8}
    with pytest.raises(_abi.AdiError):
        s32.set_fast_shape(0, 4, -24)        # no such variant


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_time_step_with_boundary_state_off_node_values(adi_lib, precision):
    """adi_time_step without a boundary update, from a state whose BOUND/VALVE cells
    differ from the node values: the fast kernels must load the node values for
    Dirichlet rows rather than read them from the nonlinear layer."""
    from adi_b200 import _abi
    d = G.random_domain(48, 40, 32, seed=87, shell=True, n_obstacles=8, rmax=4.5)
    params = (140.0, 0.72, 1.4)
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    s = solver(adi_lib, d, params, precision=prec)
    orc = O.OracleSolver(d, precision=8, params=fluid_params_tuple(("normalized", params)))
    rng = np.random.default_rng(87)
    state = [(a + 0.05 * rng.standard_normal(d.shape)).astype(np.float32).astype(np.float64)
             for a in (d.vx, d.vy, d.vz, d.T)]
    s.set_state(*[a.astype(np.float64 if precision == "fp64" else np.float32) for a in state])
    orc.set_state(*state)
    m = non_out(d)
    for _ in range(2):
        s.TimeStep(7e-4, 3, 2, True)
        assert orc.time_step(7e-4, 3, 2, True) == 0
    errs = rel_errors(s.fields(0), orc.fields(0), m)
    assert max(errs) < (1e-11 if precision == "fp64" else 2e-6), errs


@pytest.mark.parametrize("case", ["fp32", "fp64", "fp32-exact-direct"])
def test_step_io_pipelined_time_march_equals_separate_calls(adi_lib, case):
    """adi_step_io chained through host buffers (each call uploads the previous
    call's download) equals adi_set_state + adi_step + adi_get_state bit for bit,
    with and without the divergence error (graph replay, and direct launches with
    the exact solver), and adi_io_wait orders later work."""
    import torch
    from adi_b200 import _abi
    precision = "fp64" if case == "fp64" else "fp32"
    d = G.random_domain(40, 36, 44, seed=91, shell=True, n_obstacles=6, rmax=4.5)
    params = (150.0, 0.72, 1.4)
    prec = _abi.ADI_FP64 if precision == "fp64" else _abi.ADI_FP32
    a = solver(adi_lib, d, params, precision=prec)
    b = solver(adi_lib, d, params, precision=prec)
    for dr, (K, NL, _) in enumerate(a.fast_shapes()):
        b.set_fast_shape(dr, K, NL)
    if case == "fp32-exact-direct":
        for s_ in (a, b):
            s_._check(s_.lib.adi_set_solver(s_.h, _abi.ADI_SOLVER_EXACT))
            s_.set_graphs(False)
    dt_ = np.float32 if precision == "fp32" else np.float64
    pin = [torch.empty(d.shape, dtype=torch.float32 if precision == "fp32" else torch.float64,
                       pin_memory=True).numpy() for _ in range(8)]
    for x, y in zip(pin[:4], a.fields(0)):
        x[...] = y
    start = [x.copy() for x in pin[:4]]
    bufs_in, bufs_out = pin[:4], pin[4:]
    for i in range(4):
        assert a.step_io(bufs_in, bufs_out, 7e-4, 3, 2, i in (0, 3)) == 0
        bufs_in, bufs_out = bufs_out, bufs_in
    a.io_wait()
    state = start
    for i in range(4):
        b.set_state(*state)
        assert b.step(7e-4, 3, 2, i in (0, 3)) == 0
        state = [x.copy() for x in b.fields(0)]
    for f in range(4):
        assert bufs_in[f].dtype == dt_
        assert np.array_equal(bufs_in[f], state[f]), f
    assert a.div_error() == b.div_error()
    for f in range(4):
        assert np.array_equal(a.fields(0)[f], b.fields(0)[f])
