"""A domain split into X slabs (Y and Z sweeps) and Y pencils (X sweeps): adi_b200.slabs.

* CPU: the plan's ranges and the local domains (ghost planes coded NODE_BOUND,
  the solver contract holds on every part);
* CPU, two gloo ranks: the block moves (ghost planes of slabs and pencils, slab ->
  pencil and pencil -> slab transposes) give every part the same arrays as the
  single-process moves do, and those equal the slices of the global arrays;
* GPU: the split step, parts emulated on one device, equals the single-domain
  step bit for bit (every line is solved whole on one part with the same kernel),
  with the exact and the fast solvers, over several steps.
"""
import os
import socket

import numpy as np
import pytest

from adi_b200 import geometry as G
from adi_b200 import slabs as S


def test_plan_covers_the_domain_and_local_domains_keep_the_contract():
    d = G.random_domain(31, 26, 18, seed=12, shell=True, n_obstacles=5, rmax=3.5)
    for parts in (1, 2, 3):
        P = S.SlabPlan(*d.shape, parts)
        xs = [P.slab(s) for s in range(parts)]
        ys = [P.pencil(r) for r in range(parts)]
        assert xs[0][0] == 0 and xs[-1][1] == d.nx and all(a[1] == b[0] for a, b in zip(xs, xs[1:]))
        assert ys[0][0] == 0 and ys[-1][1] == d.ny and all(a[1] == b[0] for a, b in zip(ys, ys[1:]))
        for s in range(parts):
            x0, x1, lo, hi = xs[s]
            sd = S.slab_domain(d, P, s)
            assert sd.shape == (hi - lo, d.ny, d.nz)
            assert G.validate_for_solver(sd) is None
            assert np.array_equal(sd.type[x0 - lo:x1 - lo], d.type[x0:x1])
            if x0 > lo:
                assert np.all(sd.type[0] == G.NODE_BOUND)
            pd = S.pencil_domain(d, P, s)
            y0, y1, plo, phi = ys[s]
            assert G.validate_for_solver(pd) is None
            assert np.array_equal(pd.type[:, y0 - plo:y1 - plo], d.type[:, y0:y1])
    with pytest.raises(ValueError):
        S.SlabPlan(8, 8, 8, 3)


def _part_arrays(P, glob, parts_here, fill):
    """Per-part CPU arrays: slabs hold their owned x range of the global arrays
    (ghost planes `fill`), pencils all `fill`; keyed [part][role] -> 4 tensors."""
    import torch
    slab, pencil = {}, {}
    for s in parts_here:
        x0, x1, lo, hi = P.slab(s)
        slab[s] = {}
        for role in range(5):
            f = []
            for v in range(4):
                a = torch.full((hi - lo, P.ny, P.nz), fill, dtype=torch.float64)
                a[x0 - lo:x1 - lo] = torch.from_numpy(glob[role][v][x0:x1])
                f.append(a)
            slab[s][role] = f
        y0, y1, plo, phi = P.pencil(s)
        pencil[s] = {role: [torch.full((P.nx, phi - plo, P.nz), fill, dtype=torch.float64) for _ in range(4)]
                     for role in range(5)}
    return slab, pencil


def _run_moves(P, comm, parts_here):
    """Ghosts, slab -> pencil, a change on the pencils, pencil -> slab, pencil ghosts."""
    rng = np.random.default_rng(4)
    glob = [[rng.standard_normal((P.nx, P.ny, P.nz)) for _ in range(4)] for _ in range(5)]
    slab, pencil = _part_arrays(P, glob, parts_here, -7.0)
    mv = S.SlabMoves(P, comm, lambda s, r: slab[s][r], lambda s, r: pencil[s][r])
    mv.slab_halo(S.ROLE_TEMP_IN)
    mv.to_pencils([(S.ROLE_HALF, S.ROLE_HALF), (S.ROLE_TEMP_IN, S.ROLE_NEXT)])
    for r in parts_here:
        for v in range(4):
            pencil[r][S.ROLE_NEXT][v] += 1000.0 * (r + 1)
    mv.to_slabs([(S.ROLE_NEXT, S.ROLE_CUR)])
    mv.pencil_halo(S.ROLE_HALF)
    return glob, slab, pencil


def _check_moves(P, glob, slab, pencil, parts_here):
    for s in parts_here:
        x0, x1, lo, hi = P.slab(s)
        for v in range(4):
            t = slab[s][S.ROLE_TEMP_IN][v].numpy()
            assert np.array_equal(t, glob[S.ROLE_TEMP_IN][v][lo:hi])          # ghosts = neighbours' planes
            c = slab[s][S.ROLE_CUR][v].numpy()[x0 - lo:x1 - lo]
            want = glob[S.ROLE_TEMP_IN][v][x0:x1].copy()
            for r in range(P.parts):
                y0, y1, _, _ = P.pencil(r)
                want[:, y0:y1] += 1000.0 * (r + 1)
            assert np.array_equal(c, want)                                    # pencil -> slab
    for r in parts_here:
        y0, y1, plo, phi = P.pencil(r)
        for v in range(4):
            assert np.array_equal(pencil[r][S.ROLE_HALF][v].numpy(), glob[S.ROLE_HALF][v][:, plo:phi])


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "..", "cmc-fluid-solver_b200"))
    import torch.distributed as dist
    from adi_b200 import slabs as S2
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        P = S2.SlabPlan(23, 20, 9, world)
        glob, slab, pencil = _run_moves(P, S2.DistComm(), [rank])
        _check_moves(P, glob, slab, pencil, [rank])
        q.put((rank, "ok"))
    except Exception as e:   # reported to the test process
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_block_moves_over_two_gloo_ranks():
    # the single-process moves first
    P = S.SlabPlan(23, 20, 9, 2)
    glob, slab, pencil = _run_moves(P, S.LocalComm(2), [0, 1])
    _check_moves(P, glob, slab, pencil, [0, 1])
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert res == {0: "ok", 1: "ok"}, res


@pytest.mark.gpu
@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("case", ["exact-fp32", "fast-fp64", "fast-fp32-tiles"])
def test_split_step_equals_single_domain(adi_lib, parts, case):
    from adi_b200 import _abi
    d = G.spheres_channel(dims=(64, 48, 32), n_spheres=5, rmin=3.0, rmax=6.0, seed=21)
    solver = _abi.ADI_SOLVER_EXACT if case.startswith("exact") else _abi.ADI_SOLVER_FAST
    prec = _abi.ADI_FP64 if "fp64" in case else _abi.ADI_FP32
    shapes = None
    if case == "fast-fp64":
        shapes = [(8, 8), (8, 8), (8, 8)]          # the generic chunked kernel
    elif case == "fast-fp32-tiles":
        shapes = [(4, -8), (4, -1), (4, 0)]        # TMA X tiles, element-copied Y tiles, warp-resident Z
    kw = dict(Re=180.0, Pr=0.72, lam=1.4, precision=prec, solver=solver)
    whole = adi_lib.AdiSolver3D(d, **kw)
    whole.CreateSegments()
    if shapes:
        for dr, (K, NL) in enumerate(shapes):
            whole.set_fast_shape(dr, K, NL)
    split = S.SlabSolver(d, parts, shapes=shapes, **kw)
    for i in range(3):
        ce = i != 1
        assert whole.step(6e-4, 3, 2, ce) == 0
        assert split.step(6e-4, 3, 2, ce) == 0
        for a, b in zip(whole.fields(0), split.fields()):
            assert np.array_equal(a, b), i
        if ce:
            assert split.div_error() == pytest.approx(whole.div_error(), rel=1e-12)
    split.close()
