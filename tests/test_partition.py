"""Host-side sharding of a batch over ranks: LPT bin packing and the per-domain
gather, run as two gloo ranks on the CPU.  Each rank steps its share of a small
batch with the oracle (the stand-in for the GPU batch on a machine without one)
and rank 0 checks the gathered results against stepping every domain in one
process."""
import os
import socket

import numpy as np
import pytest

from adi_b200 import geometry as G
from adi_b200.partition import domain_cost, gather_per_domain, lpt_partition, part_loads


def test_lpt_partition_is_balanced_and_complete():
    rng = np.random.default_rng(2)
    shapes = [tuple(int(x) for x in rng.integers(64, 161, size=3)) for _ in range(64)]
    costs = [domain_cost(s, 4) for s in shapes]
    for n in (1, 2, 4, 8):
        parts = lpt_partition(costs, n)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = part_loads(costs, parts)
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(costs) / n + max(costs)
        assert parts == lpt_partition(costs, n)        # deterministic
    assert lpt_partition([5, 5, 4, 3, 3], 2) == [[0, 2], [1, 3, 4]]
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def _small_batch():
    return G.batch_of_domains(n_domains=6, seed=5, size_lo=10, size_hi=16, spheres=(1, 3), rmin=1.5, rmax=3.0)


def _step_all(domains, idx):
    import oracle as O
    out = {}
    for i in idx:
        d = domains[i]
        s = O.OracleSolver(d, precision=8, Re=d.meta["Re"], Pr=0.72, lam=1.4)
        assert s.step(5e-4, 2, 1, True) == 0
        out[i] = (float(s.div_error()), float(np.abs(s.fields(0)[0]).sum()))
    return out


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.join(here, "..", "cmc-fluid-solver_b200"), os.path.join(here, "..", "oracle"), here):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from adi_b200 import geometry as G2  # noqa: F401
    from adi_b200.partition import domain_cost as dc, gather_per_domain as gp, lpt_partition as lp
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        domains = _small_batch()
        parts = lp([dc(d.shape, 2) for d in domains], world)
        local = _step_all(domains, parts[rank])
        merged = gp(local, world)
        if rank == 0:
            q.put(merged)
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_batch_matches_single_process():
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    domains = _small_batch()
    want = _step_all(domains, range(len(domains)))
    assert sorted(merged) == sorted(want)
    for i in want:
        assert merged[i] == want[i]
    assert gather_per_domain({1: "a"}, 1) == {1: "a"}
