"""World-size-2 process groups (gloo, CPU): sharding of independent units,
max-over-ranks timing and result gathering, as bench.py and batched runs use
them across GPUs.  The per-unit work here is the oracle's CPU Poisson solve
on small grids, so each rank's results can be checked against a
single-process run."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gpaw_b200.replicas import shard_by_cost


def test_shard_covers_every_unit_once():
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 100, 37)
    parts = [shard_by_cost(costs, 3, r) for r in range(3)]
    allidx = sorted(i for p in parts for i in p)
    assert allidx == list(range(37))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) - min(loads) <= costs.max()


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from gpaw_b200.replicas import gather_results, max_over_ranks
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        Ns = [(8, 8, 8), (8, 6, 8), (6, 8, 10), (10, 8, 8), (8, 8, 6)]
        idx = shard_by_cost([np.prod(N) for N in Ns], world, rank)
        local = []
        for i in idx:
            gd = L.GridDescriptor(Ns[i], (3.0, 3.0, 3.0), 0)
            rho = np.random.default_rng(i).standard_normal(tuple(gd.n_c))
            rho -= rho.mean()
            ps = L.FDPoissonSolver(eps=1e-16, be='port')
            ps.set_grid_descriptor(gd)
            phi = gd.zeros()
            n = ps.solve_neutral(phi, rho)
            local.append((i, n, float(np.abs(phi).sum())))
        t = max_over_ranks(0.1 * (rank + 1))
        res = gather_results(local)
        q.put((rank, t, res))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q))
             for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    # both ranks agree on the slowest rank's time and on the merged results
    assert out[0][1] == out[1][1] == pytest.approx(0.2)
    assert out[0][2] == out[1][2]
    assert [r[0] for r in out[0][2]] == list(range(5))
    # same numbers as a single process
    from oracle import gpaw_layer as L
    Ns = [(8, 8, 8), (8, 6, 8), (6, 8, 10), (10, 8, 8), (8, 8, 6)]
    for i, n, s in out[0][2]:
        gd = L.GridDescriptor(Ns[i], (3.0, 3.0, 3.0), 0)
        rho = np.random.default_rng(i).standard_normal(tuple(gd.n_c))
        rho -= rho.mean()
        ps = L.FDPoissonSolver(eps=1e-16, be='port')
        ps.set_grid_descriptor(gd)
        phi = gd.zeros()
        assert ps.solve_neutral(phi, rho) == n
        assert float(np.abs(phi).sum()) == s
