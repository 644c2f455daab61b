"""Serving loop: request generation (CPU) and, on the GPU, continuous
batching with every result equal to the same request served alone."""
import numpy as np
import pytest

from gpaw_b200.serving import Request, latency_stats, make_requests


def test_request_stream_properties():
    reqs = make_requests(rate=500.0, count=400, seed=3)
    sides = np.array([r.N[0] for r in reqs])
    assert ((sides % 8) == 0).all()
    assert sides.min() >= 24 and sides.max() <= 160
    t = np.array([r.arrival for r in reqs])
    assert (np.diff(t) > 0).all()
    # mean inter-arrival close to 1 / rate
    assert abs(np.diff(t).mean() * 500.0 - 1.0) < 0.15
    kinds = {r.kind for r in reqs}
    assert kinds == {'poisson', 'apply'}
    # log-uniform: more small grids than large ones
    assert (sides <= 64).sum() > (sides >= 112).sum()


def test_latency_stats():
    reqs = [Request(i, 'apply', (8, 8, 8), arrival=0.1 * i) for i in range(10)]
    for r in reqs:
        r.done = r.arrival + 0.01 * (r.rid + 1)
    s = latency_stats(reqs)
    assert s['requests'] == 10
    assert abs(s['p50_ms'] - 55.0) < 1e-6
    assert s['p99_ms'] > 99.0


@pytest.mark.gpu
def test_mixed_equals_alone(cuda):
    from gpaw_b200.serving import Server
    reqs = make_requests(rate=5000.0, count=24, seed=5, smin=24, smax=64)
    srv = Server(hbm_budget=2 << 30, nslots=6)
    srv.warm(sorted({r.N for r in reqs}))
    inputs = {r.rid: srv.host_input(r) for r in reqs}
    mixed = {r.rid: r.result for r in srv.run(reqs, inputs)}
    # the same requests one at a time
    alone = {}
    for r in reqs:
        one = Request(r.rid, r.kind, r.N, 0.0, r.seed)
        alone[r.rid] = srv.run([one], {r.rid: inputs[r.rid]})[0]
    for r in reqs:
        assert np.array_equal(mixed[r.rid], alone[r.rid].result), r
        if r.kind == 'poisson':
            assert alone[r.rid].niter > 0
    stats = latency_stats(reqs)
    assert stats['requests'] == 24


@pytest.mark.gpu
def test_no_grow_waits_for_a_resident_solver(cuda):
    """With grow=False the loop builds no solver while serving: three solves
    of one shape share its single resident solver one after another, the
    apply request runs past them, and every result equals the request
    served alone."""
    from gpaw_b200.serving import Server
    reqs = [Request(i, 'poisson', (32, 32, 32), 0.0, seed=11 + i)
            for i in range(3)]
    reqs.append(Request(3, 'apply', (40, 40, 40), 0.0, seed=9))
    srv = Server(hbm_budget=1 << 30, nslots=4, grow=False)
    srv.warm([(32, 32, 32), (40, 40, 40)], per_shape=1)
    inputs = {r.rid: srv.host_input(r) for r in reqs}
    out = srv.run(reqs, inputs)
    assert len(srv.pools[('poisson', (32, 32, 32))]) == 1
    solves = sorted((r for r in out if r.kind == 'poisson'),
                    key=lambda r: r.start)
    for a, b in zip(solves, solves[1:]):
        assert b.start >= a.done
    got = {r.rid: r.result for r in out}
    for r in reqs:
        one = Request(r.rid, r.kind, r.N, 0.0, r.seed)
        alone = srv.run([one], {r.rid: inputs[r.rid]})[0]
        assert np.array_equal(got[r.rid], alone.result)


@pytest.mark.gpu
def test_anisotropic_stream_with_eviction(cuda):
    """Anisotropic requests (each axis its own side) on a loop that builds
    solvers on demand under a budget too small to keep them all: solvers
    are evicted least recently used first, every result equals the request
    served alone, and the budget holds."""
    from gpaw_b200.serving import Server
    reqs = make_requests(rate=5000.0, count=20, seed=8, smin=24, smax=56,
                         poisson_fraction=0.8, anisotropic=True)
    assert any(len(set(r.N)) > 1 for r in reqs)
    srv = Server(hbm_budget=24 << 20, nslots=4, grow=True)
    inputs = {r.rid: srv.host_input(r) for r in reqs}
    mixed = {r.rid: r.result for r in srv.run(reqs, inputs)}
    assert srv.built > 0 and srv.evicted > 0
    assert srv.resident <= srv.budget + Server.solver_bytes((56, 56, 56))
    for r in reqs:
        one = Request(r.rid, r.kind, r.N, 0.0, r.seed)
        alone = srv.run([one], {r.rid: inputs[r.rid]})[0]
        assert np.array_equal(mixed[r.rid], alone.result), r
