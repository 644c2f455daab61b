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


# ------------------------------------------------ the loop's scheduling (CPU)
class _Done:
    """An event that completes a fixed time after its launch."""

    def __init__(self, seconds):
        import time
        self.t = time.perf_counter() + seconds

    def query(self):
        import time
        return time.perf_counter() >= self.t


class _Solver:
    def __init__(self, N):
        self.N = N
        self.prepared = False

    def prepare(self):
        import time
        time.sleep(0.0005)
        self.prepared = True

    def result(self):
        return 3


def _host_server(**kw):
    """The serving loop with its device work replaced by timers: requests
    run for 0.1-0.3 ms, solvers are dummies that the builder thread
    prepares; the admission, budget, eviction and build logic is the
    product's."""
    import contextlib
    from gpaw_b200.serving import Server

    class HostServer(Server):
        def _make_stream(self):
            return None

        def _alloc_outputs(self, reqs, inputs):
            return {r.rid: None for r in reqs}

        def _sync(self):
            pass

        def reserve(self, shapes):
            pass

        def _pooled(self):
            return contextlib.nullcontext()

        def _new_solver(self, N):
            return _Solver(N)

        def _launch(self, req, host_in, host_out, slot):
            solver, extra = None, 0
            if req.kind == 'poisson':
                solver, extra = self._take_solver(req)
                self.resident += extra
                assert solver.prepared or not self.background
            return {'req': req, 'slot': slot, 'solver': solver,
                    'event': _Done(1e-4 * (1 + req.rid % 3)), 'out': None,
                    'extra': extra}

        def _result_of(self, job):
            return job['req'].rid

    return HostServer(**kw)


@pytest.mark.parametrize('background', [True, False])
def test_builds_and_evictions_always_finish(background):
    """Anisotropic streams under budgets from a few solvers to many: every
    request completes (no request waits forever for a solver that others
    keep evicting), solvers are built, and with a small budget evicted."""
    import threading
    for seed, budget in [(1, 12 << 20), (2, 24 << 20), (3, 256 << 20)]:
        reqs = make_requests(rate=20000.0, count=80, seed=seed, smin=24,
                             smax=56, poisson_fraction=0.8,
                             anisotropic=True)
        srv = _host_server(hbm_budget=budget, nslots=4, grow=True,
                           background=background, pool=False, device='cpu')
        t = threading.Thread(target=srv.run,
                             args=(reqs, {r.rid: None for r in reqs}),
                             daemon=True)
        t.start()
        t.join(timeout=60)
        assert not t.is_alive(), (seed, budget, 'the loop did not finish')
        assert all(r.done > 0 and r.result == r.rid for r in reqs)
        assert srv.built > 0
        if budget == 12 << 20:
            assert srv.evicted > 0
        assert not srv.building


def test_failed_build_is_raised_not_waited_for():
    """A solver build that fails in the builder thread ends the loop with
    that error instead of leaving its request waiting."""
    import threading
    reqs = make_requests(rate=20000.0, count=20, seed=4, smin=24, smax=48,
                         poisson_fraction=1.0, anisotropic=True)
    srv = _host_server(hbm_budget=1 << 30, nslots=4, grow=True,
                       background=True, pool=False, device='cpu')

    def broken(N):
        raise MemoryError('no room for a solver')
    srv._new_solver = broken
    err = []

    def go():
        try:
            srv.run(reqs, {r.rid: None for r in reqs})
        except MemoryError as e:
            err.append(e)
    t = threading.Thread(target=go, daemon=True)
    t.start()
    t.join(timeout=30)
    assert not t.is_alive() and err
