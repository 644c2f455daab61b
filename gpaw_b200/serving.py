"""Continuous-batching request loop for Poisson solves and FD applications.

Requests arrive over time (``Request.arrival``, seconds after start).  The
loop admits an arrived request as soon as a slot (a CUDA stream) is free and
its memory fits the HBM budget, and keeps admitting while earlier requests
are still running, so the work of many requests overlaps on the GPU.  Each
request brings its input from pinned host memory and gets its result back
into pinned host memory: its latency is completion minus arrival, measured
on the host clock.

Solvers and operators are kept resident per grid shape (a pool of
instances, one per concurrently running request of that shape), so the
multigrid hierarchies, their buffers and their captured CUDA graphs are
built once and reused.  Building a solver allocates device memory and
captures a graph, which stalls the loop; with ``grow=False`` the loop never
builds one while serving: a solve whose shape has no free solver waits, and
later arrivals that can run are admitted past it.  Every kernel is
deterministic and a request never shares a buffer with another, so a
request's result does not depend on what else runs beside it.
"""
from __future__ import annotations

import collections
import dataclasses
import gc
import queue
import sys
import threading
import time
from math import pi

import numpy as np
import torch


@dataclasses.dataclass
class Request:
    rid: int
    kind: str            # 'poisson' (mixed-precision solve) or 'apply'
    N: tuple             # grid points per axis (zero boundaries)
    arrival: float       # seconds after the start of the run
    seed: int = 0
    # filled in by the server
    start: float = 0.0
    done: float = 0.0
    niter: int = 0
    result: np.ndarray = None


def make_requests(rate, count, seed=0, poisson_fraction=0.5, smin=24,
                  smax=160, anisotropic=False):
    """Poisson-process arrivals at `rate` per second; grid side log-uniform
    in [smin, smax], rounded to a multiple of 8 (so every grid has at least
    three multigrid levels); with `anisotropic` each axis draws its own
    side."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))

    def side():
        x = np.exp(rng.uniform(np.log(smin), np.log(smax)))
        return int(max(smin, min(smax, 8 * round(x / 8))))

    out = []
    for i in range(count):
        N = tuple(side() for _ in range(3)) if anisotropic else (side(),) * 3
        kind = 'poisson' if rng.random() < poisson_fraction else 'apply'
        out.append(Request(i, kind, N, float(t[i]), int(rng.integers(1 << 30))))
    return out


class Server:
    """Continuous-batching loop on one GPU.

    hbm_budget: bytes of device memory the loop may hold for requests and
    their resident solvers; nslots: requests in flight at most."""

    SPACING = 0.18 / 0.52917721   # Bohr

    def __init__(self, hbm_budget=8 << 30, nslots=8, tol=1e-10,
                 device=None, grow=True, pool=True, background=True):
        self.device = torch.device(device if device is not None else 'cuda')
        self.budget = int(hbm_budget)
        self.tol = tol
        self.grow = grow
        self.streams = [self._make_stream() for _ in range(nslots)]
        self.free_slots = list(range(nslots))
        self.pools = collections.defaultdict(list)   # (kind, N) -> free objs
        self.resident = 0        # bytes held by pooled solvers/operators
        self.in_use = 0          # bytes held by running requests
        self.ops = {}            # N -> Laplace for apply requests
        # one input/output slab per slot, sized before serving starts, so
        # that the loop allocates no device memory (an allocation can stall
        # every stream)
        self.slabs = [None] * nslots
        # resident solvers by last use (oldest first), for eviction when a
        # new shape needs room under the budget; counters of the run
        self.lru = collections.OrderedDict()     # id(solver) -> (N, solver)
        self.built = 0
        self.evicted = 0
        # solvers are built and evicted through the library's caching
        # allocator while the loop runs (an evicted solver is idle), so a
        # new shape costs no driver allocation and no device-wide sync
        self.pool = pool
        # with `background`, a solver for a new shape is built (and its
        # solve captured) by a builder thread while the loop keeps serving;
        # the request waits for it, later arrivals pass it
        self.background = background
        self.building = set()

    # -- resources ---------------------------------------------------------
    def _gd(self, N):
        from .grid_descriptor import GridDescriptor
        return GridDescriptor(N, tuple(n * self.SPACING for n in N), 0,
                              device=self.device)

    @staticmethod
    def request_bytes(req):
        n = int(np.prod([x - 1 for x in req.N]))
        return 2 * 8 * n     # input and output array

    @staticmethod
    def solver_bytes(N):
        n = int(np.prod([x - 1 for x in N]))
        return 48 * n        # FP64 copies, FP32 levels, scratch (estimate)

    def _make_stream(self):
        return torch.cuda.Stream(device=self.device)

    def _alloc_outputs(self, reqs, inputs):
        return {r.rid: torch.empty(tuple(inputs[r.rid].shape),
                                   dtype=torch.float64).pin_memory()
                for r in reqs}

    def _sync(self):
        torch.cuda.synchronize()

    def _new_solver(self, N):
        from .poisson import MixedPoissonSolver
        # per-level coarse kernels: concurrent solves run side by side,
        # where a cooperative coarse kernel (one block on every SM) would
        # wait for the whole GPU
        ps = MixedPoissonSolver(nn=3, tol=self.tol, levels=4,
                                fused_coarse=False)
        ps.set_grid_descriptor(self._gd(N))
        return ps

    def _take_solver(self, req):
        pool = self.pools[('poisson', req.N)]
        if pool:
            ps = pool.pop()
            self.lru.pop(id(ps), None)
            return ps, 0
        ps = self._new_solver(req.N)
        self.built += 1
        return ps, self.solver_bytes(req.N)

    def _builder(self, todo, done, device_index):
        """Builder thread: a solver per shape taken from `todo`, its solve
        captured, handed back through `done` (None ends the thread).  Any
        failure goes back through `done` too, so that the loop raises it
        instead of waiting for a build that will not come."""
        try:
            if device_index is not None:
                torch.cuda.set_device(device_index)
        except BaseException as exc:
            done.put((None, exc))
            return
        while True:
            N = todo.get()
            if N is None:
                return
            try:
                ps = self._new_solver(N)
                ps.prepare()
                done.put((N, ps))
            except BaseException as exc:      # re-raised by the loop
                done.put((N, exc))

    def _evict_for(self, need, keep=None):
        """Free idle resident solvers, least recently used first, until
        `need` more bytes fit the budget; False when they cannot.  Solvers
        of shape `keep` (the one the request is about to take) stay."""
        for key in list(self.lru):
            if self.resident + self.in_use + need <= self.budget:
                break
            N, ps = self.lru[key]
            if N == keep:
                continue
            del self.lru[key]
            self.pools[('poisson', N)].remove(ps)
            self.resident -= self.solver_bytes(N)
            self.evicted += 1
        return self.resident + self.in_use + need <= self.budget

    def _pooled(self):
        from contextlib import nullcontext
        from ._lib import solver_pool
        return solver_pool(self.budget) if self.pool else nullcontext()

    def warm(self, shapes, per_shape=2):
        """Build `per_shape` resident solvers (graphs captured) and one
        operator per shape ahead of time, run each once, and size the
        slot slabs."""
        with self._pooled():
            self._warm(shapes, per_shape)

    def _warm(self, shapes, per_shape):
        for N in shapes:
            built = []
            for _ in range(per_shape):
                req = Request(-1, 'poisson', N, 0.0)
                ps, nb = self._take_solver(req)
                self.resident += nb
                phi = ps.gd.zeros()
                rho = ps.gd.zeros()
                rho[0, 0, 0] = 1.0
                rho -= rho.mean()
                try:
                    ps.solve_neutral(phi, rho)
                except RuntimeError:
                    pass
                built.append(ps)
            self.pools[('poisson', N)].extend(built)
            for ps in built:
                self.lru[id(ps)] = (N, ps)
            # first launch of each kernel loads it (lazy module loading):
            # do that here, not while serving
            op = self._op(N)
            x = op.gd.zeros()
            op.apply(x, op.gd.zeros())
        self.reserve(shapes)

    def reserve(self, shapes):
        """Size every slot's input/output slab for the largest of `shapes`
        (call before serving; allocates)."""
        n = max(int(np.prod([x - 1 for x in N])) for N in shapes)
        for i, sl in enumerate(self.slabs):
            if sl is None or sl.numel() < 2 * n:
                self.slabs[i] = torch.empty(2 * n, dtype=torch.float64,
                                            device=self.device)
        torch.cuda.synchronize()

    def _op(self, N):
        from .fd_operators import Laplace
        if N not in self.ops:
            self.ops[N] = Laplace(self._gd(N), -0.25 / pi, 3)
        return self.ops[N]

    # -- inputs --------------------------------------------------------------
    def host_input(self, req):
        """Pinned host input of a request: a neutral sum of Gaussians for a
        solve, N(0,1) values for an apply (seeded per request)."""
        from .workloads import neutral_density_device
        gd = self._gd(req.N)
        if req.kind == 'poisson':
            a = neutral_density_device(gd, 8, req.seed).cpu()
        else:
            a = torch.from_numpy(np.random.default_rng(req.seed)
                                 .standard_normal(tuple(int(x)
                                                        for x in gd.n_c)))
        return a.pin_memory()

    # -- one request ----------------------------------------------------------
    def _launch(self, req, host_in, host_out, slot):
        st = self.streams[slot]
        shape = tuple(host_in.shape)
        n = int(np.prod(shape))
        slab = self.slabs[slot]
        with torch.cuda.stream(st):
            x = slab[:n].view(shape)
            y = slab[n:2 * n].view(shape)
            x.copy_(host_in, non_blocking=True)
            solver = None
            extra = 0
            if req.kind == 'poisson':
                solver, extra = self._take_solver(req)
                self.resident += extra      # the new solver stays resident
                y.zero_()
                solver.solve_neutral_async(y, x)
            else:
                self._op(req.N).apply(x, y)
            out = host_out
            out.copy_(y, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(st)
        return {'req': req, 'slot': slot, 'event': ev, 'solver': solver,
                'out': out, 'keep': (x, y), 'extra': extra}

    def _finish(self, job, now):
        req = job['req']
        req.done = now
        req.result = self._result_of(job)
        if job['solver'] is not None:
            req.niter = job['solver'].result()
            self.pools[('poisson', req.N)].append(job['solver'])
            self.lru[id(job['solver'])] = (req.N, job['solver'])
        self.in_use -= self.request_bytes(req)
        self.free_slots.append(job['slot'])

    def _result_of(self, job):
        return job['out'].numpy()     # the request's own pinned buffer

    # -- the loop --------------------------------------------------------------
    def run(self, requests, inputs=None):
        """Serve `requests` in arrival order; returns them with start/done
        times (seconds after the run began) and results."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        if inputs is None:
            inputs = {r.rid: self.host_input(r) for r in reqs}
        outputs = self._alloc_outputs(reqs, inputs)
        self.reserve({r.N for r in reqs})
        pending = list(reqs)
        active = []
        self._sync()
        # no garbage-collector pauses inside the loop (it allocates little:
        # per-request bookkeeping only)
        gc_was_on = gc.isenabled()
        gc.collect()
        gc.disable()
        self._todo = self._done = None
        thread = None
        switch = sys.getswitchinterval()
        if self.background and self.grow:
            self._todo, self._done = queue.Queue(), queue.Queue()
            index = None
            if self.device.type == 'cuda':
                index = (self.device.index if self.device.index is not None
                         else torch.cuda.current_device())
            thread = threading.Thread(target=self._builder,
                                      args=(self._todo, self._done, index),
                                      daemon=True)
            thread.start()
            # the loop and the builder share the interpreter: short slices
            # keep the loop's polling prompt while the builder runs
            sys.setswitchinterval(1e-4)
        try:
            with self._pooled():
                return self._serve(pending, active, inputs, outputs)
        finally:
            if thread is not None:
                self._todo.put(None)
                thread.join()
                sys.setswitchinterval(switch)
                self._install_built()
                # solvers built but not used in this run become evictable
                for (kind, N), pool in self.pools.items():
                    for ps in pool:
                        if id(ps) not in self.lru:
                            self.lru[id(ps)] = (N, ps)
            if gc_was_on:
                gc.enable()

    def _install_built(self):
        """Solvers finished by the builder thread join the pools; True when
        any did."""
        got = False
        while self._done is not None:
            try:
                N, ps = self._done.get_nowait()
            except queue.Empty:
                break
            self.building.discard(N)
            if isinstance(ps, BaseException):
                raise ps
            self.built += 1
            # not in the eviction order until a request has used it: the
            # request that asked for it is still waiting (otherwise two
            # waiting requests could evict each other's new solvers
            # before either runs)
            self.pools[('poisson', N)].append(ps)
            got = True
        return got

    def _serve(self, pending, active, inputs, outputs):
        reqs = list(pending)
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            progressed = self._install_built()
            for job in list(active):
                if job['event'].query():
                    active.remove(job)
                    self._finish(job, time.perf_counter() - t0)
                    progressed = True
            # admit arrived requests in arrival order; a solve whose shape
            # has no free solver (and may not build one) lets later ones by
            i = 0
            while i < len(pending) and pending[i].arrival <= now and \
                    self.free_slots:
                req = pending[i]
                pooled = bool(self.pools[('poisson', req.N)])
                if req.kind == 'poisson' and not pooled and not self.grow:
                    i += 1
                    continue
                if req.kind == 'poisson' and not pooled and \
                        self._todo is not None:
                    # built by the builder thread; the request waits for it
                    if req.N not in self.building:
                        need = self.solver_bytes(req.N)
                        # over the budget only when nothing else could
                        # ever free memory (as the synchronous path does)
                        if self.resident + self.in_use + need <= \
                                self.budget or self._evict_for(need) or \
                                not (active or self.building):
                            self.building.add(req.N)
                            self.resident += need
                            self._todo.put(req.N)
                    i += 1
                    continue
                need = self.request_bytes(req)
                if req.kind == 'poisson' and not pooled:
                    need += self.solver_bytes(req.N)
                keep = req.N if (req.kind == 'poisson' and pooled) else None
                if self.resident + self.in_use + need > self.budget and \
                        not self._evict_for(need, keep) and active:
                    break      # wait for memory to free up
                del pending[i]
                slot = self.free_slots.pop()
                self.in_use += self.request_bytes(req)
                req.start = time.perf_counter() - t0
                active.append(self._launch(req, inputs[req.rid],
                                           outputs[req.rid], slot))
                progressed = True
            if not progressed:
                time.sleep(20e-6)
        return reqs


def latency_stats(reqs):
    lat = np.array([r.done - r.arrival for r in reqs])
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    return {'requests': len(reqs), 'throughput_per_s': len(reqs) / span,
            'p50_ms': float(np.percentile(lat, 50) * 1e3),
            'p99_ms': float(np.percentile(lat, 99) * 1e3),
            'mean_ms': float(lat.mean() * 1e3)}
