"""Many independent Poisson solves on grids of uneven sizes, overlapped on
one GPU.

Each grid gets its own solver: its own device-resident level hierarchy,
buffers and captured V-cycle loop (the whole solve runs on the device, see
gb_poisson_* / gb_mixed_*).  A mixed-precision batch is, by default, ONE
CUDA graph with a branch per grid (gb_mixed_batch_*): a single launch runs
every solve, the branches side by side.  Otherwise (FP64, or graph=False)
the batch enqueues every solve on one of ``nstreams`` CUDA streams.  Either
way there is no host synchronisation until the results are read.
"""
from __future__ import annotations

import numpy as np
import torch

import ctypes as C

from ._lib import check, solver_pool
from .cgpaw import _stream
from .poisson import FDPoissonSolver, MixedPoissonSolver


class PoissonBatch:
    def __init__(self, gds, nn=3, tol=1e-10, precision='mixed', nstreams=16,
                 maxiter=400, levels=4, graph=True):
        if precision not in ('mixed', 'fp64'):
            raise ValueError("precision must be 'mixed' or 'fp64'")
        self.gds = list(gds)
        self.tol = tol
        self.precision = precision
        self.solvers = []
        # hundreds of solvers are built at once: through the library's
        # caching allocator, which carves their buffers from a few slabs
        with solver_pool():
            self._build(nn, tol, maxiter, levels, precision)
        dev = self.gds[0].device if self.gds else torch.device('cuda')
        self.streams = [torch.cuda.Stream(device=dev)
                        for _ in range(max(1, nstreams))]
        self._batch = None
        if precision == 'mixed' and graph and self.solvers:
            lib = self.solvers[0]._h.lib
            hs = (C.c_void_p * len(self.solvers))(
                *[ps._h.h for ps in self.solvers])
            h = C.c_void_p()
            check(lib.gb_mixed_batch_new(len(self.solvers), hs, float(tol),
                                         int(maxiter), C.byref(h)))
            self._batch = (lib, h)

    def _build(self, nn, tol, maxiter, levels, precision):
        for gd in self.gds:
            if precision == 'mixed':
                # the coarse levels in one single-block kernel a solve: the
                # batch's solves run side by side, which cooperative kernels
                # (the whole GPU at once) would serialise
                ps = MixedPoissonSolver(nn=nn, tol=tol, maxiter=maxiter,
                                        levels=levels, fused_coarse='tail')
            else:
                ps = FDPoissonSolver(nn=nn, relax='J', eps=0.0,
                                     maxiter=maxiter)
            ps.set_grid_descriptor(gd)
            self.solvers.append(ps)

    def __del__(self):
        b = getattr(self, '_batch', None)
        if b is not None and b[1].value:
            b[0].gb_mixed_batch_free(b[1])
            self._batch = None

    def prepare(self, rhos):
        """FP64 batches stop at ||L phi - rho|| <= tol ||rho|| through the
        reference's absolute criterion sum(r^2) dv <= eps: compute each
        grid's eps once (one host synchronisation)."""
        self._eps = [self.tol**2 * float((r * r).sum()) * ps.gd.dv
                     for ps, r in zip(self.solvers, rhos)]

    def enqueue(self, phis, rhos):
        """Enqueue every solve; returns immediately (after prepare() for an
        FP64 batch)."""
        if len(phis) != len(self.solvers) or len(rhos) != len(self.solvers):
            raise ValueError('one phi and one rho per grid')
        if self.precision == 'fp64' and getattr(self, '_eps', None) is None:
            self.prepare(rhos)
        if self._batch is not None:
            lib, h = self._batch
            n = len(self.solvers)
            for ps, phi, rho in zip(self.solvers, phis, rhos):
                if not (phi.is_contiguous() and rho.is_contiguous()) or \
                        tuple(phi.shape) != tuple(ps.gd.n_c):
                    raise ValueError('contiguous arrays of each grid\'s shape')
            pp = (C.c_void_p * n)(*[p.data_ptr() for p in phis])
            rr = (C.c_void_p * n)(*[r.data_ptr() for r in rhos])
            self._keep = (phis, rhos)
            check(lib.gb_mixed_batch_solve_async(h, pp, rr, _stream()))
            return
        cur = torch.cuda.current_stream()
        for st in self.streams:
            st.wait_stream(cur)
        for i, (ps, phi, rho) in enumerate(zip(self.solvers, phis, rhos)):
            with torch.cuda.stream(self.streams[i % len(self.streams)]):
                if self.precision == 'mixed':
                    ps.solve_neutral_async(phi, rho)
                else:
                    ps.solve_neutral_async(phi, rho, eps=self._eps[i])
        for st in self.streams:
            cur.wait_stream(st)

    def results(self):
        """V-cycle counts (after the enqueued work completed)."""
        torch.cuda.synchronize()
        if self._batch is not None:
            lib, h = self._batch
            n = len(self.solvers)
            ni = (C.c_int * n)()
            rel = (C.c_double * n)()
            check(lib.gb_mixed_batch_result(h, ni, rel))
            return list(ni)
        return [ps.result() for ps in self.solvers]

    def solve(self, phis, rhos):
        self.enqueue(phis, rhos)
        n = self.results()
        for ps, phi in zip(self.solvers, phis):
            if ps.gd.pbc_c.all():
                phi -= phi.mean()
        return n


def c4_grids(count=512, seed=0, pbc=0, spacing=0.18, device=None):
    """Grid descriptors of the uneven batch: every side drawn uniformly from
    {32, 40, ..., 128} (anisotropic), spacing 0.18 A."""
    from .grid_descriptor import GridDescriptor
    from .workloads import BOHR
    rng = np.random.default_rng(seed)
    h = spacing / BOHR
    sides = rng.choice(np.arange(32, 129, 8), size=(count, 3))
    return [GridDescriptor(tuple(int(x) for x in N),
                           tuple(float(x) * h for x in N), pbc, device=device)
            for N in sides]
