"""Many independent Poisson solves on grids of uneven sizes, overlapped on
one GPU.

Each grid gets its own solver: its own device-resident level hierarchy,
buffers and captured CUDA graph (the whole V-cycle loop runs on the device,
see gb_poisson_* / gb_mixed_*).  A batch enqueues every solve on one of
``nstreams`` CUDA streams without any host synchronisation, so solves of
small grids — each far too small to fill a B200 alone — run side by side;
one synchronisation at the end reads all results.
"""
from __future__ import annotations

import numpy as np
import torch

from .poisson import FDPoissonSolver, MixedPoissonSolver


class PoissonBatch:
    def __init__(self, gds, nn=3, tol=1e-10, precision='mixed', nstreams=16,
                 maxiter=400, levels=4):
        if precision not in ('mixed', 'fp64'):
            raise ValueError("precision must be 'mixed' or 'fp64'")
        self.gds = list(gds)
        self.tol = tol
        self.precision = precision
        self.solvers = []
        for gd in self.gds:
            if precision == 'mixed':
                ps = MixedPoissonSolver(nn=nn, tol=tol, maxiter=maxiter,
                                        levels=levels)
            else:
                ps = FDPoissonSolver(nn=nn, relax='J', eps=0.0,
                                     maxiter=maxiter)
            ps.set_grid_descriptor(gd)
            self.solvers.append(ps)
        dev = self.gds[0].device if self.gds else torch.device('cuda')
        self.streams = [torch.cuda.Stream(device=dev)
                        for _ in range(max(1, nstreams))]

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
