"""Poisson solver with a spatially varying dielectric (drop-in for the
WeightedFDPoissonSolver of gpaw/old/solvation/poisson.py:75-124).

div(eps(r) grad phi(r)) = -4 pi rho(r) is solved by the FDPoissonSolver
V-cycle (gpaw/poisson.py:500-537) on weighted operators: every level's
operator is ``WeightedFDOperator([Laplace, d/dx, d/dy, d/dz])`` weighted by
eps and its three derivatives (the dielectric's ``eps_gradeps``); the
weights of each coarser level are the restrictions of the finer level's.
The relaxation sweeps, operator applications and grid transfers are the
sm_100a kernels of the weighted operator and the Transformer; the residual
updates are device arithmetic, and the level-0 error is read once per
V-cycle to decide whether to stop, as the reference does.

A charged system in a non-periodic cell is solved as the reference does:
a compensation charge built from a Gaussian and the dielectric
(``load_gauss``, :48-72) carries the charge, the neutral rest is solved,
and the Gaussian's potential (with the same normalisation) is added back.
Charged periodic systems raise NotImplementedError, as in the reference.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.special import erf

from ._lib import PoissonConvergenceError
from .fd_operators import Gradient, Laplace
from .gauss import SQRT_PI, coordinates
from .poisson import FDPoissonSolver, _solve_monopole
from .wfd_operators import WeightedFDOperator


class WeightedFDPoissonSolver(FDPoissonSolver):
    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 remove_moment=None, use_charge_center=False):
        if remove_moment is not None:
            raise NotImplementedError(
                'Removing arbitrary multipole moments is not implemented '
                'for SolvationPoissonSolver!')
        if nn == 'M':
            raise NotImplementedError(
                'Mehrstellen stencil is not implemented for '
                'SolvationPoissonSolver!')
        super().__init__(nn, relax, eps, maxiter)
        self.dielectric = None

    def set_dielectric(self, dielectric):
        """``dielectric.eps_gradeps``: [eps, d eps/dx, d eps/dy, d eps/dz],
        float64 CUDA tensors of the grid shape (kept, not copied)."""
        self.dielectric = dielectric
        self._graph = None

    def create_laplace(self, gd, scale=1.0, n=1, dtype=float):
        """:80-85: the Laplacian and the three gradients, weighted."""
        operators = [Laplace(gd, scale, n, dtype)]
        operators += [Gradient(gd, j, scale, n, dtype) for j in (0, 1, 2)]
        return WeightedFDOperator(operators)

    def get_description(self):
        return super().get_description().replace(
            'solver with', 'weighted FD solver with dielectric and')

    def _init(self):
        """:113-124 and gpaw/poisson.py:451-472: level 0 weighted by the
        dielectric, coarser levels by arrays that restrict_op_weights
        fills; work arrays of every level."""
        if self._initialized:
            return
        self._graph = None      # captured with the previous arrays
        if self.dielectric is None:
            raise RuntimeError('WeightedFDPoissonSolver: set_dielectric '
                               'first')
        self.operators[0].set_weights(list(self.dielectric.eps_gradeps))
        self.op_coarse_weights = []
        for operator in self.operators[1:]:
            weights = [operator.gd.empty() for _ in range(4)]
            self.op_coarse_weights.append(weights)
            operator.set_weights(weights)
        gd = self.gd
        self.rhos = [gd.empty()]
        self.phis = [None]
        self.residuals = [gd.empty()]
        for op in self.operators[1:]:
            self.phis.append(op.gd.empty())
            self.rhos.append(op.gd.empty())
            self.residuals.append(op.gd.empty())
        level = self.levels
        self.presmooths[level] = 8
        self.postsmooths[level] = 8
        self._initialized = True

    def restrict_op_weights(self):
        """:100-106: restrict the weights to the coarse grids."""
        self._init()
        weights = [self.operators[0].weights] + self.op_coarse_weights
        for i, res in enumerate(self.restrictors):
            for j in range(4):
                res.apply(weights[i][j], weights[i + 1][j])
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()

    def load_gauss(self, center=None):
        """:48-72: rho = eps g - (grad v_g . grad eps) / (4 pi) for the
        normalised Gaussian g of gpaw/utilities/gauss.py and its potential
        v_g, both scaled so that rho carries sqrt(4 pi) of charge.  Host
        float64, as the reference computes it; the results live on the
        device."""
        epsr, dx_epsr, dy_epsr, dz_epsr = [
            t.detach().cpu().numpy() for t in self.dielectric.eps_gradeps]
        gd = self.gd
        xyz, r2 = coordinates(gd, center)
        r = np.sqrt(r2)
        if center is None:
            a = 4 * 19.0 * (gd.icell_cv**2).sum(1).max()
        else:
            cell_center = gd.cell_cv.sum(1) / 2
            r_min = (cell_center - np.abs(center - cell_center)).min()
            a = 19.0 / r_min**2
        rho_g = np.sqrt(a**3 * 4) / np.pi * np.exp(-a * r2)
        phi_g = 2.0 * SQRT_PI * erf(np.sqrt(a) * r) / r
        x, y, z = xyz
        fac = 2. * np.sqrt(a) * np.exp(-a * r2)
        fac /= np.sqrt(np.pi) * r2
        fac -= erf(np.sqrt(a) * r) / (r2 * r)
        fac *= 2.0 * SQRT_PI
        sp = fac * x * dx_epsr + fac * y * dy_epsr + fac * z * dz_epsr
        rho = epsr * rho_g - 1. / (4. * np.pi) * sp
        invnorm = np.sqrt(4. * np.pi) / (rho.reshape(-1).sum() * gd.dv)
        dev = self.dielectric.eps_gradeps[0].device
        self.phi_gauss = torch.from_numpy(phi_g * invnorm).to(dev)
        self.rho_gauss = torch.from_numpy(rho * invnorm).to(dev)
        self._gauss_gd = gd

    def solve(self, phi, rho, charge=None, maxcharge=1e-6,
              zero_initial_phi=False, timer=None):
        """:87-98 and gpaw/poisson.py:182-283: neutral systems, and charged
        ones in a non-periodic cell."""
        self._init()
        actual_charge = self.gd.integrate(rho)
        if bool(self.gd.pbc_c.all()) and abs(actual_charge) > maxcharge:
            raise NotImplementedError(
                'charged periodic systems are not implemented')
        self.restrict_op_weights()
        if charge is None:
            charge = actual_charge
        if abs(charge) <= maxcharge:
            background = (actual_charge / self.gd.dv /
                          self.gd.get_size_of_global_array().prod())
            return self.solve_neutral(phi, rho - background)
        if not bool(self.gd.pbc_c.any()):
            if getattr(self, '_gauss_gd', None) is not self.gd:
                self.load_gauss()
            return _solve_monopole(self, phi, rho, actual_charge,
                                   zero_initial_phi)
        raise NotImplementedError(
            'charged system with mixed boundary conditions')

    def _vcycle_graph(self, like):
        """One V-cycle (iterate2 on the solver's own level-0 arrays, the
        squared residual left on the device) captured as a CUDA graph, so
        that a V-cycle costs one graph launch and one scalar read instead
        of some sixty launches from Python.  Built on first use; the
        weights it reads are the solver's arrays, refreshed in place by
        restrict_op_weights."""
        g = getattr(self, '_graph', None)
        if g is not None and self._graph_phi.device == like.device:
            return g
        import torch
        self._graph_phi = torch.zeros_like(like)
        self._graph_err = torch.zeros((), dtype=like.dtype,
                                      device=like.device)

        def body():
            self.phis[0] = self._graph_phi
            self._cycle_no_read(0)
            r = self.residuals[0].reshape(-1)
            self._graph_err.copy_(torch.dot(r, r))

        side = torch.cuda.Stream(device=like.device)
        side.wait_stream(torch.cuda.current_stream())
        saved = self._graph_phi.clone()
        with torch.cuda.stream(side):
            body()                        # allocates scratch, loads kernels
        torch.cuda.current_stream().wait_stream(side)
        self._graph_phi.copy_(saved)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            body()
        self._graph = g
        return g

    def _cycle_no_read(self, level):
        """iterate2's V-cycle below `level` without the final host read."""
        residual = self.residuals[level]
        op = self.operators[level]
        if level < self.levels:
            op.relax(self.relax_method, self.phis[level], self.rhos[level],
                     self.presmooths[level], self.weights[level])
            op.apply(self.phis[level], residual)
            residual -= self.rhos[level]
            self.restrictors[level].apply(residual, self.rhos[level + 1])
            self.phis[level + 1].zero_()
            self._cycle_no_read(level + 1)
            self.interpolators[level].apply(self.phis[level + 1], residual)
            self.phis[level] -= residual
        op.relax(self.relax_method, self.phis[level], self.rhos[level],
                 self.postsmooths[level], self.weights[level])
        if level == 0:
            op.apply(self.phis[level], residual)
            residual -= self.rhos[level]

    def solve_neutral(self, phi, rho, timer=None):
        """gpaw/poisson.py:474-498.  On a GPU every V-cycle is one replay
        of a captured graph (GPAW_B200_WGRAPH=0: launched op by op)."""
        import os
        self._init()
        self.rhos[0].copy_(rho)
        if phi.is_cuda and os.environ.get('GPAW_B200_WGRAPH', '1') != '0':
            g = self._vcycle_graph(phi)
            self._graph_phi.copy_(phi)
            niter = 1
            while True:
                g.replay()
                err = float(self._graph_err) * self.gd.dv
                if not (err > self.eps and niter < self.maxiter):
                    break
                niter += 1
            phi.copy_(self._graph_phi)
            self.phis[0] = phi
        else:
            self.phis[0] = phi
            niter = 1
            while self.iterate2(self.step) > self.eps and \
                    niter < self.maxiter:
                niter += 1
        if niter == self.maxiter:
            raise PoissonConvergenceError(
                'Poisson solver did not converge in %d iterations!'
                % self.maxiter)
        if bool(self.gd.pbc_c.all()):
            phi -= phi.sum() / float(self.gd.n_c.prod())
        self.niter = niter
        return niter

    def iterate2(self, step, level=0, phi=None, rho=None):
        """gpaw/poisson.py:500-537: one V-cycle; at level 0 returns
        sum(r^2) dv."""
        self._init()
        if phi is not None:
            self.phis[0] = phi
        if rho is not None:
            self.rhos[0].copy_(rho)
        residual = self.residuals[level]
        op = self.operators[level]
        if level < self.levels:
            op.relax(self.relax_method, self.phis[level], self.rhos[level],
                     self.presmooths[level], self.weights[level])
            op.apply(self.phis[level], residual)
            residual -= self.rhos[level]
            self.restrictors[level].apply(residual, self.rhos[level + 1])
            self.phis[level + 1].zero_()
            self.iterate2(4.0 * step, level + 1)
            self.interpolators[level].apply(self.phis[level + 1], residual)
            self.phis[level] -= residual
        op.relax(self.relax_method, self.phis[level], self.rhos[level],
                 self.postsmooths[level], self.weights[level])
        if level == 0:
            op.apply(self.phis[level], residual)
            residual -= self.rhos[level]
            r = residual.reshape(-1)
            return float(torch.dot(r, r)) * self.gd.dv
