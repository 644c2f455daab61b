"""Poisson solver with extra vacuum around a non-periodic system.

Drop-in for ``gpaw.poisson_extravacuum.ExtraVacuumPoissonSolver``
(gpaw/poisson_extravacuum.py:13-232): same constructor, ``solve`` return
values and results.

Why: with zero boundaries the potential is forced to vanish on the cell
faces, which is wrong when the charge sits close to them.  Solving on a
larger grid (``gpts`` points per axis, the original grid centred inside)
moves that error away.  To keep the large solve cheap it can run
``coarses`` times coarser; the fine potential is then recovered in a
second, small solve on the original grid:

1. restrict the density ``coarses`` times, embed it in the large coarse
   grid (zeros around it) and solve there (warm-started from the previous
   call's large potential);
2. interpolate the large potential back to the fine spacing on a padded
   copy of the original grid (the "auxiliary" grid), apply the fine
   Laplacian to it, and cut both out over the original grid: a potential
   and the density it exactly belongs to under the fine stencil;
3. solve the original grid for the density minus that density, starting
   from the potential minus that potential, and add the potential back.
   The boundary values of step 3 come from the large solve; inside, the
   fine solve corrects what the coarse grid could not resolve.

The padding of the auxiliary grid is derived here from the stencils' reach
(``_exact_margin``): it is just wide enough that every value that reaches
the original grid is computed from the large solution and never from the
auxiliary grid's own zero boundary, so the result does not depend on it.
Restriction, interpolation, the Laplacian and the solves are the sm_100a
kernels; embedding and cutting are device copies.
"""
from __future__ import annotations

from math import pi

import numpy as np

from .fd_operators import Laplace
from .grid_descriptor import GridDescriptor
from .transformers import Transformer


def _solver(spec):
    """A Poisson solver object from an object or a dict description."""
    if spec is None or not isinstance(spec, dict):
        return spec
    kw = dict(spec)
    name = kw.pop('name', 'fd')
    if name != 'fd':
        raise ValueError(f'Unknown poisson solver: {name}')
    from .poisson import FDPoissonSolver
    return FDPoissonSolver(**kw)


class _Embedding:
    """A grid centred inside a larger grid with the same spacing and
    boundary conditions: (N_big - N) // 2 extra points below each axis
    (gpaw/utilities/extend_grid.py's layout)."""

    def __init__(self, inner, N_big):
        N_big = np.asarray(N_big, dtype=int)
        self.inner = inner
        self.outer = GridDescriptor(N_big, inner.h_cv * N_big[:, None],
                                    inner.pbc_c, device=inner.device)
        self.lo = (N_big - inner.N_c) // 2

    def window(self, big):
        """The view of a large-grid array over the inner grid."""
        o, n = self.lo, self.inner.n_c
        return big[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]]

    def embed(self, small):
        """A large-grid array that is `small` inside and zero outside."""
        big = self.outer.zeros()
        self.window(big).copy_(small)
        return big


def _exact_margin(nn_refine, nn_laplace, coarses):
    """Padding (fine points per side) of the auxiliary grid.

    The Laplacian of order nn_laplace reads nn_laplace points beyond the
    original grid, so the refined potential must be exact that far out.
    One order-2n interpolation step computes a fine point from coarse
    points at most 2n - 1 fine spacings away, so a margin of m fine points
    needs ceil((m + 2n - 1) / 2) coarse points.  Working back through the
    coarsenings gives the margin on the coarsest grid; times 2^coarses it
    is a whole number of coarse points, so the auxiliary grid's points
    coincide with the large coarse grid's."""
    m = nn_laplace
    for _ in range(coarses):
        m = -(-(m + 2 * nn_refine - 1) // 2)
    return m * 2**coarses


class ExtraVacuumPoissonSolver:
    def __init__(self, gpts, poissonsolver_large, poissonsolver_small=None,
                 coarses=0, nn_coarse=3, nn_refine=3, nn_laplace=3,
                 use_aux_grid=True, xp=None):
        self.N_large_fine_c = np.array(gpts, dtype=int)
        self.Ncoar = int(coarses)
        self.use_coarse = self.Ncoar > 0
        if not self.use_coarse:
            assert poissonsolver_small is None
        self.ps_large_coar = _solver(poissonsolver_large)
        self.ps_small_fine = (_solver(poissonsolver_small)
                              if self.use_coarse else None)
        self.nn_coarse = nn_coarse
        self.nn_refine = nn_refine
        self.nn_laplace = nn_laplace
        self.use_aux_grid = use_aux_grid
        self._phi_large = None

    def set_grid_descriptor(self, gd):
        if bool(gd.pbc_c.any()):
            raise NotImplementedError('Only non-periodic boundary '
                                      'conditions are tested')
        assert np.all(gd.N_c <= self.N_large_fine_c), \
            'extended grid has to be larger than the original one'
        self.gd_small_fine = gd
        k = self.Ncoar
        # restriction chain of the original grid: gds[0] = gd, gds[k] the
        # spacing of the large solve
        gds = [gd]
        for _ in range(k):
            gds.append(gds[-1].coarsen())
        self.down = [Transformer(gds[i], gds[i + 1], self.nn_coarse)
                     for i in range(k)]
        self.gd_small_coar = gds[-1]
        self.large = _Embedding(gds[-1], self.N_large_fine_c // 2**k)
        self.gd_large_coar = self.large.outer
        self.ps_large_coar.set_grid_descriptor(self.gd_large_coar)
        self._phi_large = None
        if not self.use_coarse:
            return
        self.ps_small_fine.set_grid_descriptor(gd)
        # the auxiliary grid: the original grid padded by the stencils'
        # reach, or the whole large grid at fine spacing when the padding
        # would not fit inside it
        N_aux = gd.N_c + 2 * _exact_margin(self.nn_refine, self.nn_laplace,
                                           k)
        if not self.use_aux_grid or np.any(N_aux > self.N_large_fine_c):
            self.use_aux_grid = False
            N_aux = self.N_large_fine_c
        self.aux = _Embedding(gd, N_aux)
        self.gd_aux_fine = self.aux.outer
        self.laplace_aux_fine = Laplace(self.gd_aux_fine, -0.25 / pi,
                                        self.nn_laplace)
        aux = [self.gd_aux_fine]
        for _ in range(k):
            aux.append(aux[-1].coarsen())
        # interpolation chain, coarsest first
        self.up = [Transformer(aux[i + 1], aux[i], self.nn_refine)
                   for i in reversed(range(k))]
        self.gd_aux_coar = aux[-1]
        # where the coarse auxiliary grid sits in the large coarse grid
        self.aux_in_large = _Embedding(aux[-1], self.gd_large_coar.N_c)

    def get_description(self):
        lines = ['ExtraVacuumPoissonSolver',
                 '    Large grid: %s' % ' x '.join(
                     str(N) for N in self.gd_large_coar.N_c),
                 '    ' + self.ps_large_coar.get_description()]
        if self.use_coarse:
            lines += ['    Small grid:',
                      '    ' + self.ps_small_fine.get_description()]
        return '\n'.join(lines)

    def _boundary_correction(self):
        """Potential and matching density over the original grid from the
        large solution (steps 2 of the module docstring)."""
        if self.use_aux_grid:
            phi = self.aux_in_large.window(self._phi_large).contiguous()
        else:
            phi = self._phi_large
        for t in self.up:
            phi = t.apply(phi)
        rho = self.gd_aux_fine.empty()
        self.laplace_aux_fine.apply(phi, rho)
        return self.aux.window(phi), self.aux.window(rho)

    def solve(self, phi, rho, **kwargs):
        """Returns the large solve's V-cycle count, or the pair (large,
        small) when the large grid is coarser."""
        if self._phi_large is None:
            # kept between calls: each large solve starts from the last
            self._phi_large = self.gd_large_coar.zeros()
        rho_c = rho
        for t in self.down:
            rho_c = t.apply(rho_c)
        n_large = self.ps_large_coar.solve(self._phi_large,
                                           self.large.embed(rho_c), **kwargs)
        if not self.use_coarse:
            phi.copy_(self.large.window(self._phi_large))
            return n_large
        phi_b, rho_b = self._boundary_correction()
        phi -= phi_b
        n_small = self.ps_small_fine.solve(phi, rho - rho_b, **kwargs)
        phi += phi_b
        return (n_large, n_small)

    def todict(self):
        d = {'name': 'ExtraVacuumPoissonSolver',
             'gpts': self.N_large_fine_c,
             'poissonsolver_large': self.ps_large_coar.todict(),
             'coarses': self.Ncoar, 'nn_coarse': self.nn_coarse,
             'nn_refine': self.nn_refine, 'nn_laplace': self.nn_laplace,
             'use_aux_grid': self.use_aux_grid}
        if self.use_coarse:
            d['poissonsolver_small'] = self.ps_small_fine.todict()
        return d
