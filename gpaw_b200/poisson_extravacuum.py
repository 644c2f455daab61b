"""Poisson solver with extra vacuum (drop-in for gpaw/poisson_extravacuum.py).

The potential of a non-periodic system is solved on a larger grid
(``gpts`` points per axis) around the original one, so that the zero
boundary condition sits further from the charge
(gpaw/poisson_extravacuum.py:13-232).  With ``coarses`` > 0 the large grid
is ``coarses`` times coarser than the original: the density is restricted,
embedded in the large coarse grid and solved there; the coarse potential
is refined back on an auxiliary grid (the original plus a buffer for the
stencils), its Laplacian gives the density that matches it, and the
original grid is then solved for the difference, with the refined
potential as the boundary correction.  Restriction, interpolation, the
Laplacian and the solves are the sm_100a kernels; embedding a grid in a
larger one is a device copy.
"""
from __future__ import annotations

from math import pi

import numpy as np

from .fd_operators import Laplace
from .grid_descriptor import GridDescriptor
from .transformers import Transformer


def _create(ps):
    if ps is None or not isinstance(ps, dict):
        return ps
    kw = dict(ps)
    name = kw.pop('name', 'fd')
    if name != 'fd':
        raise ValueError(f'Unknown poisson solver: {name}')
    from .poisson import FDPoissonSolver
    return FDPoissonSolver(**kw)


def extended_grid_descriptor(gd, N_c):
    """gpaw/utilities/extend_grid.py:8-44 for a target size ``N_c``: the
    same spacing, (N_c - N) // 2 extra points on each side."""
    N_c = np.array(N_c, dtype=int)
    extend_N_cd = np.tile((N_c - gd.N_c) // 2, (2, 1)).T
    cell_cv = gd.h_cv * N_c
    egd = GridDescriptor(N_c, cell_cv, gd.pbc_c, device=gd.device)
    egd.extend_N_cd = extend_N_cd
    return egd


def extend_array(gd, egd, a_g, aext_g):
    """Copy a_g into its place in the larger grid (gpaw/utilities/
    extend_grid.py:47-50, one domain)."""
    o = egd.extend_N_cd[:, 0]
    n = gd.n_c
    aext_g[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]] = a_g


def deextend_array(gd, egd, a_g, aext_g):
    """Copy the part of aext_g over the smaller grid into a_g (:53-56)."""
    o = egd.extend_N_cd[:, 0]
    n = gd.n_c
    a_g[:] = aext_g[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]]


class ExtraVacuumPoissonSolver:
    def __init__(self, gpts, poissonsolver_large, poissonsolver_small=None,
                 coarses=0, nn_coarse=3, nn_refine=3, nn_laplace=3,
                 use_aux_grid=True, xp=None):
        self.N_large_fine_c = np.array(gpts, dtype=int)
        self.Ncoar = coarses
        self.use_coarse = self.Ncoar > 0
        self.ps_large_coar = _create(poissonsolver_large)
        if self.use_coarse:
            self.ps_small_fine = _create(poissonsolver_small)
        else:
            assert poissonsolver_small is None
        self.nn_coarse = nn_coarse
        self.nn_refine = nn_refine
        self.nn_laplace = nn_laplace
        self.use_aux_grid = use_aux_grid
        self._initialized = False

    def set_grid_descriptor(self, gd):
        """:62-144: coarsening chain on the original grid, the large coarse
        grid, and (with coarses) the auxiliary grid with its Laplacian and
        refining chain."""
        if bool(gd.pbc_c.any()):
            raise NotImplementedError('Only non-periodic boundary '
                                      'conditions are tested')
        self.gd_small_fine = gd
        assert np.all(gd.N_c <= self.N_large_fine_c), \
            'extended grid has to be larger than the original one'
        if self.use_coarse:
            self.coarser_i = []
            N_c = self.N_large_fine_c.copy()
            for _ in range(self.Ncoar):
                gd2 = gd.coarsen()
                self.coarser_i.append(Transformer(gd, gd2, self.nn_coarse))
                N_c //= 2
                gd = gd2
            self.gd_small_coar = gd
        else:
            self.gd_small_coar = self.gd_small_fine
            N_c = self.N_large_fine_c
        self.gd_large_coar = extended_grid_descriptor(self.gd_small_coar, N_c)
        self.ps_large_coar.set_grid_descriptor(self.gd_large_coar)
        self._initialized = False
        if not self.use_coarse:
            return
        self.ps_small_fine.set_grid_descriptor(self.gd_small_fine)
        if self.use_aux_grid:
            buf = self.nn_refine
            for _ in range(self.Ncoar):
                buf = 2 * buf + self.nn_refine
            buf += self.nn_laplace
            div = 2**self.Ncoar
            if buf % div != 0:
                buf += div - buf % div
            N_c = self.gd_small_fine.N_c + 2 * buf
            if np.any(N_c > self.N_large_fine_c):
                self.use_aux_grid = False
                N_c = self.N_large_fine_c
            self.gd_aux_fine = extended_grid_descriptor(self.gd_small_fine,
                                                        N_c)
        else:
            self.gd_aux_fine = extended_grid_descriptor(
                self.gd_small_fine, self.N_large_fine_c)
        self.laplace_aux_fine = Laplace(self.gd_aux_fine, -0.25 / pi,
                                        self.nn_laplace)
        self.refiner_i = []
        gd = self.gd_aux_fine
        for _ in range(self.Ncoar):
            gd2 = gd.coarsen()
            self.refiner_i.append(Transformer(gd2, gd, self.nn_refine))
            gd = gd2
        self.refiner_i = self.refiner_i[::-1]
        self.gd_aux_coar = gd
        if self.use_aux_grid:
            self.gd_large_coar_from_aux = extended_grid_descriptor(
                self.gd_aux_coar, self.gd_large_coar.N_c)
            assert np.all(self.gd_large_coar.N_c ==
                          self.gd_large_coar_from_aux.N_c)
            assert np.allclose(self.gd_large_coar.h_cv,
                               self.gd_large_coar_from_aux.h_cv,
                               rtol=0, atol=1e-12)

    def _init(self):
        if self._initialized:
            return
        self.phi_large_coar_g = self.gd_large_coar.zeros()
        self._initialized = True

    def get_description(self):
        lines = ['ExtraVacuumPoissonSolver',
                 '    Large grid: %s' % ' x '.join(
                     str(N) for N in self.gd_large_coar.N_c),
                 '    ' + self.ps_large_coar.get_description()]
        if self.use_coarse:
            lines += ['    Small grid:',
                      '    ' + self.ps_small_fine.get_description()]
        return '\n'.join(lines)

    def solve(self, phi, rho, **kwargs):
        """:159-231: returns the large solve's V-cycle count, or the pair
        (large, small) with coarses."""
        self._init()
        phi_small_fine_g = phi
        rho_small_fine_g = rho.clone()
        if self.use_coarse:
            tmp_g = rho_small_fine_g
            for coarser in self.coarser_i:
                tmp_g = coarser.apply(tmp_g)
            rho_small_coar_g = tmp_g
        else:
            rho_small_coar_g = rho_small_fine_g
        rho_large_coar_g = self.gd_large_coar.zeros()
        extend_array(self.gd_small_coar, self.gd_large_coar,
                     rho_small_coar_g, rho_large_coar_g)
        niter_large = self.ps_large_coar.solve(self.phi_large_coar_g,
                                               rho_large_coar_g, **kwargs)
        if not self.use_coarse:
            deextend_array(self.gd_small_fine, self.gd_large_coar,
                           phi_small_fine_g, self.phi_large_coar_g)
            return niter_large
        if self.use_aux_grid:
            phi_aux_coar_g = self.gd_aux_coar.empty()
            deextend_array(self.gd_aux_coar, self.gd_large_coar_from_aux,
                           phi_aux_coar_g, self.phi_large_coar_g)
        else:
            phi_aux_coar_g = self.phi_large_coar_g
        tmp_g = phi_aux_coar_g
        for refiner in self.refiner_i:
            tmp_g = refiner.apply(tmp_g)
        phi_aux_fine_g = tmp_g
        rho_aux_fine_g = self.gd_aux_fine.empty()
        self.laplace_aux_fine.apply(phi_aux_fine_g, rho_aux_fine_g)
        cor_phi_small_fine_g = self.gd_small_fine.empty()
        deextend_array(self.gd_small_fine, self.gd_aux_fine,
                       cor_phi_small_fine_g, phi_aux_fine_g)
        cor_rho_small_fine_g = self.gd_small_fine.empty()
        deextend_array(self.gd_small_fine, self.gd_aux_fine,
                       cor_rho_small_fine_g, rho_aux_fine_g)
        rho_small_fine_g -= cor_rho_small_fine_g
        phi_small_fine_g -= cor_phi_small_fine_g
        niter_small = self.ps_small_fine.solve(phi_small_fine_g,
                                               rho_small_fine_g, **kwargs)
        phi_small_fine_g += cor_phi_small_fine_g
        return (niter_large, niter_small)

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
