"""Poisson solver with multipole-moment corrections (drop-in for
gpaw/poisson_moment.py).

In a non-periodic cell the density's multipole moments about one or more
centres are removed with Gaussian multipoles whose potentials are known in
closed form; the rest, free of those moments, is solved by the wrapped
solver, and the Gaussians' potentials are added back
(gpaw/poisson_moment.py:210-243).  With several centres every grid point
belongs to the nearest one.  Masks, Gaussians and potentials are computed
once per grid (host float64, gpaw_b200.multipole) and kept on the device;
the moments are device sums.
"""
from __future__ import annotations

from typing import Any

import numpy as np
import torch

from .multipole import Gaussian

BOHR = 0.5291772105638411  # Angstrom: ase.units.Bohr (CODATA 2014), the
#                             reference's conversion


class MomentCorrection:
    """Moments ``moms`` (L indices) about ``center`` (Angstrom; None: the
    middle of the cell) (gpaw/poisson_moment.py:16-57)."""

    def __init__(self, center, moms):
        if center is not None:
            center = np.asarray(center) / BOHR
        self.center = center
        self.moms = np.asarray(moms)

    def todict(self) -> dict[str, Any]:
        center = self.center
        if center is not None:
            center = center * BOHR
        return dict(moms=self.moms, center=center)

    def __str__(self):
        if self.center is None:
            center = 'center'
        else:
            center = ', '.join([f'{x:.2f}' for x in self.center * BOHR])
        if np.allclose(np.diff(self.moms), 1):
            moms = f'range({self.moms[0]}, {self.moms[-1] + 1})'
        else:
            moms = '(' + ', '.join([f'{m:.0f}' for m in self.moms]) + ')'
        return f'[{center}] {moms}'

    def __repr__(self):
        """:53-57: the moments and the centre in Angstrom (the reference
        scales its stored centre in place here; this leaves it as it is)."""
        center = None if self.center is None else self.center * BOHR
        return f'{repr(self.moms)} @ {repr(center)}'


class MomentCorrectionPoissonSolver:
    """``MomentCorrectionPoissonSolver(poissonsolver, moment_corrections)``
    (gpaw/poisson_moment.py:60-249).  ``poissonsolver``: a solver object or
    a dict ``{'name': 'fd', ...}``; ``moment_corrections``: an int m
    (moments range(m) about the centre of the cell) or a list of
    ``{'moms': ..., 'center': ...}``."""

    def __init__(self, poissonsolver, moment_corrections, timer=None,
                 xp=None):
        if isinstance(poissonsolver, dict):
            kw = dict(poissonsolver)
            name = kw.pop('name', 'fd')
            if name != 'fd':
                raise ValueError(f'Unknown poisson solver: {name}')
            from .poisson import FDPoissonSolver
            poissonsolver = FDPoissonSolver(**kw)
        self.poissonsolver = poissonsolver
        self._initialized = False
        if moment_corrections is None:
            self.moment_corrections = []
        elif isinstance(moment_corrections, int):
            self.moment_corrections = [
                MomentCorrection(moms=range(moment_corrections), center=None)]
        elif isinstance(moment_corrections, list):
            assert all(['moms' in m and 'center' in m
                        for m in moment_corrections]), \
                ('each element in moment_correction must be a dictionary '
                 'with the keys "moms" and "center"')
            self.moment_corrections = [MomentCorrection(**m)
                                       for m in moment_corrections]
        else:
            raise ValueError('moment_correction must be a list of '
                             'dictionaries')

    def todict(self):
        return {'name': 'MomentCorrectionPoissonSolver',
                'poissonsolver': self.poissonsolver.todict(),
                'moment_corrections': [m.todict()
                                       for m in self.moment_corrections]}

    def set_grid_descriptor(self, gd):
        self.poissonsolver.set_grid_descriptor(gd)
        self.gd = gd
        self._initialized = False

    def get_description(self):
        n = len(self.moment_corrections)
        lines = [self.poissonsolver.get_description(),
                 f'    {n} moment corrections:']
        lines += [f'      {m}' for m in self.moment_corrections]
        return '\n'.join(lines)

    def _init(self):
        """:146-158: orthogonal, non-periodic cells only."""
        if self._initialized:
            return
        if not self.gd.orthogonal or bool(self.gd.pbc_c.any()):
            raise NotImplementedError('Only orthogonal unit cells '
                                      'and non-periodic boundary '
                                      'conditions are tested')
        self.load_moment_corrections_gauss()
        self._initialized = True

    def load_moment_corrections_gauss(self):
        """:160-195: one Gaussian helper per centre; every point is
        assigned to its nearest centre (the first on ties)."""
        self.gauss_i = []
        self.mom_ij = []
        self.mask_ig = []
        self._dev = {}
        if not self.moment_corrections:
            return
        r_ir = []
        for m in self.moment_corrections:
            g = Gaussian(self.gd, center=m.center)
            self.gauss_i.append(g)
            r_ir.append(g.r.ravel())
            self.mom_ij.append(m.moms)
        r_ir = np.array(r_ir)
        nearest = np.argmin(r_ir, axis=0)
        dev = self.gd.device
        for i in range(len(self.gauss_i)):
            mask = (nearest == i).astype(float).reshape(tuple(self.gd.n_c))
            self.mask_ig.append(torch.from_numpy(mask).to(dev))

    def _arrays(self, i, L):
        """Device copies of Y_L, g_L and v_L of centre i."""
        key = (i, int(L))
        if key not in self._dev:
            g = self.gauss_i[i]
            dev = self.gd.device
            self._dev[key] = tuple(torch.from_numpy(np.ascontiguousarray(a))
                                   .to(dev) for a in (g.get_Y(L),
                                                      g.get_gauss(L),
                                                      g.get_gauss_pot(L)))
        return self._dev[key]

    def remove_moment(self, i, n, L):
        """Gaussian.remove_moment (gpaw/utilities/gauss.py:146-160): the
        moment q of n, n -= q g_L in place, returns q v_L (0 when
        |q| < 1e-7)."""
        Y, g, v = self._arrays(i, L)
        q = float((n * Y).sum()) * self.gd.dv
        if abs(q) < 1e-7:
            return 0.0
        n -= q * g
        return q * v

    def solve(self, phi, rho, **kwargs):
        self._init()
        if not self.moment_corrections:
            return self.poissonsolver.solve(phi, rho, **kwargs)
        rho_neutral = rho * 0.0
        phi_cor_g = self.gd.zeros()
        for i, (mask_g, mom_j) in enumerate(zip(self.mask_ig, self.mom_ij)):
            rho_masked = rho * mask_g
            for mom in mom_j:
                phi_cor_g += self.remove_moment(i, rho_masked, mom)
            rho_neutral += rho_masked
        phi -= phi_cor_g
        niter = self.poissonsolver.solve(phi, rho_neutral, **kwargs)
        phi += phi_cor_g
        return niter

    def __repr__(self):
        n = len(self.moment_corrections)
        s = ('no corrections' if n == 0 else
             repr(self.moment_corrections[0]) if n < 2 else
             f'{n} corrections')
        return f'MomentCorrectionPoissonSolver ({s})'
