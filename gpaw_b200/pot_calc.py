"""Grid transfers of the finite-difference potential calculator
(drop-in for the transfer part of gpaw/new/fd/pot_calc.py).

``FDPotentialCalculator`` moves densities from the wave-function grid to the
fine grid (twice as many points per axis) with a tri-linear .. tri-heptic
interpolation and potentials back with the matching restriction
(gpaw/new/fd/pot_calc.py:37-41, 57-61).  On grids that are not periodic in
every direction the interpolated density is rescaled so that its integral
equals the coarse one (:72-80).  Both transfers are the sm_100a
``Transformer`` kernels; the two integrals are device reductions and the
rescaling a device multiply, so nothing leaves the GPU.
"""
from __future__ import annotations

import torch

from .transformers import Transformer

_NAMES = ['linear', 'cubic', 'quintic', 'heptic']


class FDDensityTransfers:
    """interpolate / restrict / interpolate_density of FDPotentialCalculator
    for a wave-function grid ``gd`` and its refinement ``finegd``."""

    def __init__(self, gd, finegd, interpolation_stencil_range=3,
                 dtype=float):
        self.grid = gd
        self.fine_grid = finegd
        n = int(interpolation_stencil_range)
        self.interpolation_stencil_range = n
        self._interpolate = Transformer(gd, finegd, n, dtype)
        self._restrict = Transformer(finegd, gd, n, dtype)

    def __str__(self):
        degree = self.interpolation_stencil_range * 2 - 1
        name = _NAMES[degree // 2]
        return (f'interpolation: tri-{name}' +
                f' # {degree}. degree polynomial\n')

    def interpolate(self, a_xR, a_xr=None):
        """gpaw/new/fd/pot_calc.py:57-58."""
        return self._interpolate.apply(a_xR, a_xr)

    def restrict(self, a_xr, a_xR=None):
        """gpaw/new/fd/pot_calc.py:60-61."""
        return self._restrict.apply(a_xr, a_xR)

    def interpolate_density(self, nt_sR, nt_sr=None):
        """_interpolate_density (gpaw/new/fd/pot_calc.py:72-80): the
        interpolated density, each spin rescaled to the coarse integral
        when the grid is not periodic in all directions (skipped where the
        fine integral is 1e-14 or less).  Returns nt_sr."""
        nt_sr = self.interpolate(nt_sR, nt_sr)
        if not bool(self.grid.pbc_c.all()):
            shape = nt_sR.shape[:-3]
            one = len(shape) == 0
            c = nt_sR.reshape((1,) + tuple(nt_sR.shape[-3:])) if one \
                else nt_sR.reshape((-1,) + tuple(nt_sR.shape[-3:]))
            f = nt_sr.reshape((1,) + tuple(nt_sr.shape[-3:])) if one \
                else nt_sr.reshape((-1,) + tuple(nt_sr.shape[-3:]))
            Nt1 = c.reshape(c.shape[0], -1).sum(dim=1) * self.grid.dv
            Nt2 = f.reshape(f.shape[0], -1).sum(dim=1) * self.fine_grid.dv
            scale = torch.where(Nt2 > 1e-14, Nt1 / Nt2,
                                torch.ones_like(Nt2))
            f.mul_(scale.view(-1, 1, 1, 1))
        return nt_sr
