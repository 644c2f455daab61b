"""Dipole-layer correction around the finite-difference Poisson solver
(drop-in for gpaw/dipole_correction.py, finite-difference branch).

For a slab that is non-periodic along one axis c, the solver is given the
density plus a compensating charge whose potential is an error function in
the c coordinate (gpaw/dipole_correction.py:125-172): the corrected problem
has no net dipole along c, and the correction's potential is added back
afterwards (:84-92).  The dipole moments are sums over the grid on the
device; the correction profile is computed on the host (float64) from the
grid coordinates, as the reference does.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.special import erf

BOHR = 0.5291772105638411  # Angstrom: ase.units.Bohr (CODATA 2014), the
#                             reference's conversion


def calculate_dipole_moment(gd, rho_g, center=False, origin_c=None):
    """-sum_g r_g rho_g dv (gpaw/old/grid_descriptor.py:648-663); rho_g a
    torch tensor or numpy array of the grid's shape."""
    r_cz = [np.arange(gd.beg_c[c], gd.end_c[c]) for c in range(3)]
    if center:
        assert origin_c is None
        r_cz = [r_cz[c] - 0.5 * gd.N_c[c] for c in range(3)]
    elif origin_c is not None:
        r_cz = [r_cz[c] - origin_c[c] for c in range(3)]
    if isinstance(rho_g, torch.Tensor):
        rho_01 = rho_g.sum(dim=2)
        rho_02 = rho_g.sum(dim=1)
        rho_cz = [t.cpu().numpy() for t in (rho_01.sum(dim=1),
                                              rho_01.sum(dim=0),
                                              rho_02.sum(dim=0))]
    else:
        rho_01 = rho_g.sum(axis=2)
        rho_02 = rho_g.sum(axis=1)
        rho_cz = [rho_01.sum(axis=1), rho_01.sum(axis=0), rho_02.sum(axis=0)]
    rhog_c = [np.dot(r_cz[c], rho_cz[c]) for c in range(3)]
    return -np.dot(rhog_c, gd.h_cv) * gd.dv


def dipole_correction(c, gd, rhot_g, center=False, origin_c=None):
    """(drho_g, dphi_g, phifactor): a charge whose potential is an error
    function along axis c and that cancels the dipole of rhot_g
    (gpaw/dipole_correction.py:125-172).  The arrays live on rhot_g's
    device."""
    dev = rhot_g.device
    moment = calculate_dipole_moment(gd, rhot_g, center, origin_c)[c]
    if abs(moment) < 1e-12:
        return gd.zeros(), gd.zeros(), 0.0
    r_g = gd.get_grid_point_coordinates()[c]
    cellsize = abs(gd.cell_cv[c, c])
    sr_g = 2.0 / cellsize * r_g - 1.0
    alpha = 12.0
    drho_g = sr_g * np.exp(-alpha * sr_g**2)
    moment2 = calculate_dipole_moment(gd, drho_g, center, origin_c)[c]
    factor = -moment / moment2
    drho_g *= factor
    phifactor = factor * (np.pi / alpha)**1.5 * cellsize**2 / 4.0
    dphi_g = -phifactor * erf(sr_g * np.sqrt(alpha))
    return (torch.from_numpy(drho_g).to(dev),
            torch.from_numpy(dphi_g).to(dev), phifactor)


class DipoleCorrection:
    """Dipole-correcting wrapper around a finite-difference Poisson solver
    (gpaw/dipole_correction.py:6-92)."""

    def __init__(self, poissonsolver, direction, width=1.0,
                 zero_vacuum=False):
        self.c = direction
        self.poissonsolver = poissonsolver
        self.width = width / BOHR
        self.zero_vacuum = zero_vacuum
        self.correction = None

    def todict(self):
        dct = self.poissonsolver.todict()
        dct['dipolelayer'] = self.c
        if self.width != 1.0 / BOHR:
            dct['width'] = self.width * BOHR
        return dct

    def get_stencil(self):
        return self.poissonsolver.get_stencil()

    def set_grid_descriptor(self, gd):
        self.poissonsolver.set_grid_descriptor(gd)
        self.check_direction(gd, gd.pbc_c)

    def check_direction(self, gd, pbc_c):
        """:40-62: the axis must be non-periodic and orthogonal to the two
        others."""
        if isinstance(self.c, str):
            axes = ['xyz'.index(d) for d in self.c]
            for c in range(3):
                if abs(gd.cell_cv[c, axes]).max() < 1e-12:
                    break
            else:
                raise ValueError('No axis perpendicular to {}-plane!'
                                 .format(self.c))
            self.c = c
        if pbc_c[self.c]:
            raise ValueError('System must be non-periodic perpendicular '
                             'to dipole-layer.')
        for c1 in range(3):
            if c1 != self.c:
                if abs(np.dot(gd.cell_cv[self.c], gd.cell_cv[c1])) > 1e-12:
                    raise ValueError('Dipole correction axis must be '
                                     'orthogonal to the two other axes.')

    def get_description(self):
        return '\n'.join([self.poissonsolver.get_description(),
                          'Dipole correction along %s-axis' % 'xyz'[self.c]])

    def solve(self, pot, dens, **kwargs):
        return self.fdsolve(pot, dens, **kwargs)

    def fdsolve(self, vHt_g, rhot_g, **kwargs):
        gd = self.poissonsolver.gd
        drhot_g, dvHt_g, self.correction = dipole_correction(self.c, gd,
                                                             rhot_g)
        if self.zero_vacuum:
            dvHt_g += self.correction
        vHt_g -= dvHt_g
        iters = self.poissonsolver.solve(vHt_g, rhot_g + drhot_g, **kwargs)
        vHt_g += dvHt_g
        return iters
