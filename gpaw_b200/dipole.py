"""Dipole-layer correction around the finite-difference Poisson solver.

Drop-in for ``gpaw.dipole_correction.DipoleCorrection`` (finite-difference
branch, gpaw/dipole_correction.py:6-92 and 125-172).

The problem: a slab that is periodic in two directions and has zero
boundaries along the third axis c carries a dipole moment p along c; with
zero boundaries the solver would put the slab's field into the vacuum on
both sides.  The cure: add a compensating charge layer q(r) whose dipole
moment is -p, solve for the sum, and take the layer's own potential back
out.  The layer is an odd Gaussian profile in the scaled coordinate
s = 2 r_c / L - 1 (L the cell length along c),

    q(s) = A s exp(-alpha s^2),          alpha = 12,

localised well inside the cell, so that its potential is flat near both
faces.  From the one-dimensional Poisson equation d^2 phi / dr^2 = -4 pi q
with dr = (L / 2) ds,

    phi_q(s) = A (pi / alpha)^(3/2) (L^2 / 4) erf(sqrt(alpha) s),

and A follows from the condition that the layer's moment is -p (the moment
of the unit profile is measured on the grid, so the cancellation is exact
on the discrete grid).  The corrected potential is
solve(rho + q) - phi_q; the constant A (pi / alpha)^(3/2) L^2 / 4 is the
potential step across the layer (``correction``), which ``zero_vacuum``
adds so that the vacuum on the low side sits at zero.

Here the unit profile, its erf potential and its moment are built once per
grid on the device (torch), and each solve costs three device sums for p,
one scalar read of it, and two scaled copies.
"""
from __future__ import annotations

from math import pi, sqrt

import numpy as np
import torch

BOHR = 0.5291772105638411  # Angstrom: ase.units.Bohr (CODATA 2014), the
#                             reference's conversion of user widths

# width parameter of the layer in the scaled coordinate (the reference's
# choice; the numbers depend on it)
ALPHA = 12.0


def _axis_positions(gd, c, origin=0.0):
    """Grid-point positions along lattice axis c (index times spacing
    units), relative to `origin` (in points)."""
    return np.arange(gd.beg_c[c], gd.end_c[c]) - origin


def calculate_dipole_moment(gd, rho_g, center=False, origin_c=None):
    """Dipole moment -sum_g r_g rho_g dv (gpaw/old/grid_descriptor.py:
    648-663) of a density on the grid (torch tensor or numpy array).
    ``center`` measures positions from the cell centre, ``origin_c`` (in
    grid points) from a given origin."""
    if center:
        assert origin_c is None
        origin = 0.5 * np.asarray(gd.N_c, float)
    elif origin_c is not None:
        origin = np.asarray(origin_c, float)
    else:
        origin = np.zeros(3)
    # the density projected on each lattice axis (sums over the other two
    # axes), then the first moment of each projection
    if isinstance(rho_g, torch.Tensor):
        proj = [rho_g.sum(dim=(1, 2)), rho_g.sum(dim=(0, 2)),
                rho_g.sum(dim=(0, 1))]
        first = torch.stack([
            torch.dot(torch.as_tensor(_axis_positions(gd, c, origin[c]),
                                      dtype=rho_g.dtype,
                                      device=rho_g.device), proj[c])
            for c in range(3)]).cpu().numpy()
    else:
        proj = [rho_g.sum(axis=(1, 2)), rho_g.sum(axis=(0, 2)),
                rho_g.sum(axis=(0, 1))]
        first = np.array([_axis_positions(gd, c, origin[c]) @ proj[c]
                          for c in range(3)])
    # lattice moments -> Cartesian: positions are sum_c n_c h_cv
    return -(first @ gd.h_cv) * gd.dv


class _LayerProfile:
    """The unit layer q1(s) = s exp(-alpha s^2), the erf potential shape
    erf(sqrt(alpha) s) and the dipole moment of q1 along axis c, on one
    grid, resident on the device."""

    def __init__(self, gd, c, device, center=False, origin_c=None):
        L = abs(float(gd.cell_cv[c, c]))
        # Cartesian coordinate c of every grid point, (beg + i) h summed
        # over the lattice axes (exact for axes orthogonal to c)
        r = None
        for d in range(3):
            idx = torch.arange(gd.beg_c[d], gd.end_c[d], dtype=torch.float64,
                               device=device) * float(gd.h_cv[d, c])
            shape = [1, 1, 1]
            shape[d] = -1
            term = idx.reshape(shape)
            r = term if r is None else r + term
        r = r.expand(*[int(n) for n in gd.n_c])
        s = (2.0 / L) * r - 1.0
        self.q1 = (s * torch.exp(-ALPHA * (s * s))).contiguous()
        self.erf_s = torch.erf(sqrt(ALPHA) * s).contiguous()
        self.moment = float(calculate_dipole_moment(
            gd, self.q1, center, origin_c)[c])
        # potential step per unit amplitude: (pi/alpha)^(3/2) L^2 / 4
        self.step = (pi / ALPHA)**1.5 * L * L / 4.0


def dipole_correction(c, gd, rhot_g, center=False, origin_c=None,
                      profile=None):
    """(drho_g, dphi_g, correction) for the density rhot_g (a device
    tensor): the compensating layer, minus its potential, and the
    potential step across it; zeros when rhot_g has no dipole along c
    (|p| < 1e-12).  Same contract as the reference's function."""
    dev = rhot_g.device
    p = float(calculate_dipole_moment(gd, rhot_g, center, origin_c)[c])
    if abs(p) < 1e-12:
        return gd.zeros(), gd.zeros(), 0.0
    if profile is None:
        profile = _LayerProfile(gd, c, dev, center, origin_c)
    amp = -p / profile.moment
    correction = amp * profile.step
    return amp * profile.q1, -correction * profile.erf_s, correction


def _layer_axis(direction, cell_cv):
    """Axis index of a dipole layer given as 0, 1, 2 or as the layer's
    plane ('xy', 'xz', 'yz'): the lattice axis with no component in that
    plane."""
    if not isinstance(direction, str):
        return direction
    plane = ['xyz'.index(ch) for ch in direction]
    perpendicular = [c for c in range(3)
                     if abs(cell_cv[c, plane]).max() < 1e-12]
    if not perpendicular:
        raise ValueError('No axis perpendicular to {}-plane!'
                         .format(direction))
    return perpendicular[0]


class DipoleCorrection:
    """Dipole-correcting wrapper around a finite-difference Poisson solver.

    direction: 0, 1, 2 or the plane of the layer ('xy', 'xz', 'yz');
    width (Angstrom) belongs to the plane-wave variant and is only kept
    for ``todict``; zero_vacuum shifts the potential so that the vacuum on
    the low side is zero."""

    def __init__(self, poissonsolver, direction, width=1.0,
                 zero_vacuum=False):
        self.poissonsolver = poissonsolver
        self.c = direction
        self.width = width / BOHR
        self.zero_vacuum = zero_vacuum
        self.correction = None
        self._profile = None

    def todict(self):
        d = dict(self.poissonsolver.todict(), dipolelayer=self.c)
        if self.width != 1.0 / BOHR:
            d['width'] = self.width * BOHR
        return d

    def get_stencil(self):
        return self.poissonsolver.get_stencil()

    def set_grid_descriptor(self, gd):
        self.poissonsolver.set_grid_descriptor(gd)
        self.check_direction(gd, gd.pbc_c)
        self._profile = None

    def check_direction(self, gd, pbc_c):
        """The layer's axis must have zero boundaries and be orthogonal to
        the two other lattice vectors (those two need not be orthogonal to
        each other)."""
        c = _layer_axis(self.c, gd.cell_cv)
        self.c = c
        if pbc_c[c]:
            raise ValueError('System must be non-periodic perpendicular '
                             'to dipole-layer.')
        dots = [abs(np.dot(gd.cell_cv[c], gd.cell_cv[d]))
                for d in range(3) if d != c]
        if max(dots) > 1e-12:
            raise ValueError('Dipole correction axis must be '
                             'orthogonal to the two other axes.')

    def get_description(self):
        return (self.poissonsolver.get_description() +
                '\nDipole correction along %s-axis' % 'xyz'[self.c])

    def solve(self, pot, dens, **kwargs):
        return self.fdsolve(pot, dens, **kwargs)

    def fdsolve(self, vHt_g, rhot_g, **kwargs):
        gd = self.poissonsolver.gd
        if self._profile is None:
            self._profile = _LayerProfile(gd, self.c, rhot_g.device)
        drho, dphi, self.correction = dipole_correction(
            self.c, gd, rhot_g, profile=self._profile)
        if self.zero_vacuum:
            dphi = dphi + self.correction
        # solve for rho + layer starting from the caller's guess shifted
        # by the layer's potential, then take that potential back out
        vHt_g -= dphi
        niter = self.poissonsolver.solve(vHt_g, rhot_g + drho, **kwargs)
        vHt_g += dphi
        return niter
