"""Normalised Gaussian charge and its potential on a grid (host side).

The charged non-periodic branch of the Poisson solver removes the monopole
of the density with a Gaussian whose potential is known in closed form
(gpaw/poisson.py:233-283, gpaw/utilities/gauss.py:33-56 and 94-123):

    g(r)   = sqrt(4 a^3) / pi * exp(-a r^2)          (unit charge / sqrt(4 pi))
    v(r)   = 2 sqrt(pi) erf(sqrt(a) r) / r

centred in the middle of the cell (or at a given point), with the width
set so that exp(-a r^2) is small at the boundary: a = 4 * 19 * max_c
|icell_c|^2, or 19 / r_min^2 for an explicit centre.  Both arrays are
computed once per grid in float64 numpy and then live on the device.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SQRT_PI = 1.7724538509055159


def coordinates(gd, origin=None, tiny=1e-12):
    """Distance vectors from `origin` (default: the cell centre) and their
    squared lengths, floored at `tiny` (gpaw/utilities/tools.py:81-100)."""
    if origin is None:
        origin = 0.5 * gd.cell_cv.sum(0)
    r_vG = gd.get_grid_point_distance_vectors(np.array(origin))
    r2_G = np.sum(r_vG**2, axis=0)
    r2_G = np.where(r2_G < tiny, tiny, r2_G)
    return r_vG, r2_G


def monopole_gaussian(gd, a=19.0, center=None):
    """(rho_gauss, phi_gauss) of gpaw/poisson.py:314-318 (L = 0)."""
    _, r2 = coordinates(gd, center)
    r = np.sqrt(r2)
    if center is None:
        a = 4 * a * (gd.icell_cv**2).sum(1).max()
    else:
        cell_center = gd.cell_cv.sum(1) / 2
        r_min = (cell_center - np.abs(center - cell_center)).min()
        a = a / r_min**2
    exp_ar2 = np.exp(-a * r2)
    erf_sar = erf(np.sqrt(a) * r)
    rho = np.sqrt(a**3 * 4) / np.pi * exp_ar2
    phi = 2.0 * SQRT_PI * erf_sar / r
    return rho, phi


def charge_center_parts(gd, rho, charge, beg=(0, 0, 0)):
    """The sums behind the centre of the majority charge
    (gpaw/poisson.py:248-252): rho times the sign of ``charge``, clipped
    at zero, then per axis sum_i i rho_i over the global grid index i
    (gpaw/old/grid_descriptor.py:648-663), and the clipped density's sum.
    ``rho`` (numpy or torch) holds the box of the grid starting ``beg``
    points past the grid's first stored point.  Returns (rhog_c, total):
    host floats that add up over the boxes of a split grid."""
    sign = 1.0 if charge > 0 else -1.0
    if hasattr(rho, 'detach'):
        rs = (rho * sign).clamp(min=0.0)
        sums = [rs.sum(dim=(1, 2)), rs.sum(dim=(0, 2)), rs.sum(dim=(0, 1))]
        sums = [x.detach().cpu().numpy() for x in sums]
        total = float(rs.sum())
    else:
        rs = np.clip(np.asarray(rho) * sign, 0.0, None)
        sums = [rs.sum(axis=(1, 2)), rs.sum(axis=(0, 2)),
                rs.sum(axis=(0, 1))]
        total = float(rs.sum())
    rhog_c = np.array([
        float(np.dot(np.arange(len(sums[c])) + int(gd.beg_c[c]) +
                     int(beg[c]), sums[c])) for c in range(3)])
    return rhog_c, total


def charge_center(gd, rhog_c, total):
    """gpaw/poisson.py:248-262 from the sums of charge_center_parts: the
    centre of the majority charge, minus the dipole moment
    -(rhog_c . h_cv) dv over the charge; RuntimeError when it lies within
    7 grid spacings of the cell's faces (the Gaussian would not fit)."""
    h_cv = np.asarray(gd.h_cv)
    absolute_charge = total * gd.dv
    d_c = -np.dot(rhog_c, h_cv) * gd.dv
    center = -d_c / absolute_charge
    border_offset = np.inner(h_cv, np.array((7, 7, 7)))
    borders = np.inner(h_cv, np.asarray(gd.N_c)) - border_offset
    if np.any(center > borders) or np.any(center < border_offset):
        raise RuntimeError('Poisson solver: center of charge outside '
                           'borders - please increase box')
    return center
