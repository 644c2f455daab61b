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
