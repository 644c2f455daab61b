"""Gaussian multipoles on a grid (host float64), for the moment corrections
of the Poisson solver (the ``Gaussian`` helper of gpaw/utilities/gauss.py:
95-160).

For L = 0..8 (l = 0, 1, 2) with the reference's ordering of the real
harmonics (1; y, z, x; xy, yz, 3z^2 - r^2, xz, x^2 - y^2):

  Y_L   = c_L P_L                        r^l times the real spherical harmonic
  g_L   = sqrt(a^(2l+3) K_L) / pi P_L exp(-a r^2)
                                         unit moment: int g_L Y_L dV = 1
  v_L   = A_L G_l(sqrt(a) r) / r^(2l+1) P_L
                                         the potential of g_L (del^2 v = -4 pi g)

with K_L = (2 pi c_L / Gamma(l + 3/2))^2, G_0 = erf(s),
G_1 = sqrt(pi) erf(s) - 2 s exp(-s^2), G_2 = 3 sqrt(pi) erf(s) -
(6 + 4 s^2) s exp(-s^2), and A_L = 4 pi c_L / ((2l + 1) gamma_l), gamma_l the
coefficient of erf in G_l -- so that far from the centre v_L tends to the
point multipole 4 pi / (2l + 1) Y_L / r^(2l+1).  The constants are computed
here from these definitions.
"""
from __future__ import annotations

from math import gamma, pi, sqrt

import numpy as np
from scipy.special import erf

from .gauss import coordinates

_L_OF = [0, 1, 1, 1, 2, 2, 2, 2, 2]
_C = [1 / (2 * sqrt(pi))] + [sqrt(3 / (4 * pi))] * 3 + \
    [sqrt(15 / (4 * pi)), sqrt(15 / (4 * pi)), sqrt(5 / (16 * pi)),
     sqrt(15 / (4 * pi)), sqrt(15 / (16 * pi))]
_GAMMA_ERF = [1.0, sqrt(pi), 3 * sqrt(pi)]


def _poly(L, x, y, z, r2):
    return [lambda: np.ones_like(r2), lambda: y, lambda: z, lambda: x,
            lambda: x * y, lambda: y * z, lambda: 3 * z * z - r2,
            lambda: x * z, lambda: x * x - y * y][L]()


def Y_L(L, x, y, z, r2):
    """r^l times the real spherical harmonic L (L = 0..8)."""
    return _C[L] * _poly(L, x, y, z, r2)


def gauss_L(a, L, x, y, z, r2, exp_ar2):
    l = _L_OF[L]
    K = (2 * pi * _C[L] / gamma(l + 1.5))**2
    return np.sqrt(a**(2 * l + 3) * K) / pi * _poly(L, x, y, z, r2) * exp_ar2


def gausspot_L(a, L, x, y, z, r, r2, erf_sar, exp_ar2):
    l = _L_OF[L]
    s = np.sqrt(a) * r
    if l == 0:
        G = erf_sar
    elif l == 1:
        G = sqrt(pi) * erf_sar - 2 * s * exp_ar2
    else:
        G = 3 * sqrt(pi) * erf_sar - (6 + 4 * s**2) * s * exp_ar2
    A = 4 * pi * _C[L] / ((2 * l + 1) * _GAMMA_ERF[l])
    return A * G / r**(2 * l + 1) * _poly(L, x, y, z, r2)


class Gaussian:
    """Generalized Gaussians centred at ``center`` (default: the middle of
    the cell), inverse width ``a`` set so that exp(-a r^2) is small at the
    boundary (gpaw/utilities/gauss.py:95-160).  Grids are host arrays."""

    def __init__(self, gd, a=19., center=None):
        self.gd = gd
        self.xyz, self.r2 = coordinates(gd, center)
        self.r = np.sqrt(self.r2)
        if center is None:
            self.a = 4 * a * (gd.icell_cv**2).sum(1).max()
        else:
            cell_center = gd.cell_cv.sum(1) / 2
            r_min = (cell_center - np.abs(center - cell_center)).min()
            self.a = a / r_min**2
        self.exp_ar2 = np.exp(-self.a * self.r2)
        self.erf_sar = erf(np.sqrt(self.a) * self.r)

    def get_gauss(self, L):
        x, y, z = self.xyz
        return gauss_L(self.a, L, x, y, z, self.r2, self.exp_ar2)

    def get_gauss_pot(self, L):
        x, y, z = self.xyz
        return gausspot_L(self.a, L, x, y, z, self.r, self.r2, self.erf_sar,
                          self.exp_ar2)

    def get_Y(self, L):
        x, y, z = self.xyz
        return Y_L(L, x, y, z, self.r2) * np.ones_like(self.r2)
