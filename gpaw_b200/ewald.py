"""Madelung correction for charged periodic cells.

A charged periodic system is solved with a homogeneous neutralising
background (gpaw/poisson.py:214-231); with
``use_charged_periodic_corrections`` the reference then adds
``charge * madelung(cell)``, the Madelung potential of the lattice
(gpaw/utilities/ewald.py:143-145): the potential at a lattice point of unit
negative point charges on every *other* lattice point, in a uniform
compensating background.

Computed here by Ewald summation (P. P. Ewald, Ann. Phys. 369, 253 (1921)),
splitting each point charge q into a Gaussian-screened part summed in real
space and its smooth complement summed over the reciprocal lattice:

    phi = q [ sum_{l != 0} erfc(G |l|) / |l|
              + (4 pi / V) sum_{g != 0} exp(-g^2 / (4 G^2)) / g^2
              - 2 G / sqrt(pi) - pi / (V G^2) ],      q = -1,

the last two terms removing the screening charge's own potential at the
origin and adding the background's.  G is scaled by the longest lattice
vector (G = 5 / |a|max), which makes both sums converge to double precision
with three real-space and nine reciprocal-space shells.
"""
from __future__ import annotations

from math import pi, sqrt

import numpy as np
from scipy.special import erfc


def madelung(cell, G=5.0, nreal=3, nrecip=9):
    cell = np.asarray(cell, float)
    V = abs(np.linalg.det(cell))
    G = G / np.sqrt((cell**2).sum(1).max())
    q = -1.0
    # real-space lattice vectors l != 0 within the shells
    r = np.arange(-nreal, nreal + 1)
    ijk = np.stack(np.meshgrid(r, r, r, indexing='ij'), -1).reshape(-1, 3)
    lv = ijk @ cell
    d = np.linalg.norm(lv, axis=1)
    d = d[d > 1e-5]
    real = np.sum(erfc(G * d) / d)
    # reciprocal lattice vectors g != 0
    k = np.arange(-nrecip, nrecip + 1)
    ijk = np.stack(np.meshgrid(k, k, k, indexing='ij'), -1).reshape(-1, 3)
    gv = 2 * pi * ijk @ np.linalg.inv(cell).T
    g2 = (gv**2).sum(1)
    g2 = g2[g2 > 1e-10]
    recip = 4 * pi / V * np.sum(np.exp(-g2 / (4 * G**2)) / g2)
    return q * (real + recip - 2 * G / sqrt(pi) - pi / (V * G**2))
