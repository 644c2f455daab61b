"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No dataset is involved: densities are sums of normalised Gaussians
q (pi w^2)^(-3/2) exp(-|r - c|^2 / w^2) at seeded positions, as the
benchmark configurations describe them; lengths in Bohr.
"""
from __future__ import annotations

import numpy as np

BOHR = 0.5291772105638411  # Angstrom: ase.units.Bohr (CODATA 2014), the
#                             reference's conversion


def gaussian_density(gd, centers, widths, charges):
    """Sum of normalised Gaussians on the points of ``gd`` (numpy, float64).

    Evaluated one Gaussian at a time (float64 throughout)."""
    r = gd.get_grid_point_coordinates()
    rho = np.zeros(tuple(int(x) for x in gd.n_c))
    for c, w, q in zip(centers, widths, charges):
        d2 = ((r - np.asarray(c)[:, None, None, None])**2).sum(0)
        rho += q * (np.pi * w * w)**-1.5 * np.exp(-d2 / (w * w))
    return rho


def c1_density(gd, seed=0):
    """8 Gaussians, width 0.8 A, centres uniform in [0.25, 0.75] of the box,
    charges +1/-1 alternating (net zero before discretisation)."""
    rng = np.random.default_rng(seed)
    L = np.diag(gd.cell_cv)
    centers = [rng.uniform(0.25, 0.75, 3) * L for _ in range(8)]
    widths = [0.8 / BOHR] * 8
    charges = [1.0 if i % 2 == 0 else -1.0 for i in range(8)]
    return gaussian_density(gd, centers, widths, charges)


def c3_density(gd, ngauss=64, seed=0):
    """`ngauss` Gaussians, widths U[0.5, 1.2] A, charges +-U[0.5, 2] with a
    random sign, centres uniform in [0.2, 0.8] of the box; the caller
    neutralises by subtracting the mean."""
    rng = np.random.default_rng(seed)
    L = np.diag(gd.cell_cv)
    centers = [rng.uniform(0.2, 0.8, 3) * L for _ in range(ngauss)]
    widths = rng.uniform(0.5, 1.2, ngauss) / BOHR
    charges = rng.uniform(0.5, 2.0, ngauss) * rng.choice([-1.0, 1.0], ngauss)
    return gaussian_density(gd, centers, widths, charges)


def neutralize(rho, gd):
    """rho - background, as the neutral branch of the solver forms it
    (gpaw/poisson.py:186-213): charge / dv / number of points."""
    charge = rho.sum() * gd.dv
    return rho - charge / gd.dv / np.prod(gd.n_c)


def eps_for_relative_residual(rho, gd, rel=1e-10):
    """The reference stops when sum(r^2) dv <= eps (gpaw/poisson.py:485,
    527-537); this eps corresponds to ||L phi - rho|| / ||rho|| = rel."""
    return (rel * float(np.sqrt((rho * rho).sum())))**2 * gd.dv


def gaussian_density_device(gd, centers, widths, charges):
    """gaussian_density evaluated on the GPU (torch, float64)."""
    import torch
    dev = gd.device
    idx = [torch.arange(int(n), dtype=torch.float64, device=dev) + int(b)
           for n, b in zip(gd.n_c, gd.beg_c)]
    h = torch.tensor(np.diag(gd.h_cv), dtype=torch.float64, device=dev)
    x = (idx[0] * h[0])[:, None, None]
    y = (idx[1] * h[1])[None, :, None]
    z = (idx[2] * h[2])[None, None, :]
    rho = torch.zeros(tuple(int(n) for n in gd.n_c), dtype=torch.float64,
                      device=dev)
    for c, w, q in zip(centers, widths, charges):
        d2 = (x - c[0])**2 + (y - c[1])**2 + (z - c[2])**2
        rho += q * (np.pi * w * w)**-1.5 * torch.exp(-d2 / (w * w))
    return rho


def random_gaussians(gd, ngauss, rng):
    """C3 distributions: widths U[0.5, 1.2] A, charges +-U[0.5, 2], centres
    uniform in [0.2, 0.8] of the (orthorhombic) box."""
    L = np.diag(gd.cell_cv)
    centers = [rng.uniform(0.2, 0.8, 3) * L for _ in range(ngauss)]
    widths = rng.uniform(0.5, 1.2, ngauss) / BOHR
    charges = rng.uniform(0.5, 2.0, ngauss) * rng.choice([-1.0, 1.0], ngauss)
    return centers, widths, charges


def neutral_density_device(gd, ngauss, seed):
    """Seeded neutral density on the GPU (mean removed as the neutral
    branch does, charge / dv / number of points)."""
    rng = np.random.default_rng(seed)
    rho = gaussian_density_device(gd, *random_gaussians(gd, ngauss, rng))
    return rho - rho.sum() / rho.numel()
