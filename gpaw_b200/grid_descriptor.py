"""Uniform real-space grid, single domain, arrays as torch CUDA tensors.

Index conventions of gpaw/old/grid_descriptor.py:119-160, 214-218, 327-342
and neighbour ranks of gpaw/old/domain.py:110-138, restricted to one domain
(the whole grid lives on one GPU):

* ``N_c``  number of grid points per axis;
* ``n_c``  points stored: ``N_c`` if periodic, ``N_c - 1`` for a zero
  boundary (index 0 is the boundary itself, never stored);
* ``beg_c``/``end_c`` global index range of the stored points;
* ``dv``   volume per grid point, ``volume / prod(N_c)``;
* ``neighbor_cd`` 0 (own rank: periodic) or -1 (zero boundary).
"""
from __future__ import annotations

import numpy as np
import torch


class BadGridError(ValueError):
    """Grid too small (gpaw/old/grid_descriptor.py:34)."""


def _torch_dtype(dtype):
    if dtype in (float, np.float64, torch.float64):
        return torch.float64
    if dtype in (complex, np.complex128, torch.complex128):
        return torch.complex128
    if dtype in (np.float32, torch.float32):
        return torch.float32
    raise TypeError(f'unsupported dtype {dtype}')


class GridDescriptor:
    def __init__(self, N_c, cell_cv=(1, 1, 1), pbc_c=True, comm=None,
                 device=None):
        if comm is not None and getattr(comm, 'size', 1) != 1:
            raise NotImplementedError('one domain per grid')
        if isinstance(pbc_c, (bool, int, np.bool_)):
            pbc_c = (bool(pbc_c),) * 3
        self.pbc_c = np.array(pbc_c, bool)
        self.N_c = np.array(N_c, int)
        if (self.N_c != np.asarray(N_c)).any():
            raise ValueError('Non-int number of grid points %s' % (N_c,))
        cell = np.array(cell_cv, float)
        if cell.ndim == 0:
            cell = np.eye(3) * cell
        elif cell.ndim == 1:
            cell = np.diag(cell)
        self.cell_cv = cell
        self.beg_c = np.where(self.pbc_c, 0, 1)
        self.end_c = self.N_c.copy()
        if (self.end_c <= self.beg_c).any():
            raise BadGridError('Grid %s too small' % 'x'.join(
                str(n) for n in self.N_c))
        self.n_c = self.end_c - self.beg_c
        self.h_cv = self.cell_cv / self.N_c[:, np.newaxis]
        self.icell_cv = np.linalg.inv(self.cell_cv).T
        self.volume = abs(np.linalg.det(self.cell_cv))
        self.dv = self.volume / self.N_c.prod()
        self.orthogonal = not (self.cell_cv -
                               np.diag(self.cell_cv.diagonal())).any()
        self.neighbor_cd = np.ascontiguousarray(
            np.where(self.pbc_c[:, None], 0, -1) * np.ones((3, 2), int),
            np.int64)
        self.device = torch.device(device if device is not None else 'cuda')

    def __repr__(self):
        return (f'GridDescriptor({self.N_c.tolist()}, pbc_c='
                f'{self.pbc_c.tolist()})')

    def new_descriptor(self, N_c):
        return GridDescriptor(N_c, self.cell_cv, self.pbc_c,
                              device=self.device)

    def coarsen(self):
        """Half the points per axis (gpaw/old/grid_descriptor.py:327-335);
        ValueError (BadGridError) if impossible."""
        if (self.N_c % 2).any():
            raise ValueError('Grid %s not divisible by 2!' % self.N_c)
        return self.new_descriptor(self.N_c // 2)

    def refine(self):
        return self.new_descriptor(self.N_c * 2)

    def get_size_of_global_array(self, pad=False):
        return self.N_c if pad else self.N_c - 1 + self.pbc_c

    def zeros(self, n=(), dtype=float, global_array=False, xp=None):
        if isinstance(n, int):
            n = (n,)
        return torch.zeros(tuple(n) + tuple(int(x) for x in self.n_c),
                           dtype=_torch_dtype(dtype), device=self.device)

    def empty(self, n=(), dtype=float, global_array=False, xp=None):
        if isinstance(n, int):
            n = (n,)
        return torch.empty(tuple(n) + tuple(int(x) for x in self.n_c),
                           dtype=_torch_dtype(dtype), device=self.device)

    def integrate(self, a_xg):
        """sum(a) * dv per grid (gpaw/old/grid_descriptor.py:292-300)."""
        r = a_xg.reshape(a_xg.shape[:-3] + (-1,)).sum(dim=-1) * self.dv
        return r.item() if r.dim() == 0 else r

    def phase_factor_cd(self, kpt_c):
        """Bloch phases for one domain (gpaw/core/uniform_grid.py:116-127):
        column 0 multiplies reads past the high edge, column 1 the low."""
        disp_cd = np.array([[1.0, -1.0]] * 3)
        return np.exp(2j * np.pi * disp_cd * np.asarray(kpt_c)[:, None])

    def get_grid_point_distance_vectors(self, r_v, mic=True):
        """Vectors from r_v to every grid point, minimum image along
        periodic axes (gpaw/old/grid_descriptor.py:716-737); numpy."""
        s_Gc = (np.indices(self.n_c, float).T + self.beg_c) / self.N_c
        r_c = np.linalg.solve(self.cell_cv.T, r_v)
        r_c = np.where(self.pbc_c, r_c % 1.0, r_c)
        s_Gc -= np.where(self.pbc_c, r_c % 1.0, r_c)
        if mic:
            s_Gc -= self.pbc_c * (2 * s_Gc).astype(int)
        return np.dot(s_Gc, self.cell_cv).T.copy()

    def get_grid_point_coordinates(self):
        idx = np.indices(self.n_c) + self.beg_c[:, None, None, None]
        return np.einsum('cv,cxyz->vxyz', self.h_cv, idx)
