"""Multigrid preconditioner for band residuals (drop-in for
gpaw/preconditioner.py:9-93): a fixed three-level V-cycle approximating the
inverse of the kinetic operator, run as eight fused kernels per chunk of
bands (gb_fd_precond)."""
from __future__ import annotations

import numpy as np

from . import cgpaw
from .fd_operators import Laplace
from .transformers import Transformer


class Preconditioner:
    def __init__(self, gd0, kin0, dtype=float, block=1, xp=None):
        gd1 = gd0.coarsen()
        gd2 = gd1.coarsen()
        self.kin0 = kin0
        self.kin1 = Laplace(gd1, -0.5, 1, dtype)
        self.kin2 = Laplace(gd2, -0.5, 1, dtype)
        self.scratch0 = gd0.zeros((2, block), dtype)
        self.scratch1 = gd1.zeros((3, block), dtype)
        self.scratch2 = gd2.zeros((3, block), dtype)
        # gpaw/preconditioner.py:19
        self.step = 0.66666666 / kin0.get_diagonal_element()
        self.restrictor_object0 = Transformer(gd0, gd1, 1, dtype)
        self.restrictor_object1 = Transformer(gd1, gd2, 1, dtype)
        self.interpolator_object2 = Transformer(gd2, gd1, 1, dtype)
        self.interpolator_object1 = Transformer(gd1, gd0, 1, dtype)
        self.restrictor0 = self.restrictor_object0.apply
        self.restrictor1 = self.restrictor_object1.apply
        self.interpolator2 = self.interpolator_object2.apply
        self.interpolator1 = self.interpolator_object1.apply
        self.use_c_precond = True
        self.xp = xp

    def calculate_kinetic_energy(self, psit_xG, kpt):
        return None

    def __call__(self, residuals, kpt, ekin=None, out=None):
        """gpaw/preconditioner.py:35-73.  ``kpt.phase_cd`` (or ``kpt``
        itself, if it is the (3, 2) phase array or None) gives the Bloch
        phases."""
        if residuals.dim() == 3:
            if out is None:
                return self.__call__(residuals[None], kpt)[0]
            return self.__call__(residuals[None], kpt, out=out[None])[0]
        nb = len(residuals)
        nb0 = self.scratch0.shape[1]
        if nb > nb0:
            assert out is not None
            for n1 in range(0, nb, nb0):
                self(residuals[n1:n1 + nb0], kpt, out=out[n1:n1 + nb0])
            return out
        phases = getattr(kpt, 'phase_cd', kpt)
        if phases is not None:
            phases = np.asarray(phases)
        if out is None:
            d0, q0 = self.scratch0[:, :nb]
        else:
            d0 = out
            q0 = self.scratch0[0, :nb]
        r1, d1, q1 = self.scratch1[:, :nb]
        r2, d2, q2 = self.scratch2[:, :nb]
        cgpaw.fd_precond(self.restrictor_object0.transformer,
                         self.restrictor_object1.transformer,
                         self.interpolator_object1.transformer,
                         self.interpolator_object2.transformer,
                         self.kin0.operator, self.kin1.operator,
                         self.kin2.operator,
                         d0, q0, r1, d1, q1, r2, d2, q2,
                         residuals.contiguous(), None, self.step, phases)
        return d0
