"""Multigrid preconditioner for band residuals.

Drop-in for ``gpaw.preconditioner.Preconditioner`` (gpaw/preconditioner.py:
9-93): the same constructor and call signature, the same numbers.  What it
computes is a fixed two-grid-deep V-cycle that approximates the inverse of
the kinetic operator K0 on each residual R (c/fd_preconditioner.cpp:106-351):
one damped-Jacobi step with weight w = 0.66666666 / diag(K0) on the fine
grid, preceded by a correction from the grids 2h and 4h, where K is the
second-order -1/2 Laplacian and the steps are 4w and 16w.

Layout here: the three grids form a short list of levels; level l holds its
kinetic operator and its work arrays, sized for ``block`` bands and sliced
per call.  Every arithmetic step runs on the device inside eight fused
kernels of one native call (``gb_fd_precond``); nothing is staged through
the host.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import cgpaw
from .fd_operators import Laplace
from .transformers import Transformer

# The reference's damping weight, 2/3 written with eight digits
# (gpaw/preconditioner.py:19); kept as written so that the steps agree to
# the last bit.
JACOBI_WEIGHT = 0.66666666


@dataclasses.dataclass
class _Level:
    gd: object
    kin: object
    work: object        # (n_work, block, *grid) device array


class Preconditioner:
    def __init__(self, gd0, kin0, dtype=float, block=1, xp=None):
        grids = [gd0]
        while len(grids) < 3:
            grids.append(grids[-1].coarsen())
        # fine level: the caller's operator and two work grids (the output
        # and the interpolated correction); coarse levels: the 2nd-order
        # kinetic operator and three work grids (restricted residual,
        # correction, operator product)
        self.levels = [
            _Level(g, kin0 if lv == 0 else Laplace(g, -0.5, 1, dtype),
                   g.zeros((2 if lv == 0 else 3, block), dtype))
            for lv, g in enumerate(grids)]
        self.kin0 = kin0
        self.block = block
        self.dtype = dtype
        self.step = JACOBI_WEIGHT / kin0.get_diagonal_element()
        # order-2 transfers between neighbouring levels
        self.down = [Transformer(grids[lv], grids[lv + 1], 1, dtype)
                     for lv in range(2)]
        self.up = [Transformer(grids[lv + 1], grids[lv], 1, dtype)
                   for lv in range(2)]

    def calculate_kinetic_energy(self, psit_xG, kpt):
        return None

    def __call__(self, residuals, kpt, ekin=None, out=None):
        """Precondition ``residuals`` (one grid or a batch of bands).  The
        Bloch phases come from ``kpt.phase_cd``, or from ``kpt`` itself
        when it is the (3, 2) phase array or None.  Returns ``out`` (or a
        work array of the fine level when ``out`` is None)."""
        if residuals.dim() == 3:
            one = None if out is None else out[None]
            return self(residuals[None], kpt, ekin, one)[0]
        nbands = residuals.shape[0]
        if nbands > self.block:
            # more bands than the work arrays hold: chunks of `block`
            assert out is not None
            for b0 in range(0, nbands, self.block):
                self(residuals[b0:b0 + self.block], kpt, ekin,
                     out[b0:b0 + self.block])
            return out
        phases = getattr(kpt, 'phase_cd', kpt)
        if phases is not None:
            phases = np.asarray(phases)
        fine, mid, coarse = (lv.work[:, :nbands] for lv in self.levels)
        result = fine[1] if out is None else out
        # native sequence; work slots as c/fd_preconditioner.cpp names
        # them: fine (d0 = result, q0), level 1 (r1, d1, q1), level 2
        # (r2, d2, q2)
        cgpaw.fd_precond(self.down[0].transformer, self.down[1].transformer,
                         self.up[0].transformer, self.up[1].transformer,
                         self.kin0.operator, self.levels[1].kin.operator,
                         self.levels[2].kin.operator,
                         result, fine[0], mid[0], mid[1], mid[2],
                         coarse[0], coarse[1], coarse[2],
                         residuals.contiguous(), None, self.step, phases)
        return result
