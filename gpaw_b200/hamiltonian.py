"""FD Hamiltonian's local part (drop-in for gpaw/new/fd/hamiltonian.py:14-32).

``FDHamiltonian(gd, kin_stencil=3, dtype=float).apply_local_potential(vt_R,
psit_nR, out)`` computes ``out = kin(psit) + psit * vt`` for a batch of
wave functions in one pass over the data: the kinetic operator -1/2 Laplacian
(``Laplace(gd, -0.5, kin_stencil)``) with the local potential's product
fused into its epilogue.  The reference applies the stencil and then adds
``p * vt`` band by band; the arithmetic here is the same (product rounded,
then the sum), so results are bit-identical.
"""
from __future__ import annotations

from .fd_operators import Laplace


class FDHamiltonian:
    def __init__(self, gd, *, kin_stencil=3, dtype=float):
        self.gd = gd
        self.kin = Laplace(gd, -0.5, kin_stencil, dtype)

    def apply_local_potential(self, vt_R, psit_nR, out, phase_cd=None):
        """out[n] = kin(psit[n]) + psit[n] * vt (gpaw/new/fd/hamiltonian.py:
        23-32).  ``phase_cd`` carries the Bloch phases of the k-point (the
        reference takes them from the array's grid); ``out is psit_nR`` is
        allowed."""
        self.kin.apply_potential(psit_nR, out, vt_R, phase_cd)
