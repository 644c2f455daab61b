"""Compound operator with per-point weights (drop-in for
gpaw/wfd_operators.py).

``WeightedFDOperator(operators)`` is A = sum_i w_i(x) L_i for a list of
FDOperators on one grid; the weights are float64 grids given later with
``set_weights`` (the dielectric Poisson solver of the solvation model uses a
Laplacian and three gradients weighted by eps and its gradient,
gpaw/old/solvation/poisson.py:75-85).  ``apply``, ``relax`` and
``get_diagonal_element`` run on the sm_100a kernels of ``gb_wfd.cu``.
"""
from __future__ import annotations

import numpy as np

from . import cgpaw
from .fd_operators import FDOperator


class WeightedFDOperator(FDOperator):
    def __init__(self, operators):
        """gpaw/wfd_operators.py:8-62: every operator's stencil is stored
        with offset 0 first (a zero coefficient is put there when the
        operator has no centre point); the weights come from set_weights."""
        self.gd = operators[0].gd
        self.shape = tuple(int(x) for x in self.gd.n_c)
        self.coef_ps = []
        self.offset_ps = []
        for op in operators:
            assert op.gd is self.gd or \
                (tuple(op.gd.N_c) == tuple(self.gd.N_c) and
                 tuple(op.gd.pbc_c) == tuple(self.gd.pbc_c))
            assert operators[0].dtype == op.dtype
            assert not hasattr(op, 'nweights')
            if 0 in op.offset_p:
                assert op.offset_p[0] == 0
                self.offset_ps.append(np.ascontiguousarray(op.offset_p.copy()))
                self.coef_ps.append(np.ascontiguousarray(op.coef_p.copy()))
            else:
                self.offset_ps.append(
                    np.ascontiguousarray(np.hstack(([0], op.offset_p))))
                self.coef_ps.append(
                    np.ascontiguousarray(np.hstack(([.0], op.coef_p))))
        self.nweights = len(operators)
        self.cfd = all(op.cfd for op in operators)
        self.mp = max(op.mp for op in operators)
        self.dtype = operators[0].dtype
        self.comm = None
        self.npoints = max(op.npoints for op in operators)
        self.weights = None
        self.operator = None
        self.description = 'Weighted Finite Difference Operator\n      '
        self.description += '\n      '.join(op.description
                                            for op in operators)
        self.xp = None

    def set_weights(self, weights):
        """gpaw/wfd_operators.py:64-81: ``weights`` is a list of float64
        CUDA tensors of the grid shape, one per operator (not copied)."""
        assert len(weights) == self.nweights
        for weight in weights:
            assert tuple(weight.shape) == self.shape
            assert weight.dtype.is_floating_point and \
                weight.element_size() == 8 and not weight.is_complex()
            assert weight.is_contiguous()
        self.weights = weights
        # each operator's offsets are flattened with its own padding and
        # read with the common range mp, as the reference passes them
        # (identical when the operators share mp, as the solvation
        # solver's do)
        self.operator = cgpaw.WOperator(
            self.nweights, self.weights, self.coef_ps, self.offset_ps,
            self.gd.n_c, self.mp, self.gd.neighbor_cd, self.dtype == float,
            None, self.cfd)

    def _require_weights(self):
        if self.operator is None:
            raise RuntimeError('WeightedFDOperator: call set_weights first')

    def apply(self, in_xg, out_xg, phase_cd=None):
        self._require_weights()
        self.operator.apply(in_xg, out_xg, phase_cd)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        self._require_weights()
        self.operator.relax(relax_method, f_g, s_g, n,
                            1.0 if w is None else w)

    def get_diagonal_element(self):
        self._require_weights()
        return self.operator.get_diagonal_element()

    def get_async_sizes(self):
        return (0, 1, 1)
