"""Restatement of the reference's Python layer on the FD hot path.

TEST INFRASTRUCTURE ONLY (the oracle).  It drives either the reference's own
C core compiled from source (``oracle/_ref/_gpaw_ref*.so``, built by
``oracle/Makefile``) or, where that library is absent, the numpy restatement
in ``oracle/port.py``.  The ``gpaw_b200`` package never imports it.

Restated from (all single-domain, ``comm.size == 1``):

* grid conventions  gpaw/old/grid_descriptor.py:119-160, 327-342
* neighbours        gpaw/old/domain.py:110-138
* Bloch phases      gpaw/core/uniform_grid.py:116-127
* Laplacian         gpaw/fd_operators.py:27-34, 43-97, 184-238
* transformer pads  gpaw/transformers.py:19-77
* Poisson solver    gpaw/poisson.py:182-213, 321-537
* preconditioner    gpaw/preconditioner.py:9-93
* weighted operator gpaw/wfd_operators.py:7-81 (C object: the reference's
  WOperator), dielectric solver gpaw/old/solvation/poisson.py:48-124,
  checked against gpaw/test/solvation/test_poisson.py:46-156
* density transfers gpaw/new/fd/pot_calc.py:37-41, 72-80
* dipole layer      gpaw/dipole_correction.py:84-172
* extra vacuum      gpaw/poisson_extravacuum.py:13-232, with
  gpaw/utilities/extend_grid.py:8-56; pinned to the golden differences of
  gpaw/test/poisson/test_poisson_extravacuum.py:100-129
* moment correction gpaw/poisson_moment.py:60-243 with the Gaussian
  multipoles of gpaw/utilities/gauss.py:11-160 written from their
  definitions, pinned to the reference's own known-answer test of them
  (gpaw/test/test_gauss_func.py:19-54: unit moments on its 48^3 grid);
  the reference's Python layer cannot be imported here, so no output of
  its own multipole code is compared
"""
from __future__ import annotations

import glob
import importlib.util
import os
from math import pi

import numpy as np

from . import port

_HERE = os.path.dirname(os.path.abspath(__file__))


def load_ref():
    """Import the compiled reference core, or return None if not built."""
    hits = glob.glob(os.path.join(_HERE, '_ref', '_gpaw_ref*.so'))
    if not hits:
        return None
    spec = importlib.util.spec_from_file_location('_gpaw_ref', hits[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


_REF = load_ref()


def backend(name='auto'):
    """'ref' = compiled reference core, 'port' = numpy restatement."""
    if name == 'ref' or (name == 'auto' and _REF is not None):
        if _REF is None:
            raise RuntimeError('reference core not built (make -C oracle)')
        return _REF
    return port


class BadGridError(ValueError):
    pass


class PoissonConvergenceError(RuntimeError):
    pass


# Chelikowsky et al., PRB 50, 11355 (1994); gpaw/fd_operators.py:27-34
LAPLACE = [[0],
           [-2, 1],
           [-5 / 2, 4 / 3, -1 / 12],
           [-49 / 18, 3 / 2, -3 / 20, 1 / 90],
           [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560],
           [-5269 / 1800, 5 / 3, -5 / 21, 5 / 126, -5 / 1008, 1 / 3150],
           [-5369 / 1800, 12 / 7, -15 / 56, 10 / 189, -1 / 112, 2 / 1925,
            -1 / 16632]]


class GridDescriptor:
    """Single-domain grid descriptor (gpaw/old/grid_descriptor.py)."""

    def __init__(self, N_c, cell_cv=(1, 1, 1), pbc_c=True):
        if isinstance(pbc_c, (bool, int, np.bool_)):
            pbc_c = (bool(pbc_c),) * 3
        self.pbc_c = np.array(pbc_c, bool)
        self.N_c = np.array(N_c, int)
        cell = np.array(cell_cv, float)
        if cell.ndim == 0:
            cell = np.eye(3) * cell
        elif cell.ndim == 1:
            cell = np.diag(cell)
        self.cell_cv = cell
        self.beg_c = np.empty(3, int)
        self.end_c = np.empty(3, int)
        for c in range(3):
            # gpaw/old/grid_descriptor.py:136-152 with one domain
            n_p = np.around(np.array([0.0, float(self.N_c[c])]) + 0.4999)
            n_p = n_p.astype(int)
            if not self.pbc_c[c]:
                n_p[0] = 1
            if n_p[1] == n_p[0]:
                raise BadGridError('Grid %s too small' % self.N_c)
            self.beg_c[c] = n_p[0]
            self.end_c[c] = n_p[1]
        self.n_c = self.end_c - self.beg_c
        self.h_cv = self.cell_cv / self.N_c[:, None]
        self.volume = abs(np.linalg.det(self.cell_cv))
        self.dv = self.volume / self.N_c.prod()
        # gpaw/old/domain.py:110-138: own rank (0) or -1 across a zero BC
        self.neighbor_cd = np.where(self.pbc_c[:, None], 0, -1) * \
            np.ones((3, 2), int)
        self.neighbor_cd = np.ascontiguousarray(self.neighbor_cd, np.int64)

    def coarsen(self):
        if (self.N_c % 2).any():
            raise ValueError('Grid %s not divisible by 2!' % self.N_c)
        return GridDescriptor(self.N_c // 2, self.cell_cv, self.pbc_c)

    def refine(self):
        return GridDescriptor(self.N_c * 2, self.cell_cv, self.pbc_c)

    def zeros(self, n=(), dtype=float):
        if isinstance(n, int):
            n = (n,)
        return np.zeros(tuple(n) + tuple(self.n_c), dtype)

    def empty(self, n=(), dtype=float):
        return self.zeros(n, dtype)

    def integrate(self, a):
        return a.sum(axis=(-3, -2, -1)) * self.dv

    def phase_factor_cd(self, kpt_c):
        """gpaw/core/uniform_grid.py:116-127, one domain: disp = (+1, -1)."""
        disp_cd = np.array([[1.0, -1.0]] * 3)
        return np.exp(2j * np.pi * disp_cd * np.asarray(kpt_c)[:, None])

    def get_grid_point_coordinates(self):
        idx = np.indices(self.n_c) + self.beg_c[:, None, None, None]
        return np.einsum('cv,cxyz->vxyz', self.h_cv, idx)


class FDOperator:
    """gpaw/fd_operators.py:43-147 (single domain)."""

    def __init__(self, coef_p, offset_pc, gd, dtype=float, be='auto'):
        offset_pc = np.asarray(offset_pc, int)
        cfd = True
        for offset_c in offset_pc:
            if sum([o != 0 for o in offset_c]) >= 2:
                cfd = False
        mp = np.abs(offset_pc).max()
        assert (mp <= gd.n_c).all(), 'Stencil longer than domain'
        n_c = gd.n_c
        M_c = n_c + 2 * mp
        stride_c = np.array([M_c[1] * M_c[2], M_c[2], 1])
        offset_p = np.ascontiguousarray(np.dot(offset_pc, stride_c))
        coef_p = np.ascontiguousarray(coef_p, float)
        self.dtype = dtype
        self.shape = tuple(n_c)
        self.mp = mp
        self.gd = gd
        self.npoints = len(coef_p)
        self.coef_p = coef_p
        self.offset_p = offset_p
        self.offset_pc = offset_pc
        self.cfd = cfd
        self.operator = backend(be).Operator(
            coef_p, offset_p, np.ascontiguousarray(n_c, np.int64), int(mp),
            gd.neighbor_cd, dtype == float, None, cfd)

    def apply(self, in_xg, out_xg, phase_cd=None):
        self.operator.apply(in_xg, out_xg, phase_cd)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        self.operator.relax(relax_method, f_g, s_g, n,
                            1.0 if w is None else w)

    def get_diagonal_element(self):
        return self.operator.get_diagonal_element()


class WeightedFDOperator:
    """gpaw/wfd_operators.py:7-81: sum_i weights_i * operators_i, the
    stencils stored with offset 0 first."""

    def __init__(self, operators, be='auto'):
        self.gd = operators[0].gd
        self.shape = tuple(self.gd.n_c)
        self.coef_ps = []
        self.offset_ps = []
        for op in operators:
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
        self.cfd = all([op.cfd for op in operators])
        self.mp = max([op.mp for op in operators])
        self.dtype = operators[0].dtype
        self.be = be
        self.operator = None

    def set_weights(self, weights):
        assert len(weights) == self.nweights
        self.weights = [np.ascontiguousarray(w, float) for w in weights]
        self.operator = backend(self.be).WOperator(
            self.nweights, self.weights, self.coef_ps,
            [np.ascontiguousarray(o, np.int64) for o in self.offset_ps],
            np.ascontiguousarray(self.gd.n_c, np.int64), int(self.mp),
            self.gd.neighbor_cd, self.dtype == float, None, self.cfd)

    def apply(self, in_xg, out_xg, phase_cd=None):
        self.operator.apply(in_xg, out_xg, phase_cd)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        self.operator.relax(relax_method, f_g, s_g, n,
                            1.0 if w is None else w)

    def get_diagonal_element(self):
        return self.operator.get_diagonal_element()


def laplace_stencil(gd, scale=1.0, n=1):
    """Coefficients and offsets of GUCLaplace (gpaw/fd_operators.py:184-238)."""
    M_ic = np.indices((3, 3, 3)).reshape((3, -3)).T[-13:] - 1
    u_cv = gd.h_cv / (gd.h_cv**2).sum(1)[:, np.newaxis]**0.5
    u2_i = (np.dot(M_ic, u_cv)**2).sum(1)
    i_d = u2_i.argsort()
    m_mv = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2),
                     (0, 1, 1), (1, 0, 1), (1, 1, 0)])
    for D in range(3, 7):
        h_dv = np.dot(M_ic[i_d[:D]], gd.h_cv)
        A_md = (h_dv**m_mv[:, np.newaxis, :]).prod(2)
        a_d, residual, rank, s = np.linalg.lstsq(A_md, [1, 1, 1, 0, 0, 0],
                                                 rcond=-1)
        if residual.sum() < 1e-14:
            if rank != D:
                raise ValueError('weird unit cell')
            break
    a_d *= scale
    offsets = [(0, 0, 0)]
    coefs = [LAPLACE[n][0] * a_d.sum()]
    for d in range(D):
        M_c = M_ic[i_d[d]]
        offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(LAPLACE[n][1:]))
        offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(LAPLACE[n][1:]))
    return coefs, offsets


def Laplace(gd, scale=1.0, n=1, dtype=float, be='auto'):
    coefs, offsets = laplace_stencil(gd, scale, n)
    return FDOperator(coefs, offsets, gd, dtype, be=be)


def ft_laplace(gd, scale, in_xg):
    """FTLaplace.apply (gpaw/fd_operators.py:399-421) in numpy: the full
    transforms of every grid of in_xg times -scale |k|^2, real part."""
    N_c1 = gd.N_c[:, np.newaxis]
    i_cq = np.indices(gd.N_c).reshape((3, -1))
    i_cq = (i_cq + N_c1 // 2) % N_c1 - N_c1 // 2
    icell_cv = np.linalg.inv(gd.cell_cv).T
    k_vq = np.dot(2.0 * pi * icell_cv.T, i_cq)
    k2_Q = (k_vq**2).sum(axis=0).reshape(gd.N_c) * (-scale)
    ax = (-3, -2, -1)
    out = np.fft.ifftn(np.fft.fftn(in_xg, axes=ax) * k2_Q, axes=ax).real
    return out.astype(in_xg.dtype)


def _mehrstellen_a(gd, scale):
    """LaplaceA's coefficients and offsets (gpaw/fd_operators.py:357-384)."""
    c = np.divide(-1 / 12, gd.h_cv.diagonal()**2) * scale
    c0 = c[1] + c[2]
    c1 = c[0] + c[2]
    c2 = c[1] + c[0]
    a = -16.0 * np.sum(c)
    b = 10.0 * c + 0.125 * a
    coefs = [a, b[0], b[0], b[1], b[1], b[2], b[2],
             c0, c0, c0, c0, c1, c1, c1, c1, c2, c2, c2, c2]
    offsets = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0),
               (0, 0, -1), (0, 0, 1),
               (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
               (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1),
               (-1, -1, 0), (-1, 1, 0), (1, -1, 0), (1, 1, 0)]
    return coefs, offsets


def LaplaceA(gd, scale, dtype=float, be='auto'):
    """O(h^4) Mehrstellen Laplacian, A (gpaw/fd_operators.py:357-384)."""
    return FDOperator(*_mehrstellen_a(gd, scale), gd, dtype, be=be)


def LaplaceB(gd, dtype=float, be='auto'):
    """Mehrstellen right-hand-side operator B (:387-396)."""
    b = 1.0 / 12.0
    return FDOperator([0.5, b, b, b, b, b, b],
                      [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0),
                       (0, 1, 0), (0, 0, -1), (0, 0, 1)], gd, dtype, be=be)


def transformer_geometry(gdin, gdout, nn):
    """Pads, neighbour pads and skip flags (gpaw/transformers.py:19-77)."""
    pad_cd = np.empty((3, 2), int)
    neighborpad_cd = np.empty((3, 2), int)
    skip_cd = np.empty((3, 2), int)
    if (gdin.N_c == 2 * gdout.N_c).all():
        pad_cd[:, 0] = 2 * nn - 1 - 2 * gdout.beg_c + gdin.beg_c
        pad_cd[:, 1] = 2 * nn - 2 + 2 * gdout.end_c - gdin.end_c
        neighborpad_cd[:, 0] = 2 * nn - 2 + 2 * gdout.beg_c - gdin.beg_c
        neighborpad_cd[:, 1] = 2 * nn - 1 - 2 * gdout.end_c + gdin.end_c
        interpolate = False
    else:
        assert (gdout.N_c == 2 * gdin.N_c).all()
        pad_cd[:, 0] = nn - 1 - gdout.beg_c // 2 + gdin.beg_c
        pad_cd[:, 1] = nn + gdout.end_c // 2 - gdin.end_c
        neighborpad_cd[:, 0] = nn + gdout.beg_c // 2 - gdin.beg_c
        neighborpad_cd[:, 1] = nn - 1 - gdout.end_c // 2 + gdin.end_c
        skip_cd[:, 0] = gdout.beg_c % 2
        skip_cd[:, 1] = gdout.end_c % 2
        interpolate = True
        inpoints = (gdin.n_c[0] + 2 * nn - 1) * (gdin.n_c[1] + 2 * nn - 1)
        outpoints = gdout.n_c[0] * gdout.n_c[1]
        if inpoints > outpoints:
            raise ValueError('Cannot construct interpolator.')
        # The reference's first interpolation pass writes s0 * s1 * o2 values
        # into the output array (c/bmgs/interpolate.cpp:87-90); its guard above
        # uses 2nn - 1 where the padded extent is n + 2nn, so some grids pass
        # the guard and still overflow the heap.  Refuse those here so that
        # the oracle never runs the reference into undefined behaviour.
        s_c = gdin.n_c + pad_cd.sum(1)
        if s_c[0] * s_c[1] > gdout.n_c[0] * gdout.n_c[1]:
            raise ValueError('grid too small for the reference interpolator '
                             '(its scratch would overflow)')
    if not interpolate:
        skip_cd[:] = 0
    assert (pad_cd.ravel() >= 0).all()
    return pad_cd, neighborpad_cd, skip_cd, interpolate


class Transformer:
    """gpaw/transformers.py:18-94."""

    def __init__(self, gdin, gdout, nn=1, dtype=float, be='auto'):
        self.gdin = gdin
        self.gdout = gdout
        self.nn = nn
        self.dtype = dtype
        pad, npad, skip, self.interpolate = transformer_geometry(gdin, gdout,
                                                                 nn)
        self.pad_cd, self.neighborpad_cd, self.skip_cd = pad, npad, skip
        self.transformer = backend(be).Transformer(
            np.ascontiguousarray(gdin.n_c, np.int64),
            np.ascontiguousarray(gdout.n_c, np.int64), 2 * nn,
            np.ascontiguousarray(pad, np.int64),
            np.ascontiguousarray(npad, np.int64),
            np.ascontiguousarray(skip, np.int64),
            gdin.neighbor_cd, dtype == float, None, self.interpolate)

    def apply(self, input, output=None, phases=None):
        if output is None:
            output = self.gdout.zeros(input.shape[:-3], self.dtype)
        self.transformer.apply(input, output, phases)
        return output


def gauss_l0(gd, a=19.0):
    """Gaussian(gd).get_gauss(0) and .get_gauss_pot(0) with the centre in
    the middle of the cell (gpaw/utilities/gauss.py:33-56, 94-123;
    coordinates: gpaw/utilities/tools.py:81-100; distance vectors:
    gpaw/old/grid_descriptor.py:716-737, no periodic axis here)."""
    rho, phi, _, _, _ = _gauss_l0_parts(gd, a)
    return rho, phi


def _gauss_l0_parts(gd, a=19.0):
    """gauss_l0 plus the distance vectors, r^2 and the exponent a."""
    from scipy.special import erf
    origin = 0.5 * gd.cell_cv.sum(0)
    s_Gc = (np.indices(gd.n_c, float).T + gd.beg_c) / gd.N_c
    r_c = np.linalg.solve(gd.cell_cv.T, origin)
    r_c = np.where(gd.pbc_c, r_c % 1.0, r_c)
    s_Gc -= np.where(gd.pbc_c, r_c % 1.0, r_c)
    s_Gc -= gd.pbc_c * (2 * s_Gc).astype(int)
    r_vG = np.dot(s_Gc, gd.cell_cv).T.copy()
    r2 = np.sum(r_vG**2, axis=0)
    r2 = np.where(r2 < 1e-12, 1e-12, r2)
    r = np.sqrt(r2)
    icell_cv = np.linalg.inv(gd.cell_cv).T
    a = 4 * a * (icell_cv**2).sum(1).max()
    exp_ar2 = np.exp(-a * r2)
    rho = np.sqrt(a**3 * 4) / pi * exp_ar2
    phi = 2.0 * 1.7724538509055159 * erf(np.sqrt(a) * r) / r
    return rho, phi, r_vG, r2, a


# ---------------------------------------------------- Gaussian multipoles
# gpaw/utilities/gauss.py:11-92 (Y_L, gauss_L, gausspot_L for L = 0..8) and
# :95-160 (Gaussian), written from the definitions: Y_L = r^l times the real
# harmonic (order 1; y, z, x; xy, yz, 3z^2 - r^2, xz, x^2 - y^2), g_L of unit
# moment int g_L Y_L dV = 1, v_L its potential (del^2 v_L = -4 pi g_L).
_MP_L = (0, 1, 1, 1, 2, 2, 2, 2, 2)
_MP_NORM = (1 / 4, 3 / 4, 3 / 4, 3 / 4, 15 / 4, 15 / 4, 5 / 16, 15 / 4, 15 / 16)


def _mp_poly(L, x, y, z, r2):
    if L == 0:
        return np.ones_like(r2)
    return (y, z, x, x * y, y * z, 3 * z * z - r2, x * z, x * x - y * y)[L - 1]


def mp_Y(L, x, y, z, r2):
    return np.sqrt(_MP_NORM[L] / pi) * _mp_poly(L, x, y, z, r2)


def mp_gauss(a, L, x, y, z, r2, exp_ar2):
    from math import gamma
    l = _MP_L[L]
    c = np.sqrt(_MP_NORM[L] / pi)
    k = (2 * pi * c / gamma(l + 1.5))**2
    return np.sqrt(a**(2 * l + 3) * k) / pi * _mp_poly(L, x, y, z, r2) * \
        exp_ar2


def mp_gausspot(a, L, x, y, z, r, r2, erf_sar, exp_ar2):
    l = _MP_L[L]
    c = np.sqrt(_MP_NORM[L] / pi)
    sa = np.sqrt(a) * r
    if l == 0:
        rad, e0 = erf_sar, 1.0
    elif l == 1:
        rad, e0 = np.sqrt(pi) * erf_sar - 2 * sa * exp_ar2, np.sqrt(pi)
    else:
        rad = 3 * np.sqrt(pi) * erf_sar - (6 + 4 * sa**2) * sa * exp_ar2
        e0 = 3 * np.sqrt(pi)
    return 4 * pi * c / ((2 * l + 1) * e0) * rad / r**(2 * l + 1) * \
        _mp_poly(L, x, y, z, r2)


class GaussianMP:
    """Gaussian(gd, a, center) (gpaw/utilities/gauss.py:95-160) on numpy
    grids; coordinates as gpaw/utilities/tools.py:81-100 forms them."""

    def __init__(self, gd, a=19., center=None):
        from scipy.special import erf
        self.gd = gd
        origin = 0.5 * gd.cell_cv.sum(0) if center is None else \
            np.asarray(center, float)
        s_Gc = (np.indices(gd.n_c, float).T + gd.beg_c) / gd.N_c
        r_c = np.linalg.solve(gd.cell_cv.T, origin)
        s_Gc -= np.where(gd.pbc_c, r_c % 1.0, r_c)
        s_Gc -= gd.pbc_c * (2 * s_Gc).astype(int)
        self.xyz = np.dot(s_Gc, gd.cell_cv).T.copy()
        r2 = np.sum(self.xyz**2, axis=0)
        self.r2 = np.where(r2 < 1e-12, 1e-12, r2)
        self.r = np.sqrt(self.r2)
        if center is None:
            icell_cv = np.linalg.inv(gd.cell_cv).T
            self.a = 4 * a * (icell_cv**2).sum(1).max()
        else:
            cell_center = gd.cell_cv.sum(1) / 2
            r_min = (cell_center - np.abs(center - cell_center)).min()
            self.a = a / r_min**2
        self.exp_ar2 = np.exp(-self.a * self.r2)
        self.erf_sar = erf(np.sqrt(self.a) * self.r)

    def get_gauss(self, L):
        x, y, z = self.xyz
        return mp_gauss(self.a, L, x, y, z, self.r2, self.exp_ar2)

    def get_gauss_pot(self, L):
        x, y, z = self.xyz
        return mp_gausspot(self.a, L, x, y, z, self.r, self.r2,
                           self.erf_sar, self.exp_ar2)

    def get_moment(self, n, L):
        x, y, z = self.xyz
        return self.gd.integrate(n * mp_Y(L, x, y, z, self.r2))

    def remove_moment(self, n, L, q=None):
        if q is None:
            q = self.get_moment(n, L)
        if abs(q) < 1e-7:
            return 0.
        n -= q * self.get_gauss(L)
        return q * self.get_gauss_pot(L)


class MomentCorrectionPoissonSolver:
    """gpaw/poisson_moment.py:60-243: moments ``moms`` about each centre
    (Bohr; None = the middle of the cell) removed with Gaussian multipoles,
    every grid point assigned to its nearest centre."""

    def __init__(self, poissonsolver, moment_corrections):
        self.poissonsolver = poissonsolver
        if isinstance(moment_corrections, int):
            moment_corrections = [{'moms': range(moment_corrections),
                                   'center': None}]
        self.moment_corrections = moment_corrections

    def set_grid_descriptor(self, gd):
        self.poissonsolver.set_grid_descriptor(gd)
        self.gd = gd
        self.gauss_i = [GaussianMP(gd, center=m['center'])
                        for m in moment_corrections_list(self)]
        self.mom_ij = [np.asarray(m['moms'])
                       for m in moment_corrections_list(self)]
        r_ir = np.array([g.r.ravel() for g in self.gauss_i])
        mask_ir = np.zeros(r_ir.shape, int)
        for r in range(r_ir.shape[1]):
            mask_ir[np.argmin(r_ir[:, r]), r] = 1
        self.mask_ig = [m.reshape(gd.n_c) for m in mask_ir]

    def solve(self, phi, rho, **kwargs):
        rho_neutral = rho * 0.0
        phi_cor_g = self.gd.zeros()
        for gauss, mask_g, mom_j in zip(self.gauss_i, self.mask_ig,
                                        self.mom_ij):
            rho_masked = rho * mask_g
            for mom in mom_j:
                phi_cor_g += gauss.remove_moment(rho_masked, mom)
            rho_neutral += rho_masked
        phi -= phi_cor_g
        niter = self.poissonsolver.solve(phi, rho_neutral, **kwargs)
        phi += phi_cor_g
        return niter


def moment_corrections_list(ps):
    return ps.moment_corrections


# ------------------------------------------------------------ extra vacuum
def extended_gd(gd, N_c):
    """gpaw/utilities/extend_grid.py:8-44 with a target size N_c."""
    N_c = np.array(N_c, dtype=int)
    ext = np.tile((N_c - gd.N_c) // 2, (2, 1)).T
    egd = GridDescriptor(N_c, gd.h_cv * N_c, gd.pbc_c)
    egd.extend_N_cd = ext
    return egd


def _window(gd, egd):
    o = egd.extend_N_cd[:, 0]
    return tuple(slice(o[c], o[c] + gd.n_c[c]) for c in range(3))


class ExtraVacuumPoissonSolver:
    """gpaw/poisson_extravacuum.py:13-232 (one domain, zero boundary);
    grid2grid between a grid and its extension is the copy of the
    overlapping window (gpaw/utilities/grid.py:127-162)."""

    def __init__(self, gpts, ps_large, ps_small=None, coarses=0,
                 nn_coarse=3, nn_refine=3, nn_laplace=3, use_aux_grid=True,
                 be='auto'):
        self.N_large = np.array(gpts, dtype=int)
        self.Ncoar = coarses
        self.ps_large, self.ps_small = ps_large, ps_small
        self.nn_coarse, self.nn_refine = nn_coarse, nn_refine
        self.nn_laplace, self.use_aux = nn_laplace, use_aux_grid
        self.be = be

    def set_grid_descriptor(self, gd):
        self.gd_sf = gd
        N_c = self.N_large.copy()
        self.coarser = []
        for _ in range(self.Ncoar):
            gd2 = gd.coarsen()
            self.coarser.append(Transformer(gd, gd2, self.nn_coarse,
                                            be=self.be))
            N_c //= 2
            gd = gd2
        self.gd_sc = gd
        self.gd_lc = extended_gd(self.gd_sc, N_c)
        self.ps_large.set_grid_descriptor(self.gd_lc)
        self.phi_lc = self.gd_lc.zeros()
        if self.Ncoar == 0:
            return
        self.ps_small.set_grid_descriptor(self.gd_sf)
        if self.use_aux:
            buf = self.nn_refine
            for _ in range(self.Ncoar):
                buf = 2 * buf + self.nn_refine
            buf += self.nn_laplace
            div = 2**self.Ncoar
            if buf % div != 0:
                buf += div - buf % div
            N_c = self.gd_sf.N_c + 2 * buf
            if np.any(N_c > self.N_large):
                self.use_aux = False
                N_c = self.N_large
            self.gd_af = extended_gd(self.gd_sf, N_c)
        else:
            self.gd_af = extended_gd(self.gd_sf, self.N_large)
        self.lap = Laplace(self.gd_af, -0.25 / pi, self.nn_laplace,
                           be=self.be)
        self.refiner = []
        gd = self.gd_af
        for _ in range(self.Ncoar):
            gd2 = gd.coarsen()
            self.refiner.append(Transformer(gd2, gd, self.nn_refine,
                                            be=self.be))
            gd = gd2
        self.refiner = self.refiner[::-1]
        self.gd_ac = gd
        if self.use_aux:
            self.gd_lc_aux = extended_gd(self.gd_ac, self.gd_lc.N_c)

    def solve(self, phi, rho):
        rho_sf = rho.copy()
        tmp = rho_sf
        for t in self.coarser:
            tmp = t.apply(tmp)
        rho_lc = self.gd_lc.zeros()
        rho_lc[_window(self.gd_sc, self.gd_lc)] = tmp
        n_large = self.ps_large.solve(self.phi_lc, rho_lc)
        if self.Ncoar == 0:
            phi[:] = self.phi_lc[_window(self.gd_sf, self.gd_lc)]
            return n_large
        if self.use_aux:
            tmp = self.phi_lc[_window(self.gd_ac, self.gd_lc_aux)].copy()
        else:
            tmp = self.phi_lc
        for t in self.refiner:
            tmp = t.apply(tmp)
        rho_af = self.gd_af.zeros()
        self.lap.apply(tmp, rho_af)
        w = _window(self.gd_sf, self.gd_af)
        cor_phi = tmp[w].copy()
        cor_rho = rho_af[w].copy()
        rho_sf -= cor_rho
        phi -= cor_phi
        n_small = self.ps_small.solve(phi, rho_sf)
        phi += cor_phi
        return (n_large, n_small)


class FDPoissonSolver:
    """gpaw/poisson.py:321-537 (neutral, periodic-charged and non-periodic
    charged (Gaussian monopole) branches)."""

    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000, be='auto'):
        self.nn = nn
        self.eps = eps
        self.maxiter = maxiter
        self.relax = relax
        self.relax_method = {'GS': 1, 'J': 2}[relax]
        self.be = be
        self._initialized = False

    def set_grid_descriptor(self, gd):
        self.gd = gd
        scale = -0.25 / pi
        if self.nn == 'M':
            # :371-377: Mehrstellen A on level 0, B applied to rho
            self.operators = [LaplaceA(gd, -scale, be=self.be)]
            self.B = LaplaceB(gd, be=self.be)
        else:
            self.operators = [Laplace(gd, scale, self.nn, be=self.be)]
            self.B = None
        self.interpolators = []
        self.restrictors = []
        level = 0
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2.0 / 3.0]
        while level < 8:
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.operators.append(Laplace(gd2, scale, 1, be=self.be))
            self.interpolators.append(Transformer(gd2, gd, be=self.be))
            self.restrictors.append(Transformer(gd, gd2, be=self.be))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level
        self._initialized = False

    def _init(self):
        if self._initialized:
            return
        gd = self.gd
        self.rhos = [gd.empty()]
        self.phis = [None]
        self.residuals = [gd.empty()]
        for level in range(self.levels):
            gd2 = gd.coarsen()
            self.phis.append(gd2.empty())
            self.rhos.append(gd2.empty())
            self.residuals.append(gd2.empty())
            gd = gd2
        level = self.levels
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()
        self.presmooths[level] = 8
        self.postsmooths[level] = 8
        self._initialized = True

    def solve(self, phi, rho, charge=None, maxcharge=1e-6,
              zero_initial_phi=False):
        """gpaw/poisson.py:182-213 (+ periodic charged :217-231)."""
        self._init()
        actual_charge = self.gd.integrate(rho)
        # get_size_of_global_array() = N_c - 1 + pbc_c = n_c on one domain
        # (gpaw/old/grid_descriptor.py:214-218)
        background = (actual_charge / self.gd.dv / self.gd.n_c.prod())
        if charge is None:
            charge = actual_charge
        if abs(charge) <= maxcharge:
            return self.solve_neutral(phi, rho - background)
        if self.gd.pbc_c.all():
            if zero_initial_phi:
                phi[:] = 0.0
            return self.solve_neutral(phi, rho - background)
        if not self.gd.pbc_c.any():
            # :233-283 without use_charge_center: Gaussian monopole removal
            if not hasattr(self, 'rho_gauss'):
                self.rho_gauss, self.phi_gauss = gauss_l0(self.gd)
            q = actual_charge / np.sqrt(4 * pi)
            rho_neutral = rho - q * self.rho_gauss
            if zero_initial_phi:
                phi[:] = 0.0
            else:
                phi -= q * self.phi_gauss
            niter = self.solve_neutral(phi, rho_neutral)
            phi += q * self.phi_gauss
            return niter
        raise NotImplementedError('charged system, mixed boundaries')

    def solve_neutral(self, phi, rho):
        self._init()
        self.phis[0] = phi
        if self.B is None:
            self.rhos[0][:] = rho
        else:
            self.B.apply(rho, self.rhos[0])
        niter = 1
        self.errors = []
        while self.iterate2(self.step) > self.eps and niter < self.maxiter:
            niter += 1
        if niter == self.maxiter:
            raise PoissonConvergenceError('did not converge')
        if self.gd.pbc_c.all():
            phi_ave = float(np.sum(phi.ravel()))
            phi_ave /= np.prod(self.gd.n_c)
            phi -= phi_ave
        return niter

    def iterate2(self, step, level=0):
        residual = self.residuals[level]
        if level < self.levels:
            self.operators[level].relax(self.relax_method, self.phis[level],
                                        self.rhos[level],
                                        self.presmooths[level],
                                        self.weights[level])
            self.operators[level].apply(self.phis[level], residual)
            residual -= self.rhos[level]
            self.restrictors[level].apply(residual, self.rhos[level + 1])
            self.phis[level + 1][:] = 0.0
            self.iterate2(4.0 * step, level + 1)
            self.interpolators[level].apply(self.phis[level + 1], residual)
            self.phis[level] -= residual
        self.operators[level].relax(self.relax_method, self.phis[level],
                                    self.rhos[level],
                                    self.postsmooths[level],
                                    self.weights[level])
        if level == 0:
            self.operators[level].apply(self.phis[level], residual)
            residual -= self.rhos[level]
            error = float(np.dot(residual.ravel(), residual.ravel())) * \
                self.gd.dv
            self.errors.append(error)
            return error


class WeightedFDPoissonSolver(FDPoissonSolver):
    """gpaw/old/solvation/poisson.py:75-124, neutral systems: the V-cycle of
    FDPoissonSolver on WeightedFDOperator([Laplace, d/dx, d/dy, d/dz])
    weighted by eps and its gradient (div(eps grad phi) = -4 pi rho); the
    weights of each coarser level are the restrictions of the finer ones.
    ``stencils(gd, scale, n)`` returns the four (coefs, offsets_pc) pairs
    of a level (the Laplacian first)."""

    def __init__(self, stencils, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 be='auto'):
        super().__init__(nn, relax, eps, maxiter, be)
        self.stencils = stencils
        self.eps_gradeps = None

    def set_dielectric(self, eps_gradeps):
        self.eps_gradeps = [np.ascontiguousarray(a, float)
                            for a in eps_gradeps]

    def set_grid_descriptor(self, gd):
        super().set_grid_descriptor(gd)
        scale = -0.25 / pi
        gds = [gd]
        for _ in range(self.levels):
            gds.append(gds[-1].coarsen())
        self.operators = [
            WeightedFDOperator([FDOperator(c, o, g, be=self.be) for c, o in
                                self.stencils(g, scale,
                                              self.nn if i == 0 else 1)],
                               be=self.be)
            for i, g in enumerate(gds)]
        self.gds = gds

    def _init(self):
        """:113-124: level 0 weighted by the dielectric, coarser levels by
        arrays that restrict_op_weights fills."""
        if self._initialized:
            return
        self.operators[0].set_weights(self.eps_gradeps)
        self.op_coarse_weights = []
        for op, g in zip(self.operators[1:], self.gds[1:]):
            weights = [g.zeros() for _ in range(4)]
            self.op_coarse_weights.append(weights)
            op.set_weights(weights)
        super()._init()

    def restrict_op_weights(self):
        """:100-106."""
        self._init()
        weights = [self.operators[0].weights] + self.op_coarse_weights
        for i, res in enumerate(self.restrictors):
            for j in range(4):
                res.apply(weights[i][j], weights[i + 1][j])
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()

    def load_gauss(self):
        """:48-72: the compensation charge of a charged system in the
        dielectric, rho = eps g - (grad v_g . grad eps) / (4 pi), normalised
        to sqrt(4 pi), and its potential v_g with the same factor."""
        from scipy.special import erf
        epsr, dx_epsr, dy_epsr, dz_epsr = self.eps_gradeps
        rho_g, phi_g, xyz, r2, a = _gauss_l0_parts(self.gd)
        r = np.sqrt(r2)
        x, y, z = xyz
        fac = 2. * np.sqrt(a) * np.exp(-a * r2)
        fac /= np.sqrt(np.pi) * r2
        fac -= erf(np.sqrt(a) * r) / (r2 * r)
        fac *= 2.0 * 1.7724538509055159
        dx_phi_g = fac * x
        dy_phi_g = fac * y
        dz_phi_g = fac * z
        sp = dx_phi_g * dx_epsr + dy_phi_g * dy_epsr + dz_phi_g * dz_epsr
        rho = epsr * rho_g - 1. / (4. * np.pi) * sp
        invnorm = np.sqrt(4. * np.pi) / self.gd.integrate(rho)
        self.phi_gauss = phi_g * invnorm
        self.rho_gauss = rho * invnorm

    def solve(self, phi, rho, charge=None, maxcharge=1e-6,
              zero_initial_phi=False):
        """:87-98: periodic systems must be neutral; a charged
        non-periodic one gets the dielectric's compensation charge."""
        self._init()
        if self.gd.pbc_c.all() and abs(self.gd.integrate(rho)) > maxcharge:
            raise NotImplementedError(
                'charged periodic systems are not implemented')
        self.restrict_op_weights()
        if not hasattr(self, 'rho_gauss'):
            self.load_gauss()
        return super().solve(phi, rho, charge, maxcharge, zero_initial_phi)


class Preconditioner:
    """gpaw/preconditioner.py:9-73 (C path)."""

    def __init__(self, gd0, kin0, dtype=float, block=1, be='auto'):
        gd1 = gd0.coarsen()
        gd2 = gd1.coarsen()
        self.be = backend(be)
        self.kin0 = kin0
        self.kin1 = Laplace(gd1, -0.5, 1, dtype, be=be)
        self.kin2 = Laplace(gd2, -0.5, 1, dtype, be=be)
        self.scratch0 = gd0.zeros((2, block), dtype)
        self.scratch1 = gd1.zeros((3, block), dtype)
        self.scratch2 = gd2.zeros((3, block), dtype)
        self.step = 0.66666666 / kin0.get_diagonal_element()
        self.restrictor_object0 = Transformer(gd0, gd1, 1, dtype, be=be)
        self.restrictor_object1 = Transformer(gd1, gd2, 1, dtype, be=be)
        self.interpolator_object2 = Transformer(gd2, gd1, 1, dtype, be=be)
        self.interpolator_object1 = Transformer(gd1, gd0, 1, dtype, be=be)

    def __call__(self, residuals, phases=None, out=None):
        if residuals.ndim == 3:
            if out is None:
                return self.__call__(residuals[np.newaxis], phases)[0]
            return self.__call__(residuals[np.newaxis], phases,
                                 out=out[np.newaxis])[0]
        nb = len(residuals)
        nb0 = self.scratch0.shape[1]
        if nb > nb0:
            assert out is not None
            for n1 in range(0, nb, nb0):
                self(residuals[n1:n1 + nb0], phases, out=out[n1:n1 + nb0])
            return out
        if out is None:
            d0, q0 = self.scratch0[:, :nb]
        else:
            d0 = out
            q0 = self.scratch0[0, :nb]
        r1, d1, q1 = self.scratch1[:, :nb]
        r2, d2, q2 = self.scratch2[:, :nb]
        self.be.fd_precond(self.restrictor_object0.transformer,
                           self.restrictor_object1.transformer,
                           self.interpolator_object1.transformer,
                           self.interpolator_object2.transformer,
                           self.kin0.operator, self.kin1.operator,
                           self.kin2.operator,
                           d0, q0, r1, d1, q1, r2, d2, q2,
                           residuals, -residuals, self.step, phases)
        return d0


class FDHamiltonian:
    """gpaw/new/fd/hamiltonian.py:14-32: kinetic operator -1/2 Laplacian of
    order kin_stencil and the local-potential product."""

    def __init__(self, gd, kin_stencil=3, dtype=float, be='auto'):
        self.kin = Laplace(gd, -0.5, kin_stencil, dtype, be=be)

    def apply_local_potential(self, vt_R, psit_nR, out, phase_cd=None):
        """:23-32: ``self.kin(psit_nR, out)``, then ``o += p * vt_R`` per
        band (numpy: the product rounded, then the sum)."""
        self.kin.apply(psit_nR, out, phase_cd)
        for p, o in zip(psit_nR, out):
            o += p * vt_R


def interpolate_density(gd, finegd, nt_sR, n=3):
    """FDPotentialCalculator._interpolate_density
    (gpaw/new/fd/pot_calc.py:37-41, 72-80): interpolate with the order-2n
    transformer; off fully periodic grids rescale each spin's fine density
    to the coarse integral when the fine integral exceeds 1e-14."""
    nt_sR = np.asarray(nt_sR)
    one = nt_sR.ndim == 3
    c = nt_sR[None] if one else nt_sR
    f = np.zeros((c.shape[0],) + tuple(finegd.n_c))
    Transformer(gd, finegd, n).apply(c, f)
    if not gd.pbc_c.all():
        Nt1_s = gd.integrate(c)
        Nt2_s = finegd.integrate(f)
        for Nt1, Nt2, nt_r in zip(Nt1_s, Nt2_s, f):
            if float(Nt2) > 1e-14:
                nt_r *= Nt1 / Nt2
    return f[0] if one else f


def calculate_dipole_moment(gd, rho_g, origin_c=None):
    """gpaw/old/grid_descriptor.py:648-663 (center=False)."""
    r_cz = [np.arange(gd.beg_c[c], gd.end_c[c]) for c in range(3)]
    if origin_c is not None:
        r_cz = [r_cz[c] - origin_c[c] for c in range(3)]
    rho_01 = rho_g.sum(axis=2)
    rho_02 = rho_g.sum(axis=1)
    rho_cz = [rho_01.sum(axis=1), rho_01.sum(axis=0), rho_02.sum(axis=0)]
    rhog_c = [np.dot(r_cz[c], rho_cz[c]) for c in range(3)]
    return -np.dot(rhog_c, gd.h_cv) * gd.dv


def dipole_correction(c, gd, rhot_g, origin_c=None):
    """gpaw/dipole_correction.py:125-172 (center=False)."""
    from scipy.special import erf
    moment = calculate_dipole_moment(gd, rhot_g, origin_c)[c]
    if abs(moment) < 1e-12:
        return gd.zeros(), gd.zeros(), 0.0
    r_g = gd.get_grid_point_coordinates()[c]
    cellsize = abs(gd.cell_cv[c, c])
    sr_g = 2.0 / cellsize * r_g - 1.0
    alpha = 12.0
    drho_g = sr_g * np.exp(-alpha * sr_g**2)
    moment2 = calculate_dipole_moment(gd, drho_g, origin_c)[c]
    factor = -moment / moment2
    drho_g *= factor
    phifactor = factor * (np.pi / alpha)**1.5 * cellsize**2 / 4.0
    dphi_g = -phifactor * erf(sr_g * np.sqrt(alpha))
    return drho_g, dphi_g, phifactor


def dipole_fdsolve(poissonsolver, c, vHt_g, rhot_g, zero_vacuum=False):
    """DipoleCorrection.fdsolve (gpaw/dipole_correction.py:84-92)."""
    drhot_g, dvHt_g, correction = dipole_correction(c, poissonsolver.gd,
                                                    rhot_g)
    if zero_vacuum:
        dvHt_g += correction
    vHt_g -= dvHt_g
    iters = poissonsolver.solve(vHt_g, rhot_g + drhot_g)
    vHt_g += dvHt_g
    return iters
