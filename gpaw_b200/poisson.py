"""Finite-difference multigrid Poisson solver (drop-in for the
FDPoissonSolver of gpaw/poisson.py:321-554).

The level hierarchy, smoothing counts and weights are built exactly as the
reference builds them; one V-cycle (``iterate2``) runs in the native
executor of the C ABI (gb_poisson_*), level 0 residual norm included, so the
only host synchronisation per V-cycle is reading that norm.
"""
from __future__ import annotations

import ctypes as C
from math import pi

import numpy as np
import torch

from . import _lib
from ._lib import PoissonConvergenceError, check
from .cgpaw import _stream
from .fd_operators import Laplace
from .transformers import Transformer

__all__ = ['FDPoissonSolver', 'MixedPoissonSolver', 'PoissonConvergenceError']


class FDPoissonSolver:
    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 remove_moment=None, use_charge_center=False,
                 metallic_electrodes=False,
                 use_charged_periodic_corrections=False, xp=None):
        assert metallic_electrodes in [False, None, 'single', 'both']
        self.remove_moment = remove_moment
        self.metallic_electrodes = metallic_electrodes
        self.use_charged_periodic_corrections = \
            use_charged_periodic_corrections
        self.charged_periodic_correction = None
        self.use_charge_center = bool(use_charge_center)
        self.eps = eps
        self.relax = relax
        self.nn = nn
        self.maxiter = maxiter
        if relax == 'GS':
            self.relax_method = 1
        elif relax == 'J':
            self.relax_method = 2
        else:
            raise NotImplementedError('Relaxation method %s' % relax)
        self.description = None
        self._initialized = False
        self._exec = None

    def todict(self):
        d = {'name': 'fd', 'nn': self.nn, 'relax': self.relax,
             'eps': self.eps}
        if self.remove_moment:
            d['remove_moment'] = self.remove_moment
        if self.use_charge_center:
            d['use_charge_center'] = True
        if self.use_charged_periodic_corrections:
            d['use_charged_periodic_corrections'] = True
        if self.metallic_electrodes:
            d['metallic_electrodes'] = self.metallic_electrodes
        return d

    def get_stencil(self):
        return self.nn

    def create_laplace(self, gd, scale=1.0, n=1, dtype=float):
        return Laplace(gd, scale, n, dtype)

    def set_grid_descriptor(self, gd):
        """gpaw/poisson.py:366-430: level 0 uses the nn-order Laplacian
        scaled by -1/(4 pi), 2 pre- and 1 post-sweep with weight 2/3; every
        coarser level (up to 8, until coarsen() fails) a 2nd-order Laplacian,
        4 + 4 sweeps, weight 1."""
        self.gd = gd
        scale = -0.25 / pi
        if self.nn == 'M':
            # :371-377: Mehrstellen A on level 0; B is applied to rho
            from .fd_operators import LaplaceA, LaplaceB
            if not gd.orthogonal:
                raise RuntimeError('Cannot use Mehrstellen stencil with '
                                   'non orthogonal cell.')
            self.operators = [LaplaceA(gd, -scale)]
            self.B = LaplaceB(gd)
        else:
            self.operators = [self.create_laplace(gd, scale, self.nn)]
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
            self.operators.append(self.create_laplace(gd2, scale, 1))
            self.interpolators.append(Transformer(gd2, gd))
            self.restrictors.append(Transformer(gd, gd2))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level
        self._initialized = False
        self._exec = None

    def get_description(self):
        name = {1: 'Gauss-Seidel', 2: 'Jacobi'}[self.relax_method]
        coarsest_grid = self.operators[-1].gd.N_c
        lines = ['%s solver with %d multi-grid levels'
                 % (name, self.levels + 1),
                 '    Coarsest grid: %s points' % ' x '.join(
                     str(N) for N in coarsest_grid)]
        if coarsest_grid.max() > 24:
            lines.extend(['    Warning: Coarse grid has more than 24 points.',
                          '             More multi-grid levels recommended.'])
        lines.extend(['    Stencil: %s' % self.operators[0].description,
                      '    Max iterations: %d' % self.maxiter,
                      '    Tolerance: %e' % self.eps])
        return '\n'.join(lines)

    def _init(self):
        """gpaw/poisson.py:451-472: coarsest level smooths 8 + 8."""
        if self._initialized:
            return
        level = self.levels
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()
        self.presmooths[level] = 8
        self.postsmooths[level] = 8
        lib = _lib.load()
        nl = self.levels + 1
        ops = (C.c_void_p * nl)(*[o.operator._h for o in self.operators])
        rst = (C.c_void_p * max(1, self.levels))(
            *[t.transformer._h for t in self.restrictors])
        itp = (C.c_void_p * max(1, self.levels))(
            *[t.transformer._h for t in self.interpolators])
        pre = (C.c_int * nl)(*self.presmooths)
        post = (C.c_int * nl)(*self.postsmooths)
        w = (C.c_double * nl)(*self.weights)
        h = C.c_void_p()
        check(lib.gb_poisson_new(nl, ops, rst, itp, pre, post, w,
                                 self.relax_method, float(self.gd.dv),
                                 C.byref(h)))
        self._exec = _Exec(lib, h, self)
        self._initialized = True

    def solve(self, phi, rho, charge=None, maxcharge=1e-6,
              zero_initial_phi=False, timer=None):
        """gpaw/poisson.py:182-312: neutral systems; multipole removal
        (``remove_moment``, non-periodic cells); charged periodic ones
        (homogeneous background, plus the Madelung correction with
        ``use_charged_periodic_corrections``); charged non-periodic ones
        (Gaussian monopole); charged ones with mixed boundaries
        (``metallic_electrodes``).  Returns the number of V-cycles."""
        self._init()
        assert tuple(phi.shape) == tuple(self.gd.n_c)
        assert tuple(rho.shape) == tuple(self.gd.n_c)
        actual_charge = self.gd.integrate(rho)
        background = (actual_charge / self.gd.dv /
                      self.gd.get_size_of_global_array().prod())
        if self.remove_moment:
            return _solve_removing_moments(self, phi, rho)
        if charge is None:
            charge = actual_charge
        if abs(charge) <= maxcharge:
            return self.solve_neutral(phi, rho - background)
        if self.gd.pbc_c.all():
            if zero_initial_phi:
                phi.zero_()
            niter = self.solve_neutral(phi, rho - background)
            if self.use_charged_periodic_corrections:
                if self.charged_periodic_correction is None:
                    from .ewald import madelung
                    self.charged_periodic_correction = madelung(
                        self.gd.cell_cv)
                phi += actual_charge * self.charged_periodic_correction
            return niter
        if not self.gd.pbc_c.any():
            center = None
            if self.use_charge_center:
                from .gauss import charge_center, charge_center_parts
                center = charge_center(self.gd, *charge_center_parts(
                    self.gd, rho, actual_charge))
            return _solve_monopole(self, phi, rho, actual_charge,
                                   zero_initial_phi, center)
        if self.metallic_electrodes == 'single':
            # a dipole layer against the far electrode along axis 2
            # (gpaw/poisson.py:286-301)
            from .dipole import dipole_correction
            origin = [0, 0, int(self.gd.N_c[2])]
            drho, dphi, corr = dipole_correction(2, self.gd, rho,
                                                 origin_c=origin)
            phi -= dphi
            niter = self.solve_neutral(phi, rho + drho)
            phi += dphi
            phi -= corr
            self.correction = 0.0
            return niter
        if self.metallic_electrodes == 'both':
            return self.solve_neutral(phi, rho)
        raise NotImplementedError(
            'Charged systems with mixed periodic/zero boundary conditions')

    def _rhs(self, rho):
        """rho, or B rho for the Mehrstellen stencil (gpaw/poisson.py:
        478-481); the B-applied copy lives in a buffer of the solver."""
        rho = rho.contiguous()
        if self.B is None:
            return rho
        if getattr(self, '_rhoB', None) is None or \
                self._rhoB.device != rho.device:
            self._rhoB = torch.empty_like(rho)
        self.B.apply(rho, self._rhoB)
        return self._rhoB

    def solve_neutral(self, phi, rho, timer=None):
        """gpaw/poisson.py:474-498 in the native executor."""
        self._init()
        rho = self._rhs(rho)
        niter = C.c_int(0)
        err = C.c_double(0.0)
        rc = self._exec.lib.gb_poisson_solve_neutral(
            self._exec.h, C.c_void_p(phi.data_ptr()),
            C.c_void_p(rho.data_ptr()), float(self.eps), int(self.maxiter),
            C.byref(niter), C.byref(err), _stream())
        self.last_error = err.value
        self.niter = niter.value
        check(rc)
        return niter.value

    def solve_neutral_async(self, phi, rho, eps=None):
        """Enqueue solve_neutral on the current stream; read the outcome with
        result() once the stream has reached this point.  ``rho`` must stay
        alive and unchanged until then."""
        self._init()
        rho = self._rhs(rho)
        check(self._exec.lib.gb_poisson_solve_neutral_async(
            self._exec.h, C.c_void_p(phi.data_ptr()),
            C.c_void_p(rho.data_ptr()),
            float(self.eps if eps is None else eps), int(self.maxiter),
            _stream()))

    def result(self):
        """V-cycle count of the last asynchronous solve (raises
        PoissonConvergenceError if it stopped at maxiter)."""
        niter = C.c_int(0)
        err = C.c_double(0.0)
        rc = self._exec.lib.gb_poisson_result(self._exec.h, C.byref(niter),
                                              C.byref(err))
        self.niter = niter.value
        self.last_error = err.value
        check(rc)
        return niter.value

    def iterate2(self, step, level=0, phi=None, rho=None):
        """One V-cycle from level 0 (gpaw/poisson.py:500-537); returns the
        level-0 error sum(r^2) * dv."""
        if level != 0:
            raise NotImplementedError('V-cycles start at level 0')
        self._init()
        err = C.c_double(0.0)
        check(self._exec.lib.gb_poisson_iterate(
            self._exec.h, C.c_void_p(phi.data_ptr()),
            C.c_void_p(rho.data_ptr()), C.byref(err), _stream()))
        return err.value

    def estimate_memory(self, mem=None):
        gdbytes = int(np.prod(self.gd.n_c)) * 8
        nbytes = -gdbytes
        for level in range(self.levels):
            nbytes += 3 * gdbytes
            gdbytes //= 8
        return nbytes

    def __repr__(self):
        return 'FDPoissonSolver(relax=\'%s\', nn=%s, eps=%e)' % (
            self.relax, repr(self.nn), self.eps)


class _Exec:
    def __init__(self, lib, h, owner):
        self.lib = lib
        self.h = h
        # keep level objects alive as long as the executor
        self._keep = (owner.operators, owner.restrictors,
                      owner.interpolators)

    def __del__(self):
        if self.h is not None and self.h.value:
            self.lib.gb_poisson_free(self.h)
            self.h = None


def stencil_spectrum(op, gd):
    """(min over non-constant modes, max) of the eigenvalues of D^-1 A for
    an axis-aligned stencil on ``gd`` (zero boundary: sine modes
    theta = pi j / N, j = 1..N-1; periodic: theta = 2 pi j / N)."""
    c0 = op.coef_p[0]
    f = []
    for a in range(3):
        N = int(gd.N_c[a])
        if gd.pbc_c[a]:
            th = 2 * np.pi * np.arange(N) / N
        else:
            th = np.pi * np.arange(1, N) / N
        fa = np.zeros_like(th)
        for c, o in zip(op.coef_p[1:], op.offset_pc[1:]):
            if o[a] != 0:
                fa += c * np.cos(th * o[a])
        f.append(fa / c0)
    # lam = ((1 + f0[i]) + f1[j]) + f2[k] over all (i, j, k).  Rounded
    # addition is monotone in each operand, so the largest (smallest) value
    # is the one at every axis's largest (smallest) term, and the second
    # smallest is the least of the values with one axis at its second
    # smallest term: O(N) per axis, the same numbers as sorting all N^3.
    def lam(x0, x1, x2):
        return float(1.0 + x0 + x1 + x2)

    srt = [np.sort(fa) for fa in f]
    lmax = lam(*(sa[-1] for sa in srt))
    lo = [sa[0] for sa in srt]
    if not gd.pbc_c.all():
        return lam(*lo), lmax
    second = []
    for a in range(3):
        if len(srt[a]) > 1:
            x = list(lo)
            x[a] = srt[a][1]
            second.append(lam(*x))
    return min(second), lmax


def _stencil_spectrum_dense(op, gd):
    """stencil_spectrum by sorting every eigenvalue (the test's check)."""
    c0 = op.coef_p[0]
    f = []
    for a in range(3):
        N = int(gd.N_c[a])
        if gd.pbc_c[a]:
            th = 2 * np.pi * np.arange(N) / N
        else:
            th = np.pi * np.arange(1, N) / N
        fa = np.zeros_like(th)
        for c, o in zip(op.coef_p[1:], op.offset_pc[1:]):
            if o[a] != 0:
                fa += c * np.cos(th * o[a])
        f.append(fa / c0)
    lam = 1.0 + f[0][:, None, None] + f[1][None, :, None] + f[2][None, None, :]
    flat = np.sort(lam.ravel())
    return float(flat[1] if gd.pbc_c.all() else flat[0]), float(lam.max())


def _solve_removing_moments(ps, phi, rho):
    """``remove_moment = n`` (gpaw/poisson.py:192-208, non-periodic cells):
    the density's multipole moments L = 0 .. n-1 about the cell centre are
    taken out with the generalised Gaussians g_L (moments below 1e-7 are
    left), the rest is solved, and the Gaussians' potentials are added back
    (they also shift the initial guess).  Gaussians, their potentials and
    the harmonics are built once per grid (host float64) and kept on the
    device; the moments are device sums."""
    assert not ps.gd.pbc_c.any()
    n = int(ps.remove_moment)
    cache = getattr(ps, '_moment_gd', None)
    dev = phi.device
    if cache is not ps.gd or len(ps._moment_g) < n:
        from .multipole import Gaussian
        G = Gaussian(ps.gd)
        ps._moment_g = [torch.from_numpy(G.get_gauss(L)).to(dev)
                        for L in range(n)]
        ps._moment_v = [torch.from_numpy(G.get_gauss_pot(L)).to(dev)
                        for L in range(n)]
        ps._moment_y = [torch.from_numpy(G.get_Y(L)).to(dev)
                        for L in range(n)]
        ps._moment_gd = ps.gd
    rho_n = rho.clone()
    cors = []
    for L in range(n):
        q = float((rho_n * ps._moment_y[L]).sum()) * ps.gd.dv
        if abs(q) < 1e-7:
            continue
        rho_n -= q * ps._moment_g[L]
        cors.append(q * ps._moment_v[L])
    for c in cors:
        phi -= c
    niter = ps.solve_neutral(phi, rho_n)
    for c in cors:
        phi += c
    return niter


def _solve_monopole(ps, phi, rho, actual_charge, zero_initial_phi,
                    center=None):
    """Charged system in a non-periodic cell (gpaw/poisson.py:233-283):
    subtract a Gaussian carrying the charge, solve the neutral problem,
    add the Gaussian's potential back.  The Gaussian and its potential are
    computed once per grid, or per ``center`` when the charge centre is
    used (host, float64), and kept on the device."""
    key = None if center is None else tuple(float(x) for x in center)
    if getattr(ps, '_gauss_gd', None) is not ps.gd or \
            getattr(ps, '_gauss_center', None) != key:
        from .gauss import monopole_gaussian
        rg, pg = monopole_gaussian(ps.gd, center=None if key is None
                                   else np.array(key))
        ps.rho_gauss = torch.from_numpy(rg).to(phi.device)
        ps.phi_gauss = torch.from_numpy(pg).to(phi.device)
        ps._gauss_gd = ps.gd
        ps._gauss_center = key
    q = actual_charge / np.sqrt(4 * pi)
    rho_neutral = rho - q * ps.rho_gauss
    if zero_initial_phi:
        phi.zero_()
    else:
        phi -= q * ps.phi_gauss
    niter = ps.solve_neutral(phi, rho_neutral)
    phi += q * ps.phi_gauss
    return niter


class MixedPoissonSolver:
    """FP32 V-cycles inside FP64 defect correction (no counterpart in the
    reference, whose FDPoissonSolver is FP64 throughout).

    Same problem and operators as FDPoissonSolver: level 0 is the nn-order
    Laplacian scaled by -1/(4 pi), coarser levels the 2nd-order one, grids
    coarsened as set_grid_descriptor does (gpaw/poisson.py:366-430).  The
    V-cycle spans ``levels`` grids (fewer when the grid cannot be coarsened
    that often) with degree-2 Chebyshev smoothing (two sweeps before, two
    after); the coarsest grid is solved in FP64: by default exactly, by fast
    diagonalisation in one cooperative kernel over every SM; with
    ``fused_coarse=False`` by a Chebyshev iteration, each level its own
    kernels (the form for solves that run beside others and want low
    latency); with ``fused_coarse='tail'`` the small coarse levels and the
    exact coarsest solve in one single-block kernel (the form for batches:
    fewest launches).  The residual, its norm, |rho| and the stopping test
    ||rho - L phi|| <= tol ||rho|| are FP64, on the device.  On a 192^3 grid
    four levels solve to 1e-10 in 14 V-cycles and 5.2 ms, six in 14 and
    5.4 ms.
    """

    def __init__(self, nn=3, tol=1e-10, maxiter=200, levels=6,
                 coarse_accuracy=0.2, fused_coarse=True):
        if nn == 'M':
            raise NotImplementedError(
                'Mehrstellen stencil: use FDPoissonSolver(nn="M")')
        self.nn = nn
        self.tol = tol
        self.maxiter = maxiter
        self.nlevels = levels
        self.coarse_accuracy = coarse_accuracy
        self.fused_coarse = fused_coarse
        self._h = None

    def set_grid_descriptor(self, gd):
        from .fd_operators import Laplace
        from .transformers import Transformer
        self.gd = gd
        scale = -0.25 / pi
        gds = [gd]
        while len(gds) < self.nlevels:
            try:
                gds.append(gds[-1].coarsen())
            except ValueError:
                break
        if len(gds) < 2:
            raise ValueError('grid %s cannot be coarsened' % gd.N_c)
        self.gds = gds
        self.operators = [Laplace(gds[0], scale, self.nn)] + \
            [Laplace(g, scale, 1) for g in gds[1:]]
        self.restrictors = [Transformer(gds[i], gds[i + 1])
                            for i in range(len(gds) - 1)]
        self.interpolators = [Transformer(gds[i + 1], gds[i])
                              for i in range(len(gds) - 1)]
        bounds = [stencil_spectrum(op, g)
                  for op, g in zip(self.operators, gds)]
        self.lam_max = [b[1] for b in bounds]
        lmin, lmax = bounds[-1]
        kappa = lmax / lmin
        q = (np.sqrt(kappa) - 1) / (np.sqrt(kappa) + 1)
        # a one-point coarsest grid has kappa = 1 (q = 0): the minimum degree
        deg = 4 if q <= 0.0 else np.ceil(np.log(self.coarse_accuracy / 2) /
                                          np.log(q))
        self.coarse_degree = int(np.clip(deg, 4, 256))
        self.lam_min_coarse = 0.98 * lmin
        lib = _lib.load()
        nl = len(gds)
        ops = (C.c_void_p * nl)(*[o.operator._h for o in self.operators])
        rst = (C.c_void_p * (nl - 1))(*[t.transformer._h
                                        for t in self.restrictors])
        itp = (C.c_void_p * (nl - 1))(*[t.transformer._h
                                        for t in self.interpolators])
        lam = (C.c_double * nl)(*self.lam_max)
        h = C.c_void_p()
        check(lib.gb_mixed_new(nl, self.operators[0].operator._h, ops, rst,
                               itp, lam, float(self.lam_min_coarse),
                               int(self.coarse_degree), C.byref(h)))
        self._h = _MixedHandle(lib, h, self)
        mode = 2 if self.fused_coarse == 'tail' else int(bool(self.fused_coarse))
        check(lib.gb_mixed_set_fused_coarse(h, mode))

    def solve(self, phi, rho, charge=None, maxcharge=1e-6,
              zero_initial_phi=False, timer=None):
        """Neutral and charged-periodic branches of gpaw/poisson.py:182-231."""
        actual_charge = self.gd.integrate(rho)
        background = (actual_charge / self.gd.dv /
                      self.gd.get_size_of_global_array().prod())
        if charge is None:
            charge = actual_charge
        if abs(charge) <= maxcharge or self.gd.pbc_c.all():
            if zero_initial_phi:
                phi.zero_()
            return self.solve_neutral(phi, rho - background)
        if not self.gd.pbc_c.any():
            return _solve_monopole(self, phi, rho, actual_charge,
                                   zero_initial_phi)
        raise NotImplementedError(
            'charged system with mixed boundary conditions (dipole '
            'correction / metallic electrodes)')

    def solve_neutral(self, phi, rho, timer=None):
        rho = rho.contiguous()
        niter = C.c_int(0)
        rel = C.c_double(0.0)
        rc = self._h.lib.gb_mixed_solve(
            self._h.h, C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()),
            float(self.tol), int(self.maxiter), C.byref(niter), C.byref(rel),
            _stream())
        self.niter = niter.value
        self.rel_residual = rel.value
        check(rc)
        if self.gd.pbc_c.all():
            phi -= phi.mean()
        return niter.value


def _mixed_async(self, phi, rho):
    """Enqueue solve_neutral on the current stream (no host sync); the
    periodic mean removal is left to the caller."""
    check(self._h.lib.gb_mixed_solve_async(
        self._h.h, C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()),
        float(self.tol), int(self.maxiter), _stream()))


def _mixed_result(self):
    niter = C.c_int(0)
    rel = C.c_double(0.0)
    rc = self._h.lib.gb_mixed_result(self._h.h, C.byref(niter),
                                     C.byref(rel))
    self.niter = niter.value
    self.rel_residual = rel.value
    check(rc)
    return niter.value


def _mixed_prepare(self):
    """Capture the solve now (synchronous; otherwise the first
    solve_neutral_async does it)."""
    check(self._h.lib.gb_mixed_prepare(self._h.h))


MixedPoissonSolver.solve_neutral_async = _mixed_async
MixedPoissonSolver.prepare = _mixed_prepare
MixedPoissonSolver.result = _mixed_result


class _MixedHandle:
    def __init__(self, lib, h, owner):
        self.lib = lib
        self.h = h
        self._keep = (owner.operators, owner.restrictors,
                      owner.interpolators)

    def __del__(self):
        if self.h is not None and self.h.value:
            self.lib.gb_mixed_free(self.h)
            self.h = None
