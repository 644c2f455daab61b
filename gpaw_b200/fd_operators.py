"""Finite-difference operators (drop-in for gpaw/fd_operators.py).

``FDOperator``, ``Laplace`` and ``GUCLaplace`` keep the reference's
signatures (gpaw/fd_operators.py:43-238); arrays are torch CUDA tensors and
the work runs in the sm_100a kernels behind the C ABI.  There is no CPU
path: a non-CUDA tensor raises TypeError.
"""
from __future__ import annotations

import functools

import numpy as np

from . import cgpaw

# Expansion coefficients of the finite-difference Laplacian,
# J. R. Chelikowsky et al., Phys. Rev. B 50, 11355 (1994)
# (table as in gpaw/fd_operators.py:27-34).
laplace = [[0],
           [-2, 1],
           [-5 / 2, 4 / 3, -1 / 12],
           [-49 / 18, 3 / 2, -3 / 20, 1 / 90],
           [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560],
           [-5269 / 1800, 5 / 3, -5 / 21, 5 / 126, -5 / 1008, 1 / 3150],
           [-5369 / 1800, 12 / 7, -15 / 56, 10 / 189, -1 / 112, 2 / 1925,
            -1 / 16632]]


class FDOperator:
    """Stencil operator ``out[g] = sum_p coef_p in[g + offset_p]`` with the
    grid's boundary conditions (gpaw/fd_operators.py:43-147)."""

    def __init__(self, coef_p, offset_pc, gd, dtype=float, description=None,
                 xp=None):
        offset_pc = np.asarray(offset_pc, int)
        # central finite difference: every offset along one axis
        cfd = True
        for offset_c in offset_pc:
            if sum(int(o != 0) for o in offset_c) >= 2:
                cfd = False
        mp = int(np.abs(offset_pc).max())
        assert (mp <= gd.n_c).all(), 'Stencil longer than domain'
        n_c = gd.n_c
        M_c = n_c + 2 * mp
        stride_c = np.array([M_c[1] * M_c[2], M_c[2], 1])
        offset_p = np.ascontiguousarray(np.dot(offset_pc, stride_c))
        coef_p = np.ascontiguousarray(coef_p, float)
        assert coef_p.ndim == 1
        assert coef_p.shape == offset_p.shape
        assert dtype in [float, complex]
        self.dtype = dtype
        self.shape = tuple(int(x) for x in n_c)
        self.mp = mp
        self.gd = gd
        self.npoints = len(coef_p)
        self.coef_p = coef_p
        self.offset_p = offset_p
        self.offset_pc = offset_pc
        self.cfd = cfd
        self.xp = xp
        self.operator = cgpaw.Operator(coef_p, offset_p, n_c, mp,
                                       gd.neighbor_cd, dtype == float, None,
                                       cfd)
        if description is None:
            description = '%d point finite-difference stencil' % self.npoints
        self.description = description

    def __str__(self):
        return '<' + self.description + '>'

    def __call__(self, in_xR, out_xR=None, phase_cd=None):
        """Tensor interface: returns ``out_xR`` (allocated if None)."""
        if out_xR is None:
            out_xR = in_xR.new_empty(in_xR.shape)
        self.apply(in_xR, out_xR, phase_cd)
        return out_xR

    def apply(self, in_xg, out_xg, phase_cd=None):
        """gpaw/fd_operators.py:120-130; ``in_xg is out_xg`` is allowed."""
        self.operator.apply(in_xg, out_xg, phase_cd)

    def apply_potential(self, in_xg, out_xg, v_g, phase_cd=None):
        """out = L in + in * v (v real, one grid for the whole batch) in
        one pass: FDHamiltonian.apply_local_potential's ``self.kin(psit,
        out)`` then ``o += p * vt`` (gpaw/new/fd/hamiltonian.py:23-32),
        bit for bit."""
        self.operator.apply_potential(in_xg, out_xg, v_g, phase_cd)

    def relax(self, relax_method, f_g, s_g, n, w=None):
        """gpaw/fd_operators.py:132-141: 1 = Gauss-Seidel, 2 = weighted
        Jacobi (float64 only)."""
        self.operator.relax(relax_method, f_g, s_g, n,
                            1.0 if w is None else w)

    def residual(self, phi, rho, r=None, phase_cd=None, scale=None,
                 norm2=None):
        """r = L(phi) - rho in one pass (+ optional scaled |r|^2 per grid)."""
        self.operator.residual(phi, rho, r, phase_cd, scale, norm2)

    def get_diagonal_element(self):
        return self.operator.get_diagonal_element()

    def set_chunk(self, chunk):
        """Axis-0 planes per CTA (z-block depth) of the plane-marching
        kernels; 0 = automatic.  See gpaw_b200.autotune."""
        self.operator.set_chunk(chunk)

    def get_async_sizes(self):
        return self.operator.get_async_sizes()


def laplace_stencil(gd, scale=1.0, n=1):
    """Coefficients and offsets of the general-cell Laplacian
    (gpaw/fd_operators.py:184-238): pick the 3..6 shortest lattice
    directions whose second differences reproduce x^2, y^2, z^2 and no
    cross terms (least squares), then lay Chelikowsky's 1-D coefficients
    along each.  They depend on the grid spacing only, so they are cached
    per (spacing vectors, scale, n): a solver hierarchy, or a serving loop
    building solvers for many grid shapes of one spacing, computes them
    once."""
    coefs, offsets = _laplace_stencil(np.asarray(gd.h_cv, float).tobytes(),
                                      float(scale), int(n))
    return list(coefs), [np.array(o) for o in offsets]


@functools.lru_cache(maxsize=256)
def _laplace_stencil(h_bytes, scale, n):
    h_cv = np.frombuffer(h_bytes).reshape(3, 3)
    M_ic = np.indices((3, 3, 3)).reshape((3, -3)).T[-13:] - 1
    u_cv = h_cv / (h_cv**2).sum(1)[:, np.newaxis]**0.5
    u2_i = (np.dot(M_ic, u_cv)**2).sum(1)
    i_d = u2_i.argsort()
    m_mv = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2),
                     (0, 1, 1), (1, 0, 1), (1, 1, 0)])
    for D in range(3, 7):
        h_dv = np.dot(M_ic[i_d[:D]], h_cv)
        A_md = (h_dv**m_mv[:, np.newaxis, :]).prod(2)
        a_d, residual, rank, s = np.linalg.lstsq(A_md, [1, 1, 1, 0, 0, 0],
                                                 rcond=-1)
        if residual.sum() < 1e-14:
            if rank != D:
                raise ValueError(
                    'You have a weird unit cell!  '
                    'Try to use the maximally reduced Niggli cell.')
            break
    a_d *= scale
    offsets = [(0, 0, 0)]
    coefs = [laplace[n][0] * a_d.sum()]
    for d in range(D):
        M_c = M_ic[i_d[d]]
        offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(laplace[n][1:]))
        offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(laplace[n][1:]))
    return tuple(coefs), tuple(tuple(int(x) for x in o) for o in offsets)


class GUCLaplace(FDOperator):
    """Laplacian for a general (also non-orthorhombic) cell,
    O(h^(2n)) error; scale=-0.5 gives the kinetic-energy operator."""

    def __init__(self, gd, scale=1.0, n=1, dtype=float, xp=None):
        if not 1 <= n <= 6:
            raise ValueError('stencil range n must be 1..6')
        coefs, offsets = laplace_stencil(gd, scale, n)
        super().__init__(coefs, offsets, gd, dtype, xp=xp)
        self.description = (
            '%d*%d+1=%d point O(h^%d) finite-difference Laplacian' %
            ((self.npoints - 1) // n, n, self.npoints, 2 * n))


def Laplace(gd, scale=1.0, n=1, dtype=float, xp=None):
    """gpaw/fd_operators.py:177-181: n = 9 selects the spectral Laplacian
    of a periodic cell, 1..6 the finite-difference stencils."""
    if n == 9:
        return FTLaplace(gd, scale, dtype)
    return GUCLaplace(gd, scale, n, dtype, xp=xp)


class FTLaplace:
    """Spectral Laplacian of a fully periodic cell (gpaw/fd_operators.py:
    399-424): the input's discrete Fourier transform is multiplied by
    -scale |k|^2, with k = 2 pi B^T i for the integer frequencies i folded
    into [-N/2, N/2), and transformed back; the real part is kept (for
    complex input too, as the reference does, and Bloch phases are
    ignored).  The transforms are cuFFT's (through torch.fft); the factor
    table lives on the device.  For real input the half-spectrum transform
    is used with the table averaged over i and -i (folded): the real part
    of the full transform equals exactly that, because the spectrum of real
    data is Hermitian.  (The table itself is not symmetric on the Nyquist
    planes of a non-orthogonal cell.)"""

    def __init__(self, gd, scale, dtype=float):
        import torch
        assert gd.pbc_c.all(), 'the spectral Laplacian needs a periodic cell'
        N = np.asarray(gd.N_c)
        i_cq = np.indices(tuple(N)).reshape((3, -1))
        i_cq = (i_cq + N[:, None] // 2) % N[:, None] - N[:, None] // 2
        k_vq = np.dot(2.0 * np.pi * gd.icell_cv.T, i_cq)
        k2 = (k_vq * k_vq).sum(axis=0).reshape(tuple(N)) * (-scale)
        self.gd = gd
        self.dtype = dtype
        self.shape = tuple(int(n) for n in N)
        self.k2_Q = torch.from_numpy(k2).to(gd.device)
        k2_neg = np.roll(np.flip(k2), 1, axis=(0, 1, 2))   # k2 at -i
        half = self.shape[2] // 2 + 1
        self.k2_half = torch.from_numpy(
            np.ascontiguousarray(0.5 * (k2 + k2_neg)[:, :, :half])).to(
                gd.device)
        self.d = 6.0 / gd.h_cv[0, 0]**2
        self.npoints = 1000
        self.description = 'FFT Laplacian'

    def apply(self, in_xg, out_xg, phase_cd=None):
        import torch
        if not (in_xg.is_cuda and out_xg.is_cuda):
            raise TypeError('FTLaplace works on CUDA tensors')
        assert tuple(in_xg.shape[-3:]) == self.shape
        dims = (-3, -2, -1)
        if in_xg.is_complex():
            out = torch.fft.ifftn(torch.fft.fftn(in_xg, dim=dims) *
                                  self.k2_Q, dim=dims).real
        else:
            out = torch.fft.irfftn(torch.fft.rfftn(in_xg, dim=dims) *
                                   self.k2_half, s=self.shape, dim=dims)
        out_xg.copy_(out)

    def get_diagonal_element(self):
        return self.d

    def get_description(self):
        return self.description


class LaplaceA(FDOperator):
    """O(h^4) Mehrstellen Laplacian, left-hand side (gpaw/fd_operators.py:
    357-384): 19 points (centre, 6 faces, 12 edges); orthorhombic cells."""

    def __init__(self, gd, scale, dtype=float, xp=None):
        assert gd.orthogonal
        c = np.divide(-1 / 12, gd.h_cv.diagonal()**2) * scale
        c0 = c[1] + c[2]
        c1 = c[0] + c[2]
        c2 = c[1] + c[0]
        a = -16.0 * np.sum(c)
        b = 10.0 * c + 0.125 * a
        super().__init__([a, b[0], b[0], b[1], b[1], b[2], b[2],
                          c0, c0, c0, c0, c1, c1, c1, c1, c2, c2, c2, c2],
                         [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0),
                          (0, 1, 0), (0, 0, -1), (0, 0, 1),
                          (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
                          (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1),
                          (-1, -1, 0), (-1, 1, 0), (1, -1, 0), (1, 1, 0)],
                         gd, dtype, 'O(h^4) Mehrstellen Laplacian (A)', xp)


class LaplaceB(FDOperator):
    """Mehrstellen right-hand side B = 1/2 + 1/12 (6 faces)
    (gpaw/fd_operators.py:387-396)."""

    def __init__(self, gd, dtype=float, xp=None):
        a = 0.5
        b = 1.0 / 12.0
        super().__init__([a, b, b, b, b, b, b],
                         [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0),
                          (0, 1, 0), (0, 0, -1), (0, 0, 1)],
                         gd, dtype, 'O(h^4) Mehrstellen Laplacian (B)', xp)


# Central-difference first-derivative coefficients, orders 2..8
# (gpaw/fd_operators.py:36-39).
derivatives = [[1 / 2],
               [2 / 3, -1 / 12],
               [3 / 4, -3 / 20, 1 / 60],
               [4 / 5, -1 / 5, 4 / 105, -1 / 280]]


def find_neighbors_orthogonal(h_cv):
    """Neighbour directions of an orthorhombic grid sorted by distance, as
    gpaw/fd_operators.py:240-282 finds them (Voronoi ridges of the centre
    of the 27-point block; an orthogonal basis is already Minkowski
    reduced, so no reduction step)."""
    from scipy.spatial import Voronoi
    M_ib = np.indices((3, 3, 3)).reshape((3, -1)).T - 1
    h_iv = M_ib.dot(h_cv)
    voro = Voronoi(h_iv)
    i_d = []
    for i1, i2 in voro.ridge_points:
        if i1 == 13 and i2 > 13:
            i_d.append(i2)
        elif i2 == 13 and i1 > 13:
            i_d.append(i1)
    h2_d = (h_iv[i_d]**2).sum(1)
    return M_ib[[i_d[d] for d in h2_d.argsort()]]


def minkowski_basis(h_cv):
    """A Minkowski-reduced basis of the lattice spanned by the rows of h_cv
    and the integer matrix U_bc with h_bv = U_bc @ h_cv.  In three
    dimensions the successive minima form a reduced basis: the shortest
    lattice vector, the shortest one independent of it, and the shortest
    one independent of both.  Candidates are the combinations with
    coefficients in -3..3 of the rows of h_cv after a pairwise size
    reduction (enough for grid spacings of any cell a DFT code meets); on
    ties the positive combination wins, so an already reduced basis is
    kept as it is.
    Serves the role of ASE's reduction_full in gpaw/fd_operators.py:264;
    the basis may differ from ASE's by order and signs, which changes
    neither the set of neighbour directions nor the stencil, only the order
    of its terms."""
    h = np.array(h_cv, float)
    U = np.eye(3, dtype=int)
    # size reduction until no pairwise step shortens a vector
    for _ in range(100):
        changed = False
        for i in range(3):
            for j in range(3):
                if i == j:
                    continue
                k = int(np.rint(h[i] @ h[j] / (h[j] @ h[j])))
                if k and np.linalg.norm(h[i] - k * h[j]) < \
                        np.linalg.norm(h[i]) - 1e-12:
                    h[i] -= k * h[j]
                    U[i] -= k * U[j]
                    changed = True
        if not changed:
            break
    M = np.array(np.meshgrid(*[np.arange(-3, 4)] * 3,
                             indexing='ij')).reshape(3, -1).T
    M = M[np.abs(M).sum(1) > 0]
    vecs = M @ h
    # shortest first; among equal lengths the combination with the larger
    # coefficients (so +v before -v, and the size-reduced rows themselves)
    order = np.lexsort((-M[:, 2], -M[:, 1], -M[:, 0],
                        np.round((vecs**2).sum(1), 12)))
    basis = []
    for i in order:
        cand = basis + [i]
        if np.linalg.matrix_rank(M[cand], tol=0.5) == len(cand):
            basis = cand
            if len(basis) == 3:
                break
    U_bc = M[basis] @ U
    return U_bc @ np.asarray(h_cv, float), U_bc


def find_neighbors(h_cv):
    """Neighbour directions of a general grid sorted by distance
    (gpaw/fd_operators.py:241-282): Voronoi ridges of the centre of the
    27-point block of a reduced basis, mapped back to the grid's axes."""
    if np.allclose(h_cv, np.diag(np.diag(h_cv)), rtol=0, atol=1e-12):
        return find_neighbors_orthogonal(h_cv)
    h_bv, U_bc = minkowski_basis(h_cv)
    return find_neighbors_orthogonal(h_bv) @ U_bc


class Gradient(FDOperator):
    """Symmetric finite-difference derivative along x, y or z
    (gpaw/fd_operators.py:285-354), O(h^(2n)) error, for any cell: the
    neighbour directions come from a reduced basis of the grid (see
    minkowski_basis)."""

    def __init__(self, gd, v, scale=1.0, n=1, dtype=float, xp=None):
        M_dc = find_neighbors(gd.h_cv)
        h_dv = M_dc @ gd.h_cv
        D = len(h_dv)
        invh_vc = np.linalg.inv(gd.h_cv)
        n_cv = (invh_vc / (invh_vc**2).sum(axis=0)**0.5).T
        coef_cd = np.zeros((3, D))
        for c, n_v in enumerate(n_cv):
            ok_d = abs(h_dv.dot(n_v)) > 1e-10
            h_mv = h_dv[ok_d]
            A_jm = np.array([h_mv.dot(n_v),
                             h_mv.dot(gd.h_cv[c - 1]),
                             h_mv.dot(gd.h_cv[c - 2])])
            U_jm, S_m, V_mm = np.linalg.svd(A_jm, full_matrices=False)
            coef_m = V_mm.T.dot(np.diag(S_m**-1).dot(U_jm.T.dot([1, 0, 0])))
            coef_cd[c, ok_d] = coef_m
        coef_d = np.linalg.inv(n_cv)[v].dot(coef_cd) * scale
        offsets = []
        coefs = []
        stencil = np.array(derivatives[n - 1])
        for d, c in enumerate(coef_d):
            if abs(c) < 1e-10:
                continue
            M_c = M_dc[d]
            offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
            coefs.extend(c * stencil)
            offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
            coefs.extend(-c * stencil)
        super().__init__(coefs, offsets, gd, dtype, xp=xp)
        self.description = (
            'Finite-difference {}-derivative with O(h^{}) error ({} points)'
            .format('xyz'[v], 2 * n, self.npoints))
