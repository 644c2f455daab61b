"""Host-side logic of gpaw_b200 against the oracle's restatement of the
reference's Python layer: stencil coefficients, grid conventions,
transformer geometry, multigrid schedule.  No GPU needed."""
import numpy as np
import pytest

from oracle import gpaw_layer as L
from oracle import port

CELLS = {
    'sc': (1.1, 1.02, 1.03),
    'hexagonal': [(1, 0, 0), (0.5, 3**0.5 / 2, 0), (0, 0, 1.1)],
    'fcc': [(0, 1, 1), (1, 0, 1), (1, 1, 0)],
    'bcc': [(-1, 1, 1), (1, -1, 1), (1, 1, -1)],
    'distorted sc': [(1, 0, 0), (0.01, 1, 0), (0, 0.02, 1)],
}


@pytest.mark.parametrize('cell', sorted(CELLS))
@pytest.mark.parametrize('n', range(1, 7))
def test_laplace_coefficients_match(cell, n):
    from gpaw_b200.fd_operators import laplace_stencil
    from gpaw_b200.grid_descriptor import GridDescriptor
    N = (2 * n + 2,) * 3
    c1, o1 = laplace_stencil(GridDescriptor(N, CELLS[cell], device='cpu'),
                             -0.5, n)
    c2, o2 = L.laplace_stencil(L.GridDescriptor(N, CELLS[cell]), -0.5, n)
    assert np.array_equal(np.array(c1), np.array(c2))
    assert np.array_equal(np.array(o1), np.array(o2))


@pytest.mark.parametrize('cell,D', [('sc', 3), ('hexagonal', 4), ('fcc', 6),
                                    ('bcc', 4), ('distorted sc', 6)])
@pytest.mark.parametrize('n', range(1, 5))
def test_laplace_exact_on_polynomials(cell, D, n):
    """Known-answer test of gpaw/test/fd_ops/test_laplace.py:15-103: the
    stencil is exact on polynomials of degree <= 2n at the central point;
    the product's coefficients are applied by the oracle."""
    from gpaw_b200.fd_operators import laplace_stencil
    from gpaw_b200.grid_descriptor import GridDescriptor
    N = 2 * n + 2
    gdp = GridDescriptor((N, N, N), CELLS[cell], device='cpu')
    coefs, offsets = laplace_stencil(gdp, 1.0, n)
    assert len(coefs) == D * 2 * n + 1
    gd = L.GridDescriptor((N, N, N), CELLS[cell])
    op = L.FDOperator(coefs, offsets, gd, be='port')
    r_gv = gd.get_grid_point_coordinates().transpose((1, 2, 3, 0))
    r_gv = r_gv - gd.cell_cv.sum(0) / 2
    b = gd.zeros()
    for m in range(0, 2 * n + 1):
        for ix in range(m + 1):
            for iy in range(m - ix + 1):
                iz = m - ix - iy
                a = (r_gv**(ix, iy, iz)).prod(3)
                r = 2.0 if (m == 2 and max(ix, iy, iz) == 2) else 0.0
                op.apply(a, b)
                assert abs(b[n + 1, n + 1, n + 1] - r) < 2e-12


@pytest.mark.parametrize('N,pbc', [((64, 64, 64), 0), ((96, 96, 96), 1),
                                   ((40, 32, 128), 0), ((2, 4, 6), 1),
                                   ((2, 2, 2), 0)])
def test_grid_conventions(N, pbc):
    from gpaw_b200.grid_descriptor import GridDescriptor
    g1 = GridDescriptor(N, (5.0, 6.0, 7.0), pbc, device='cpu')
    g2 = L.GridDescriptor(N, (5.0, 6.0, 7.0), pbc)
    for attr in ('N_c', 'n_c', 'beg_c', 'end_c', 'neighbor_cd'):
        assert np.array_equal(getattr(g1, attr), getattr(g2, attr)), attr
    assert g1.dv == g2.dv
    assert np.array_equal(g1.get_size_of_global_array(), g2.n_c)
    # coarsening stops where the reference stops (gpaw/poisson.py:393-397)
    levels = [0, 0]
    for i, g in enumerate((g1, g2)):
        while True:
            try:
                g = g.coarsen()
            except ValueError:
                break
            levels[i] += 1
    assert levels[0] == levels[1]


def test_poisson_hierarchy_64_zero():
    """64^3 zero BC: 6 grids, coarsest N = 2 (one unknown per axis)."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    g = GridDescriptor((64, 64, 64), 1.0, 0, device='cpu')
    sizes = [int(g.n_c[0])]
    while True:
        try:
            g = g.coarsen()
        except ValueError:
            break
        sizes.append(int(g.n_c[0]))
    assert sizes == [63, 31, 15, 7, 3, 1]


@pytest.mark.parametrize('nn', [1, 2, 3, 4])
@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
def test_transformer_geometry(nn, pbc):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.transformers import transformer_geometry
    N = (32, 28, 24)
    a1, a2 = (GridDescriptor(N, 3.0, pbc, device='cpu'),
              L.GridDescriptor(N, 3.0, pbc))
    for fwd in (True, False):
        g1 = (a1, a1.coarsen()) if fwd else (a1.coarsen(), a1)
        g2 = (a2, a2.coarsen()) if fwd else (a2.coarsen(), a2)
        r1 = transformer_geometry(*g1, nn)
        r2 = L.transformer_geometry(*g2, nn)
        for x, y in zip(r1, r2):
            assert np.array_equal(np.asarray(x), np.asarray(y))


def test_interpolator_guard():
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.transformers import transformer_geometry
    gd = GridDescriptor((4, 4, 4), 1.0, 0, device='cpu')
    with pytest.raises(ValueError, match='Cannot construct interpolator'):
        transformer_geometry(gd.coarsen(), gd, 3)


def test_lagrange_weights_are_the_reference_constants():
    # c/bmgs/restrict.cpp:37-57 and c/bmgs/interpolate.cpp:29-40
    assert port.lagrange_midpoint_weights(2) == [0.5]
    assert port.lagrange_midpoint_weights(4) == [0.5625, -0.0625]
    assert port.lagrange_midpoint_weights(6) == [0.58593750, -0.09765625,
                                                 0.01171875]
    assert port.lagrange_midpoint_weights(8) == [
        0.59814453125, -0.11962890625, 0.02392578125, -0.00244140625]


def test_cgpaw_objects_build_without_gpu():
    """Operator / Transformer construction is host-only (no CUDA call)."""
    from gpaw_b200 import cgpaw
    from gpaw_b200.fd_operators import laplace_stencil
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((16, 16, 16), 3.0, 1, device='cpu')
    coefs, offs = laplace_stencil(gd, -0.5, 3)
    M = gd.n_c + 6
    offp = np.dot(np.array(offs), [M[1] * M[2], M[2], 1])
    op = cgpaw.Operator(coefs, offp, gd.n_c, 3, gd.neighbor_cd, 1, None, 1)
    assert op.get_diagonal_element() == coefs[0]
    with pytest.raises(ValueError):
        cgpaw.Operator(coefs, offp * 1000, gd.n_c, 3, gd.neighbor_cd, 1,
                       None, 1)
    with pytest.raises(NotImplementedError):
        cgpaw.Operator(coefs, offp, gd.n_c, 3, gd.neighbor_cd, 1, object(),
                       1)


def test_dipole_moment_matches_oracle():
    """The dipole moment of the product's wrapper (numpy path) agrees with
    the restatement of the reference's grid method."""
    import numpy as np
    from gpaw_b200 import GridDescriptor
    from gpaw_b200.dipole import calculate_dipole_moment
    from oracle import gpaw_layer as L
    rng = np.random.default_rng(5)
    for pbc in ((0, 0, 0), (1, 1, 0)):
        gd = GridDescriptor((12, 10, 14), (3.0, 2.5, 3.5), pbc, device='cpu')
        go = L.GridDescriptor((12, 10, 14), (3.0, 2.5, 3.5), pbc)
        rho = rng.standard_normal(tuple(go.n_c))
        got = calculate_dipole_moment(gd, rho)
        want = L.calculate_dipole_moment(go, rho)
        # the projections are summed in another order than the oracle's
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_oracle_interpolate_density_conserves_charge():
    """The oracle's _interpolate_density restatement keeps each spin's
    integral on a zero-boundary grid (gpaw/new/fd/pot_calc.py:72-80)."""
    import numpy as np
    from oracle import gpaw_layer as L
    gd = L.GridDescriptor((12, 10, 14), (3.0, 2.5, 3.5), (0, 0, 0))
    fg = gd.refine()
    nt = np.random.default_rng(0).uniform(0.0, 1.0, (2,) + tuple(gd.n_c))
    f = L.interpolate_density(gd, fg, nt, 3)
    assert f.shape == (2,) + tuple(fg.n_c)
    assert np.allclose(gd.integrate(nt), fg.integrate(f), rtol=1e-13, atol=0)


def test_gaussian_multipoles_unit_moments_and_far_field():
    """The multipole Gaussians of the moment corrections (product host code
    and the oracle's restatement): int g_L Y_L' dV = delta_LL' for
    L, L' = 0..8 on a fine grid, the potentials tend to the point multipole
    4 pi / (2l+1) Y_L / r^(2l+1) far out, and both restatements agree."""
    import numpy as np
    from oracle import gpaw_layer as L
    from gpaw_b200 import multipole as M
    gd = L.GridDescriptor((64, 64, 64), (12.0, 12.0, 12.0), (0, 0, 0))
    g = L.GaussianMP(gd, a=19.0)
    x, y, z = g.xyz
    for La in range(9):
        gl = g.get_gauss(La)
        for Lb in range(9):
            m = gd.integrate(gl * L.mp_Y(Lb, x, y, z, g.r2))
            assert abs(m - (La == Lb)) < 1e-6, (La, Lb, m)
        far = g.r > 8.0      # erfc(sqrt(a) r) < 1e-14 there
        lv = L._MP_L[La]
        point = 4 * np.pi / (2 * lv + 1) * L.mp_Y(La, x, y, z, g.r2) / \
            g.r**(2 * lv + 1)
        v = g.get_gauss_pot(La)
        assert np.allclose(v[far], point[far], rtol=1e-9, atol=1e-14)
        mine = M.gausspot_L(g.a, La, x, y, z, g.r, g.r2, g.erf_sar, g.exp_ar2)
        assert np.allclose(mine, v, rtol=1e-13, atol=0)
        mineg = M.gauss_L(g.a, La, x, y, z, g.r2, g.exp_ar2)
        assert np.allclose(mineg, gl, rtol=1e-13, atol=1e-300)


def test_gaussians_reference_known_answers():
    """The reference's own checks of its Gaussians
    (gpaw/test/test_gauss_func.py:19-54: a 48^3 zero-boundary grid in a
    20 Bohr cell), on the product's host Gaussians: the moments of g_L for
    L = 2..8 are delta_LL' to 1e-4, those of the hydrogen density
    exp(-2 r) / pi are delta_L0 / sqrt(4 pi) to 1.5e-3 for L < 4, and
    subtracting its monopole with g_0 leaves a zero moment below 1e-7;
    the oracle's Gaussians meet the moment checks too."""
    import numpy as np
    from gpaw_b200 import GridDescriptor
    from gpaw_b200 import multipole as M
    gd = GridDescriptor((48, 48, 48), (20.0, 20.0, 20.0), False,
                        device='cpu')
    g = M.Gaussian(gd)

    def moment(f, L):
        return float((f * g.get_Y(L)).sum() * gd.dv)
    for gL in range(2, 9):
        gl = g.get_gauss(gL)
        for mL in range(9):
            assert abs(moment(gl, mL) - (gL == mL)) < 1e-4, (gL, mL)
    nH = np.exp(-2 * g.r) / np.pi
    for L in range(4):
        assert abs(moment(nH, L) - (L == 0) / np.sqrt(4 * np.pi)) < 1.5e-3
    nH = nH - moment(nH, 0) * g.get_gauss(0)
    assert abs(moment(nH, 0)) < 1e-7
    # the oracle's restatement meets the same known answers
    from oracle import gpaw_layer as L
    go = L.GaussianMP(L.GridDescriptor((48, 48, 48), (20.0, 20.0, 20.0),
                                       (0, 0, 0)))
    x, y, z = go.xyz
    for gL in range(2, 9):
        gl = go.get_gauss(gL)
        for mL in range(9):
            m = float((gl * L.mp_Y(mL, x, y, z, go.r2)).sum() * gd.dv)
            assert abs(m - (gL == mL)) < 1e-4, (gL, mL)


def _port_apply(op, N, cell, pbc, a):
    """The product operator's stencil applied by the oracle's restatement
    of the reference's C apply, on the host."""
    import numpy as np
    from oracle import gpaw_layer as L
    gdo = L.GridDescriptor(N, cell, pbc)
    o = L.FDOperator(op.coef_p, op.offset_pc, gdo, float, be='port')
    out = np.zeros_like(a)
    o.apply(a, out)
    return out


def test_gradient_reference_known_answers():
    """The reference's gradient checks (gpaw/test/fd_ops/test_gradient.py:
    29-92), the product's stencils applied by the oracle: d/dx of
    0..7 on a periodic 8-point line is [-3, 1, ..., 1, -3], the backward
    difference [-1, 1] gives [-7, 1, ..., 1]; d/dy on a zero-boundary
    7-point line starts at 0.5 and sums to 3; on a GUC cell it starts at
    -3.5 and sums to 0 (1e-12)."""
    import numpy as np
    from gpaw_b200 import FDOperator, GridDescriptor, Gradient
    gd = GridDescriptor((8, 1, 1), (8.0, 1.0, 1.0), True)
    a = np.zeros((8, 1, 1))
    a[:, 0, 0] = np.arange(8)
    d = _port_apply(Gradient(gd, 0), (8, 1, 1), (8.0, 1.0, 1.0), True, a)
    assert d[:, 0, 0].tolist() == [-3, 1, 1, 1, 1, 1, 1, -3]
    back = FDOperator([-1, 1], [[-1, 0, 0], [0, 0, 0]], gd)
    d = _port_apply(back, (8, 1, 1), (8.0, 1.0, 1.0), True, a)
    assert d[:, 0, 0].tolist() == [-7, 1, 1, 1, 1, 1, 1, 1]
    gd = GridDescriptor((1, 8, 1), (1.0, 8.0, 1.0), (1, 0, 1))
    a = np.zeros((1, 7, 1))
    a[0, :, 0] = np.arange(1, 8) - 1
    d = _port_apply(Gradient(gd, 1), (1, 8, 1), (1.0, 8.0, 1.0), (1, 0, 1),
                    a)
    assert d[0, 0, 0] == 0.5 and np.sum(d[0, :, 0]) == 3.0
    cell = ((1.0, 0.0, 0.0), (5.0, 5.0, 0.0), (0.0, 0.0, 0.7))
    gd = GridDescriptor((1, 7, 1), cell, True)
    a = np.zeros((1, 7, 1))
    a[0, :, 0] = np.arange(0, 7) - 1
    d = _port_apply(Gradient(gd, 1), (1, 7, 1), cell, True, a)
    assert abs(d[0, 0, 0] + 3.5) < 1e-12 and abs(np.sum(d[0, :, 0])) < 1e-12


def _cellpar_to_cell(a, b, c, alpha, beta, gamma):
    """Cell vectors from lengths and angles (degrees): a along x, b in the
    xy plane, c from the remaining two angles; right angles give exact
    zeros."""
    import numpy as np

    def cs(t):
        if t == 90:
            return 0.0, 1.0
        r = np.radians(t)
        return np.cos(r), np.sin(r)
    ca, _ = cs(alpha)
    cb, _ = cs(beta)
    cg, sg = cs(gamma)
    cy = (ca - cb * cg) / sg
    return np.array([[a, 0, 0], [b * cg, b * sg, 0],
                     [c * cb, c * cy, c * np.sqrt(1 - cb**2 - cy**2)]])


def test_gradient_strange_cells_reference_known_answer():
    """gpaw/test/fd_ops/test_gradient.py:10-25: on two strongly skewed
    periodic cells the x-derivative of x at the middle of the grid is 1
    (relative 1e-6) -- the product's general-cell stencil applied by the
    oracle."""
    import numpy as np
    from gpaw_b200 import GridDescriptor, Gradient
    for cellpar, size in (((8.7, 5.7, 7.7, 28, 120, 95), (60, 40, 54)),
                          ((2, 2, 2, 120.1, 120.1, 90), (20, 20, 20))):
        cell = _cellpar_to_cell(*cellpar)
        gd = GridDescriptor(size, cell, True)
        s = np.indices(size, float).reshape(3, -1).T / np.array(size)
        x = (s @ cell)[:, 0].reshape(size)
        d = _port_apply(Gradient(gd, 0), size, cell, True, x)
        n1, n2, n3 = (k // 2 for k in size)
        assert abs(d[n1, n2, n3] - 1.0) < 1e-6, cellpar


def test_transfers_conserve_integrals_reference_known_answer():
    """gpaw/test/fd_ops/test_non_periodic.py:6-26 on the oracle's
    transformers (nn = 1, zero boundary, 20^3 -> 40^3 and back, the
    fine grid's outer planes zeroed before restricting): the integral is
    kept to 1e-10 both ways."""
    import numpy as np
    from oracle import gpaw_layer as L
    gd1 = L.GridDescriptor((20, 20, 20), (8.0, 8.0, 8.0), 0)
    a1 = np.random.default_rng(8).random(tuple(gd1.n_c))
    gd2 = gd1.refine()
    a2 = np.zeros(tuple(gd2.n_c))
    L.Transformer(gd1, gd2, be='port').apply(a1, a2)
    assert abs(gd1.integrate(a1) - gd2.integrate(a2)) < 1e-10
    for sl in (np.s_[0], np.s_[:, 0], np.s_[:, :, 0], np.s_[-1],
               np.s_[:, -1], np.s_[:, :, -1]):
        a2[sl] = 0.0
    L.Transformer(gd2, gd1, be='port').apply(a2, a1)
    assert abs(gd1.integrate(a1) - gd2.integrate(a2)) < 1e-10


def test_find_neighbors_reference_examples():
    """The examples of find_neighbors' docstring in the reference
    (gpaw/fd_operators.py:241-260), with the reduction of minkowski_basis
    standing in for ASE's."""
    import numpy as np
    from gpaw_b200.fd_operators import find_neighbors
    assert find_neighbors([[0.1, 0, 0], [0, 0.11, 0],
                           [0, 0, 0.12]]).tolist() == \
        [[1, 0, 0], [0, 1, 0], [0, 0, 1]]
    assert find_neighbors(np.array([[0.1, 0, 0], [0.2, 0.11, 0],
                                    [0, 0, 0.12]])).tolist() == \
        [[1, 0, 0], [-2, 1, 0], [0, 0, 1]]


def test_gradient_stencil_general_cells():
    """Gradient on hexagonal and triclinic cells (gpaw/fd_operators.py:
    285-354): sum_p c_p (o_p h) = scale e_v, so linear functions are
    differentiated exactly, for every range and direction."""
    import numpy as np
    from gpaw_b200 import GridDescriptor, Gradient
    cells = [[(3.0, 0, 0), (1.5, 3.0 * 3**0.5 / 2, 0), (0, 0, 3.2)],
             [(3.0, 0, 0), (0.6, 2.8, 0), (0.4, 0.5, 3.1)]]
    for cell in cells:
        gd = GridDescriptor((12, 12, 12), cell, True)
        for n in (1, 2, 3):
            for v in range(3):
                g = Gradient(gd, v, 0.7, n)
                first = (g.coef_p[:, None] * (g.offset_pc @ gd.h_cv)).sum(0)
                e = np.zeros(3)
                e[v] = 0.7
                assert np.allclose(first, e, rtol=0, atol=1e-12), (cell, n, v)


class _NoSolver:
    """A stand-in wrapped solver: description and dict only."""

    def get_description(self):
        return 'No interaction'

    def todict(self):
        return {'name': 'nointeraction'}


_MC_CASES = [
    (None, 0, None, 'no corrections'),
    ([], 0, None, 'no corrections'),
    (4, 1, ['1 moment corrections', 'center', 'range(0, 4)'],
     'array([0, 1, 2, 3]) @ None'),
    (9, 1, ['1 moment corrections', 'center', 'range(0, 9)'],
     'array([0, 1, 2, 3, 4, 5, 6, 7, 8]) @ None'),
    ([dict(moms=range(4), center=[1., 1., 1.])], 1,
     ['1 moment corrections', '[1.00, 1.00, 1.00]', 'range(0, 4)'],
     'array([0, 1, 2, 3]) @ array([1., 1., 1.])'),
    ([dict(moms=[1, 2, 3], center=[1., 1., 1.])], 1,
     ['1 moment corrections', '[1.00, 1.00, 1.00]', 'range(1, 4)'],
     'array([1, 2, 3]) @ array([1., 1., 1.])'),
    ([dict(moms=[0, 2, 3], center=[1., 1., 1.])], 1,
     ['1 moment corrections', '[1.00, 1.00, 1.00]', '(0, 2, 3)'],
     'array([0, 2, 3]) @ array([1., 1., 1.])'),
    ([dict(moms=range(4), center=[2, 3, 4]),
      dict(moms=range(4), center=[7.4, 3.1, 0.1])], 2,
     ['2 moment corrections', '[2.00, 3.00, 4.00]', '[7.40, 3.10, 0.10]',
      'range(0, 4)'], '2 corrections'),
]


@pytest.mark.parametrize('mc, n, strings, rep', _MC_CASES)
def test_moment_correction_api_reference_cases(mc, n, strings, rep):
    """gpaw/test/poisson/test_poisson_moment.py:11-116: the number of
    corrections each form of ``moment_corrections`` makes, the
    description (the wrapped solver's, then '<n> moment corrections' and
    each centre in Angstrom with its moments) and the repr."""
    import numpy as np
    from gpaw_b200.poisson_moment import (MomentCorrection,
                                          MomentCorrectionPoissonSolver)
    if isinstance(mc, list):
        mc = [dict(moms=m['moms'], center=np.array(m['center']))
              for m in mc]
    ps = MomentCorrectionPoissonSolver(_NoSolver(), mc)
    assert isinstance(ps.moment_corrections, list)
    assert len(ps.moment_corrections) == n
    assert all(isinstance(m, MomentCorrection)
               for m in ps.moment_corrections)
    desc = ps.get_description()
    assert desc.startswith('No interaction')
    rest = desc[len('No interaction'):]
    for s in strings or ['0 moment corrections']:
        assert s in rest, (s, rest)
    assert repr(ps) == f'MomentCorrectionPoissonSolver ({rep})'


def test_grid_descriptor_reference_known_answers():
    """gpaw/test/fd_ops/test_gd.py:7-46 on the product's GridDescriptor:
    the integral of ones over a 4^3 unit cell is 1; distance vectors fold
    a point outside the box along periodic axes only (minimum image); on
    the sheared cell [[1, 1, 0], [0, 1, 0], [0, 0, 1]] the distances of
    row (1, 1) are [-0.5, -0.25, -1, -0.75]."""
    import numpy as np
    import torch
    from gpaw_b200 import GridDescriptor
    gd = GridDescriptor([4, 4, 4], (1.0, 1.0, 1.0), True, device='cpu')
    a = torch.ones(tuple(gd.n_c), dtype=torch.float64)
    assert float(gd.integrate(a)) == 1.0

    def mic(r_v, pbc_c):
        r_c = r_v % 1.0
        r_c -= (2 * r_c).astype(int)
        return np.where(pbc_c, r_c, r_v)
    pbc_c = [1, 1, 0]
    gd = GridDescriptor([10] * 3, (1.0, 1.0, 1.0), pbc_c, device='cpu')
    for r_v in (np.array([0.01, 2.49, 0.01]), np.array([2.49, 0.01, 0.01])):
        dr = gd.get_grid_point_distance_vectors(r_v)
        want = mic(np.dot(gd.h_cv, gd.beg_c) - r_v, pbc_c)
        assert np.abs(dr[:, 0, 0, 0] - want).max() < 1e-15
    cell = np.eye(3)
    cell[0, 1] = 1
    gd = GridDescriptor([2, 4, 1], cell, True, device='cpu')
    r = gd.get_grid_point_distance_vectors(np.zeros(3))
    assert np.allclose(r[1, 1].reshape(4), [-0.5, -0.25, -1., -0.75],
                       rtol=1e-6, atol=1e-12)


def test_madelung_matches_reference_golden():
    """The Madelung potential of the charged-periodic correction
    (gpaw_b200.ewald, an Ewald sum of our own) equals the reference's own
    Ewald code (gpaw/utilities/ewald.py:143-145) on four cells, cubic to
    triclinic: golden values made by tests/golden/make_madelung_golden.py."""
    import json
    import os
    import numpy as np
    from gpaw_b200.ewald import madelung
    path = os.path.join(os.path.dirname(__file__), 'golden', 'madelung.json')
    for case in json.load(open(path)):
        got = madelung(np.array(case['cell']))
        assert abs(got - case['madelung']) <= 1e-12 * abs(case['madelung'])


def test_stencil_spectrum_bounds_equal_dense_sort():
    """The solver's eigenvalue bounds of D^-1 A come from the per-axis
    terms (rounded addition is monotone), in O(N): they equal, bit for bit,
    the smallest / second smallest and largest of all N^3 values sorted."""
    import numpy as np
    from gpaw_b200 import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.poisson import _stencil_spectrum_dense, stencil_spectrum
    rng = np.random.default_rng(0)
    n = 0
    for t in range(120):
        N = tuple(int(x) for x in rng.integers(2, 30, 3))
        pbc = (1, 1, 1) if t % 3 == 0 else \
            tuple(int(x) for x in rng.integers(0, 2, 3))
        cell = tuple(float(x) for x in rng.uniform(2, 12, 3))
        try:
            gd = GridDescriptor(N, cell, pbc, device='cpu')
        except Exception:
            continue
        for nn in (1, 3):
            try:
                op = Laplace(gd, -0.25 / np.pi, nn)
            except AssertionError:      # stencil longer than the grid
                continue
            assert stencil_spectrum(op, gd) == \
                _stencil_spectrum_dense(op, gd), (N, pbc, nn)
            n += 1
    assert n > 100
