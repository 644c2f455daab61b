"""GPU parity: every CUDA kernel against the oracle (the reference's own C
core under oracle/_ref, or its numpy restatement), through the C ABI.

Bar: FP64 outputs within 1e-12 relative (max norm) of the oracle; the
kernels keep the reference's operation order without FMA contraction, so
the tests also assert the measured difference is exactly 0 where the
arithmetic is deterministic."""
import numpy as np
import pytest

from oracle import gpaw_layer as L
from tests.helpers import RTOL_FP64, max_rel, to_dev, to_np

pytestmark = pytest.mark.gpu
KPT = (0.25, 0.0, 0.1)


def prod_gd(N, cell, pbc):
    from gpaw_b200 import GridDescriptor
    return GridDescriptor(N, cell, pbc)


# ------------------------------------------------------------ golden cases
def test_golden_fd(golden, cuda):
    from gpaw_b200 import FDOperator
    n = 0
    for name, c in golden.items():
        if not name.startswith('fd_'):
            continue
        gd = prod_gd(tuple(c['N']), c['cell'], tuple(c['pbc']))
        dtype = complex if np.iscomplexobj(c['inp']) else float
        op = FDOperator(c['coefs'], c['offsets'], gd, dtype)
        a = to_dev(c['inp'])
        b = a.new_zeros(a.shape)
        op.apply(a, b, c.get('phases'))
        got = to_np(b)
        assert max_rel(got, c['out']) <= RTOL_FP64, name
        assert np.array_equal(got, c['out']), name
        n += 1
    assert n == 38


def test_golden_relax(golden, cuda):
    from gpaw_b200 import Laplace
    for name, c in golden.items():
        if not name.startswith('relax_'):
            continue
        m = int(name.split('_')[1][1:])
        gd = prod_gd(tuple(c['N']), (3.0, 2.6, 3.3), tuple(c['pbc']))
        op = Laplace(gd, -0.25 / np.pi, 3)
        f = to_dev(c['f'])
        op.relax(m, f, to_dev(c['s']), 3, 2.0 / 3.0)
        assert np.array_equal(to_np(f), c['out']), name


def test_golden_transformers(golden, cuda):
    from gpaw_b200 import Transformer
    for name, c in golden.items():
        if not name.startswith('tr_'):
            continue
        nn = int(name.split('_')[1][2:])
        gd = prod_gd(tuple(c['N']), (3.0, 3.4, 3.9), tuple(c['pbc']))
        gd2 = gd.coarsen()
        dtype = complex if np.iscomplexobj(c['fine']) else float
        ph = c.get('phases')
        r = Transformer(gd, gd2, nn, dtype).apply(to_dev(c['fine']),
                                                  phases=ph)
        i = Transformer(gd2, gd, nn, dtype).apply(to_dev(c['coarse']),
                                                  phases=ph)
        assert np.array_equal(to_np(r), c['restricted']), name
        assert np.array_equal(to_np(i), c['interpolated']), name


def test_golden_preconditioner(golden, cuda):
    from gpaw_b200 import Laplace, Preconditioner
    for name, c in golden.items():
        if not name.startswith('pc_'):
            continue
        gd = prod_gd(tuple(c['N']), (3.0, 3.0, 4.5), tuple(c['pbc']))
        dtype = complex if np.iscomplexobj(c['res']) else float
        kin = Laplace(gd, -0.5, 3, dtype)
        pc = Preconditioner(gd, kin, dtype, block=2)
        R = to_dev(c['res'])
        out = R.new_zeros(R.shape)
        pc(R, c.get('phases'), out=out)
        assert np.array_equal(to_np(out), c['out']), name


def test_golden_poisson(golden, cuda):
    from gpaw_b200 import FDPoissonSolver
    for name, c in golden.items():
        if not name.startswith('ps_'):
            continue
        gd = prod_gd(tuple(c['N']), (4.0, 2.0, 4.0), tuple(c['pbc']))
        ps = FDPoissonSolver(nn=3, eps=1e-18)
        ps.set_grid_descriptor(gd)
        phi = gd.zeros()
        # the neutral branch of solve() (gpaw/poisson.py:186-213), in numpy
        # so that the right-hand side is bit-identical to the oracle's
        n = np.prod(c['N'] - 1 + c['pbc'])
        dv = 4.0 * 2.0 * 4.0 / np.prod(c['N'])
        rho = c['rho'] - c['rho'].sum() * dv / dv / n
        niter = ps.solve_neutral(phi, to_dev(rho))
        assert niter == int(c['niter']), name
        got = to_np(phi)
        # the periodic branch subtracts a mean formed by a reduction whose
        # order differs from numpy's: allow the 1e-12 bar there
        if c['pbc'].all():
            assert max_rel(got, c['phi']) <= RTOL_FP64, name
        else:
            assert np.array_equal(got, c['phi']), name


# -------------------------------------------------- random, larger, batched
@pytest.mark.parametrize('nn', [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0), (0, 1, 1)])
@pytest.mark.parametrize('dtype', [float, complex])
def test_fd_apply_random(nn, pbc, dtype, cuda):
    from gpaw_b200 import Laplace
    rng = np.random.default_rng(nn * 7 + sum(pbc))
    N = (24, 20, 26)
    cell = (4.1, 3.3, 4.4)
    gd = prod_gd(N, cell, pbc)
    a = rng.standard_normal((3,) + tuple(gd.n_c))
    if dtype == complex:
        a = a + 1j * rng.standard_normal(a.shape)
    ph = gd.phase_factor_cd((0.25, -0.1, 0.4)) if dtype == complex else None
    ref = np.zeros_like(a)
    L.Laplace(L.GridDescriptor(N, cell, pbc), -0.5, nn, dtype).apply(a, ref,
                                                                     ph)
    op = Laplace(gd, -0.5, nn, dtype)
    x = to_dev(a)
    y = x.new_zeros(x.shape)
    op.apply(x, y, ph)
    assert max_rel(to_np(y), ref) <= RTOL_FP64
    assert np.array_equal(to_np(y), ref)
    # in-place (in is out), as gpaw/new/fd/hamiltonian.py:47-49 calls it
    op.apply(x, x, ph)
    assert np.array_equal(to_np(x), ref)


def test_fd_nonorthogonal_cell(cuda):
    from gpaw_b200 import Laplace
    cell = [(3.0, 0, 0), (1.5, 3.0 * 3**0.5 / 2, 0), (0, 0, 3.2)]
    for pbc in ((1, 1, 1), (1, 1, 0)):
        for dtype in (float, complex):
            gd = prod_gd((18, 18, 16), cell, pbc)
            rng = np.random.default_rng(3)
            a = rng.standard_normal((2,) + tuple(gd.n_c))
            if dtype == complex:
                a = a + 1j * rng.standard_normal(a.shape)
            ph = gd.phase_factor_cd(KPT) if dtype == complex else None
            ref = np.zeros_like(a)
            L.Laplace(L.GridDescriptor((18, 18, 16), cell, pbc), 1.0, 3,
                      dtype).apply(a, ref, ph)
            op = Laplace(gd, 1.0, 3, dtype)
            assert not op.cfd
            y = to_dev(a)
            z = y.new_zeros(y.shape)
            op.apply(y, z, ph)
            assert np.array_equal(to_np(z), ref), (pbc, dtype)


def test_fd_gaussian_analytic(cuda):
    """gpaw/test/gpu/test_fd_laplace.py:8-60: against the analytic Laplacian
    of a Gaussian (interior, 1e-2)."""
    from gpaw_b200 import Laplace
    lat = 8.0
    gd = prod_gd((32, 32, 32), (lat, lat, lat), 0)
    x, y, z = gd.get_grid_point_coordinates()
    sigma, mu = 1.5, lat / 2
    a = np.exp(-((x - mu)**2 + (y - mu)**2 + (z - mu)**2) / (2.0 * sigma))
    ana = (((x - mu)**2 + (y - mu)**2 + (z - mu)**2) / sigma**2 -
           3.0 / sigma) * a
    b = to_dev(np.zeros_like(a))
    Laplace(gd, 1.0, 3).apply(to_dev(a), b)
    assert np.abs(to_np(b)[2:-2, 2:-2, 2:-2] - ana[2:-2, 2:-2, 2:-2]).max() \
        < 1e-2


@pytest.mark.parametrize('nn', [1, 2, 3, 4])
@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
@pytest.mark.parametrize('dtype', [float, complex])
def test_transformers_random(nn, pbc, dtype, cuda):
    from gpaw_b200 import Transformer
    N = (40, 36, 44)
    cell = (4.0, 3.6, 4.4)
    gdp = prod_gd(N, cell, pbc)
    gdo = L.GridDescriptor(N, cell, pbc)
    rng = np.random.default_rng(nn)
    ph = gdp.phase_factor_cd((0.3, 0.0, -0.15)) if dtype == complex else None

    def rand(g):
        a = rng.standard_normal((2,) + tuple(g.n_c))
        return a + 1j * rng.standard_normal(a.shape) if dtype == complex \
            else a

    a = rand(gdo)
    ref = L.Transformer(gdo, gdo.coarsen(), nn, dtype).apply(a, phases=ph)
    got = Transformer(gdp, gdp.coarsen(), nn, dtype).apply(to_dev(a),
                                                           phases=ph)
    assert np.array_equal(to_np(got), ref)
    c = rand(gdo.coarsen())
    ref = L.Transformer(gdo.coarsen(), gdo, nn, dtype).apply(c, phases=ph)
    got = Transformer(gdp.coarsen(), gdp, nn, dtype).apply(to_dev(c),
                                                           phases=ph)
    assert np.array_equal(to_np(got), ref)


def test_transformers_conserve_integral(cuda):
    """gpaw/test/fd_ops/test_transformations.py:11-52 (periodic, default
    unit cell, k = 2..8, real and complex) and test_non_periodic.py:7-27."""
    from gpaw_b200 import Transformer

    def integrate(g, t):
        # numpy's pairwise sum, as gd.integrate in the reference tests
        return to_np(t).sum() * g.dv

    n = 20
    gd = prod_gd((n, n, n), (1, 1, 1), 1)
    rng = np.random.RandomState(8)
    a = rng.random(tuple(gd.n_c))
    for dtype, phase in ((float, None), (complex, np.ones((3, 2), complex))):
        if dtype == complex:
            a = np.empty(tuple(gd.n_c), complex)
            a.real = rng.random(a.shape)
            a.imag = rng.random(a.shape)
        for g2 in (gd.refine(), gd.coarsen()):
            for k in (2, 4, 6, 8):
                b = Transformer(gd, g2, k // 2, dtype).apply(to_dev(a),
                                                             phases=phase)
                assert abs(integrate(gd, to_dev(a)) - integrate(g2, b)) \
                    < 1e-14
    # zero boundaries
    gd1 = prod_gd((n, n, n), (8.0, 8.0, 8.0), 0)
    rng = np.random.default_rng(8)
    a1 = rng.random(tuple(gd1.n_c))
    gd2 = gd1.refine()
    a2 = to_np(Transformer(gd1, gd2).apply(to_dev(a1)))
    assert abs(a1.sum() * gd1.dv - a2.sum() * gd2.dv) < 1e-10
    for sl in (0, -1):
        a2[sl] = 0.0
        a2[:, sl] = 0.0
        a2[:, :, sl] = 0.0
    a1 = to_np(Transformer(gd2, gd1).apply(to_dev(a2)))
    assert abs(a1.sum() * gd1.dv - a2.sum() * gd2.dv) < 1e-10


@pytest.mark.parametrize('method', [1, 2])
@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0)])
def test_relax_random(method, pbc, cuda):
    from gpaw_b200 import Laplace
    N = (24, 22, 20)
    gd = prod_gd(N, (3.0, 2.8, 2.6), pbc)
    rng = np.random.default_rng(5)
    f = rng.standard_normal(tuple(gd.n_c))
    s = rng.standard_normal(f.shape)
    ref = f.copy()
    L.Laplace(L.GridDescriptor(N, (3.0, 2.8, 2.6), pbc), -0.25 / np.pi,
              3).relax(method, ref, s, 4, 2.0 / 3.0)
    g = to_dev(f)
    Laplace(gd, -0.25 / np.pi, 3).relax(method, g, to_dev(s), 4, 2.0 / 3.0)
    assert np.array_equal(to_np(g), ref)


@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0)])
@pytest.mark.parametrize('dtype', [float, complex])
def test_preconditioner_random(pbc, dtype, cuda):
    from gpaw_b200 import Laplace, Preconditioner
    N = (32, 28, 24)
    cell = (4.0, 3.5, 3.0)
    gdp = prod_gd(N, cell, pbc)
    gdo = L.GridDescriptor(N, cell, pbc)
    rng = np.random.default_rng(11)
    R = rng.standard_normal((5,) + tuple(gdo.n_c))
    if dtype == complex:
        R = R + 1j * rng.standard_normal(R.shape)
    ph = gdo.phase_factor_cd(KPT) if dtype == complex else None
    ref = np.zeros_like(R)
    L.Preconditioner(gdo, L.Laplace(gdo, -0.5, 3, dtype), dtype,
                     block=2)(R, ph, out=ref)
    pc = Preconditioner(gdp, Laplace(gdp, -0.5, 3, dtype), dtype, block=2)
    out = to_dev(np.zeros_like(R))
    pc(to_dev(R), ph, out=out)
    assert np.array_equal(to_np(out), ref)


@pytest.mark.parametrize('relax', ['J', 'GS'])
def test_poisson_c1_against_oracle(relax, cuda):
    """64^3 zero-BC FDPoissonSolver (nn=3): same V-cycle count and the same
    potential as the reference, to the reference's eps=2e-10."""
    from gpaw_b200 import FDPoissonSolver
    h = 0.2 / 0.52917721
    N = (64, 64, 64) if relax == 'J' else (32, 32, 32)
    L_ = N[0] * h
    gdo = L.GridDescriptor(N, (L_,) * 3, 0)
    gdp = prod_gd(N, (L_,) * 3, 0)
    x = gdo.get_grid_point_coordinates()
    rng = np.random.default_rng(1)
    w = 0.8 / 0.52917721
    rho = np.zeros(tuple(gdo.n_c))
    for i in range(8):
        c = rng.uniform(0.25, 0.75, 3) * L_
        q = 1.0 if i % 2 == 0 else -1.0
        r2 = ((x - c[:, None, None, None])**2).sum(0)
        rho += q * (np.pi * w**2)**-1.5 * np.exp(-r2 / w**2)
    rho -= rho.mean()
    ps_o = L.FDPoissonSolver(nn=3, relax=relax, eps=2e-10)
    ps_o.set_grid_descriptor(gdo)
    phi_o = gdo.zeros()
    n_o = ps_o.solve_neutral(phi_o, rho)
    ps = FDPoissonSolver(nn=3, relax=relax, eps=2e-10)
    ps.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    n = ps.solve_neutral(phi, to_dev(rho))
    assert n == n_o
    assert np.array_equal(to_np(phi), phi_o)


@pytest.mark.parametrize('N,pbc', [((64, 64, 64), (0, 0, 0)),
                                   ((32, 32, 32), (1, 1, 1)),
                                   ((48, 32, 40), (1, 1, 0)),
                                   ((40, 24, 56), (0, 1, 0))])
def test_poisson_fused_coarse_levels(N, pbc, cuda, monkeypatch):
    """The coarse levels run as one kernel (all arrays in shared memory)
    give the same V-cycles as the per-level kernels, bit for bit: zero,
    periodic and mixed boundaries; the fused run starting at level 1, at
    level 2, and holding only the coarsest level."""
    from gpaw_b200 import FDPoissonSolver
    gd = prod_gd(N, tuple(0.35 * n for n in N), pbc)
    rng = np.random.default_rng(sum(N))
    rho = rng.standard_normal(tuple(gd.n_c))
    rho -= rho.mean()
    rho_d = to_dev(rho)
    runs = {}
    for tail in ('1', '0'):
        monkeypatch.setenv('GPAW_B200_POISSON_TAIL', tail)
        ps = FDPoissonSolver(nn=3, relax='J')
        ps.set_grid_descriptor(gd)
        phi = gd.zeros()
        errs = [ps.iterate2(0.0, phi=phi, rho=rho_d) for _ in range(5)]
        runs[tail] = (to_np(phi), errs)
        fused = ps._exec.lib.gb_poisson_fused_levels(ps._exec.h)
        assert (fused > 0) == (tail == '1')
    assert np.array_equal(runs['1'][0], runs['0'][0])
    assert runs['1'][1] == runs['0'][1]
    assert runs['1'][1][-1] < runs['1'][1][0]


def test_errors_are_reference_exceptions(cuda):
    import torch
    from gpaw_b200 import FDPoissonSolver, Laplace, PoissonConvergenceError
    gd = prod_gd((16, 16, 16), 3.0, 0)
    op = Laplace(gd, 1.0, 2)
    with pytest.raises(TypeError):
        op.apply(np.zeros(tuple(gd.n_c)), np.zeros(tuple(gd.n_c)))
    a = gd.zeros(dtype=complex)
    with pytest.raises(ValueError, match='dtype'):
        op.apply(a, a.clone())
    ps = FDPoissonSolver(eps=1e-30, maxiter=3)
    ps.set_grid_descriptor(gd)
    rho = torch.randn(tuple(gd.n_c), dtype=torch.float64, device='cuda')
    rho -= rho.mean()
    with pytest.raises(PoissonConvergenceError):
        ps.solve_neutral(gd.zeros(), rho)


@pytest.mark.parametrize('nn', [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize('dtype', [float, complex])
def test_tiled_and_generic_paths_agree(nn, dtype, cuda, monkeypatch):
    """The plane-marching kernels (axis-aligned stencils) and the generic
    kernel give identical results for apply, residual and (real) Jacobi,
    on odd sizes, mixed boundaries, batches and tiles cut by the grid
    edge."""
    import torch
    from gpaw_b200 import Laplace
    rng = np.random.default_rng(100 + nn)
    for N, pbc in (((37, 45, 70), (1, 0, 1)), ((20, 18, 33), (0, 1, 0)),
                   ((12, 14, 16), (1, 1, 1))):
        gd = prod_gd(N, (5.0, 5.5, 6.0), pbc)
        if (gd.n_c < nn).any():
            continue
        ops = {}
        for path in ('generic', 'tiled'):
            monkeypatch.setenv('GPAW_B200_FD_PATH', path)
            ops[path] = Laplace(gd, -0.5, nn, dtype)
        a = rng.standard_normal((3,) + tuple(gd.n_c))
        rho = rng.standard_normal((3,) + tuple(gd.n_c))
        if dtype == complex:
            a = a + 1j * rng.standard_normal(a.shape)
            rho = rho + 1j * rng.standard_normal(a.shape)
        ph = gd.phase_factor_cd((0.2, -0.35, 0.1)) if dtype == complex \
            else None
        x, r = to_dev(a), to_dev(rho)
        outs = {}
        for path, op in ops.items():
            y = x.new_zeros(x.shape)
            op.apply(x, y, ph)
            res = x.new_zeros(x.shape)
            n2 = torch.zeros(3, dtype=torch.float64, device='cuda')
            op.residual(x, r, res, ph, 0.5, n2)
            outs[path] = (to_np(y), to_np(res), to_np(n2))
        assert np.array_equal(outs['generic'][0], outs['tiled'][0])
        assert np.array_equal(outs['generic'][1], outs['tiled'][1])
        assert max_rel(outs['tiled'][2], outs['generic'][2]) < 1e-13
        if dtype == float:
            f = {}
            for path, op in ops.items():
                g = to_dev(a[0])
                op.relax(2, g, to_dev(rho[0]), 3, 0.7)
                f[path] = to_np(g)
            assert np.array_equal(f['generic'], f['tiled'])


def test_fused_apply_opt_in(cuda, monkeypatch):
    """GPAW_B200_FMA=1 switches the complex nn = 3 apply to fused
    multiply-adds: within 1e-12 relative of the reference, and the default
    (switch off) stays bit-identical."""
    from gpaw_b200 import Laplace
    rng = np.random.default_rng(77)
    N, pbc = (40, 36, 44), (1, 1, 1)
    cell = (6.0, 5.4, 6.6)
    gref = L.GridDescriptor(N, cell, pbc)
    want_op = L.Laplace(gref, -0.5, 3, complex)
    gd = prod_gd(N, cell, pbc)
    op = Laplace(gd, -0.5, 3, complex)
    a = rng.standard_normal((2,) + tuple(gd.n_c)) + \
        1j * rng.standard_normal((2,) + tuple(gd.n_c))
    ph = gref.phase_factor_cd(KPT)
    want = np.zeros_like(a)
    want_op.apply(a, want, ph)
    x = to_dev(a)
    for fma in ('1', '0'):
        monkeypatch.setenv('GPAW_B200_FMA', fma)
        y = x.new_zeros(x.shape)
        op.apply(x, y, gd.phase_factor_cd(KPT))
        got = to_np(y)
        assert max_rel(got, want) <= RTOL_FP64
        if fma == '0':
            assert np.array_equal(got, want)


# ------------------------------------------------------- FD Hamiltonian
def test_golden_hamiltonian(golden, cuda):
    """FDHamiltonian.apply_local_potential: kinetic stencil and v * psi in
    one pass, bit-identical to the reference's stencil-then-add."""
    from gpaw_b200 import FDHamiltonian
    n = 0
    for name, c in golden.items():
        if not name.startswith('ham_'):
            continue
        nn = int(name.split('_')[1][2:])
        gd = prod_gd(tuple(c['N']), (3.0, 2.8, 3.6), tuple(c['pbc']))
        dtype = complex if np.iscomplexobj(c['psit']) else float
        ham = FDHamiltonian(gd, kin_stencil=nn, dtype=dtype)
        psit = to_dev(c['psit'])
        out = psit.new_zeros(psit.shape)
        ham.apply_local_potential(to_dev(c['vt']), psit, out, c.get('phases'))
        assert np.array_equal(to_np(out), c['out']), name
        # in place (out is psit)
        ham.apply_local_potential(to_dev(c['vt']), psit, psit, c.get('phases'))
        assert np.array_equal(to_np(psit), c['out']), name
        n += 1
    assert n == 4


@pytest.mark.parametrize('nn', [1, 3, 6])
@pytest.mark.parametrize('dtype', [float, complex])
def test_hamiltonian_random(nn, dtype, cuda):
    """Random batches on odd, mixed-boundary grids against the oracle; the
    generic-stencil path (non-orthogonal cell) too."""
    from gpaw_b200 import FDHamiltonian, GUCLaplace
    rng = np.random.default_rng(300 + nn)
    N, pbc, cell = (23, 19, 30), (1, 0, 1), (4.0, 3.5, 5.0)
    gref = L.GridDescriptor(N, cell, pbc)
    ref = L.FDHamiltonian(gref, nn, dtype)
    gd = prod_gd(N, cell, pbc)
    ham = FDHamiltonian(gd, kin_stencil=nn, dtype=dtype)
    psit = rng.standard_normal((3,) + tuple(gd.n_c))
    if dtype == complex:
        psit = psit + 1j * rng.standard_normal(psit.shape)
    vt = rng.standard_normal(tuple(gd.n_c))
    ph = gref.phase_factor_cd(KPT) if dtype == complex else None
    want = np.zeros_like(psit)
    ref.apply_local_potential(vt, psit, want, ph)
    out = to_dev(np.zeros_like(psit))
    ham.apply_local_potential(to_dev(vt), to_dev(psit), out, ph)
    assert max_rel(to_np(out), want) <= RTOL_FP64
    assert np.array_equal(to_np(out), want)
    if nn == 3:
        # a hexagonal cell: the generic kernel plus the separate v * psi pass
        hcell = [(4.0, 0, 0), (2.0, 4.0 * 3**0.5 / 2, 0), (0, 0, 5.0)]
        gh_ref = L.GridDescriptor((12, 12, 10), hcell, (1, 1, 1))
        gh = prod_gd((12, 12, 10), hcell, (1, 1, 1))
        kin_ref = L.Laplace(gh_ref, -0.5, 2, dtype)
        kin = GUCLaplace(gh, -0.5, 2, dtype)
        p = rng.standard_normal((2,) + tuple(gh.n_c))
        if dtype == complex:
            p = p + 1j * rng.standard_normal(p.shape)
        v = rng.standard_normal(tuple(gh.n_c))
        phh = gh_ref.phase_factor_cd(KPT) if dtype == complex else None
        w = np.zeros_like(p)
        kin_ref.apply(p, w, phh)
        for a, b in zip(p, w):
            b += a * v
        o = to_dev(np.zeros_like(p))
        kin.apply_potential(to_dev(p), o, to_dev(v), phh)
        assert np.array_equal(to_np(o), w)


# ---------------------------------------- charged non-periodic Poisson
def _charged_blob(gdo):
    x = gdo.get_grid_point_coordinates()
    L_ = np.diag(gdo.cell_cv)
    rho = np.zeros(tuple(gdo.n_c))
    for c, w, q in (((0.45, 0.5, 0.55), 1.1, 1.0), ((0.6, 0.4, 0.5), 0.9, 0.6),
                    ((0.35, 0.6, 0.4), 1.3, -0.3)):
        r2 = ((x - (np.array(c) * L_)[:, None, None, None])**2).sum(0)
        rho += q * (np.pi * w**2)**-1.5 * np.exp(-r2 / w**2)
    return rho                      # net charge +1.3


def test_poisson_charged_nonperiodic(cuda):
    """FDPoissonSolver.solve on a charged zero-boundary system (Gaussian
    monopole removal, gpaw/poisson.py:233-283) against the reference."""
    from gpaw_b200 import FDPoissonSolver
    N, cell = (40, 36, 48), (10.0, 9.0, 12.0)
    gdo = L.GridDescriptor(N, cell, 0)
    gdp = prod_gd(N, cell, 0)
    rho = _charged_blob(gdo)
    assert abs(gdo.integrate(rho) - 1.3) < 1e-3
    ps_o = L.FDPoissonSolver(nn=3, eps=1e-16)
    ps_o.set_grid_descriptor(gdo)
    phi_o = gdo.zeros()
    n_o = ps_o.solve(phi_o, rho)
    ps = FDPoissonSolver(nn=3, eps=1e-16)
    ps.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    n = ps.solve(phi, to_dev(rho))
    assert n == n_o
    # the charge is summed on the device (another order than numpy's), so
    # agreement is to rounding, not bit for bit
    assert max_rel(to_np(phi), phi_o) <= RTOL_FP64


def test_mixed_poisson_charged_nonperiodic(cuda):
    from gpaw_b200 import MixedPoissonSolver
    N, cell = (48, 40, 48), (10.0, 9.0, 10.0)
    gdo = L.GridDescriptor(N, cell, 0)
    gdp = prod_gd(N, cell, 0)
    rho = _charged_blob(gdo)
    ps_o = L.FDPoissonSolver(nn=3, eps=1e-24)
    ps_o.set_grid_descriptor(gdo)
    phi_o = gdo.zeros()
    ps_o.solve(phi_o, rho)
    ps = MixedPoissonSolver(nn=3, tol=1e-11)
    ps.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    ps.solve(phi, to_dev(rho))
    assert max_rel(to_np(phi), phi_o) < 1e-9


# ------------------------------------------------------------ Mehrstellen
def test_golden_mehrstellen(golden, cuda):
    """LaplaceA / LaplaceB (gpaw/fd_operators.py:357-396) and the
    FDPoissonSolver(nn='M') branch, bit for bit."""
    from gpaw_b200 import FDPoissonSolver
    from gpaw_b200.fd_operators import LaplaceA, LaplaceB
    n = 0
    for name, c in golden.items():
        if name.startswith('mst_'):
            gd = prod_gd(tuple(c['N']), (3.0, 3.3, 2.8), tuple(c['pbc']))
            dtype = complex if np.iscomplexobj(c['inp']) else float
            a = to_dev(c['inp'])
            oa, ob = a.new_zeros(a.shape), a.new_zeros(a.shape)
            LaplaceA(gd, 0.3, dtype).apply(a, oa, c.get('phases'))
            LaplaceB(gd, dtype).apply(a, ob, c.get('phases'))
            assert np.array_equal(to_np(oa), c['outA']), name
            assert np.array_equal(to_np(ob), c['outB']), name
            n += 1
        elif name.startswith('psM_'):
            gd = prod_gd(tuple(c['N']), (4.0, 4.0, 2.0), tuple(c['pbc']))
            ps = FDPoissonSolver(nn='M', eps=1e-18)
            ps.set_grid_descriptor(gd)
            phi = gd.zeros()
            assert ps.solve(phi, to_dev(c['rho'])) == int(c['niter']), name
            assert max_rel(to_np(phi), c['phi']) <= RTOL_FP64, name
            n += 1
    assert n == 5


@pytest.mark.parametrize('n', [1, 2, 3, 4])
def test_gradient_polynomial_exact(n, cuda):
    """The order-2n central difference differentiates polynomials of degree
    <= 2n exactly (away from the zero boundary); the stencil runs through
    the generic kernel against the oracle's apply of the same stencil."""
    from gpaw_b200.fd_operators import Gradient
    N, cell = (24, 20, 28), (4.8, 4.0, 5.6)
    gd = prod_gd(N, cell, 0)
    gref = L.GridDescriptor(N, cell, 0)
    x = gref.get_grid_point_coordinates()
    f = 0.3 * x[0]**2 * x[1] - 0.2 * x[2]**2 + x[1] * x[2]
    df = [0.6 * x[0] * x[1], 0.3 * x[0]**2 + x[2], -0.4 * x[2] + x[1]]
    m = 2 * n
    for v in range(3):
        gr = Gradient(gd, v, 1.0, n)
        want = np.zeros_like(f)
        L.FDOperator(gr.coef_p, gr.offset_pc, gref).apply(f, want)
        out = to_dev(np.zeros_like(f))
        gr.apply(to_dev(f), out)
        got = to_np(out)
        assert np.array_equal(got, want)
        inner = (slice(m, -m),) * 3
        assert np.allclose(got[inner], df[v][inner], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize('n', [1, 2, 3])
def test_gradient_general_cell(n, cuda):
    """Gradient on a hexagonal, periodic cell (neighbour directions from the
    reduced basis, four of them): the generic kernel against the oracle's
    apply of the same stencil (bit for bit), and against the analytic
    derivative of a smooth periodic function (order-2n accuracy)."""
    from gpaw_b200.fd_operators import Gradient
    a, c = 3.0, 3.2
    cell = [(a, 0, 0), (a / 2, a * 3**0.5 / 2, 0), (0, 0, c)]
    N = (24, 24, 24)
    gd = prod_gd(N, cell, 1)
    gref = L.GridDescriptor(N, cell, 1)
    # reciprocal vectors: exp(i G.r) is periodic in the cell
    G = 2 * np.pi * np.linalg.inv(np.array(cell, float)).T
    x = gref.get_grid_point_coordinates()
    k1, k2 = G[0] + G[1], G[2] - G[0]
    ph1 = np.einsum('v,vxyz->xyz', k1, x)
    ph2 = np.einsum('v,vxyz->xyz', k2, x)
    f = np.sin(ph1) + 0.5 * np.cos(ph2)
    tol = {1: 5e-2, 2: 5e-3, 3: 5e-4}[n]
    for v in range(3):
        gr = Gradient(gd, v, 1.0, n)
        assert gr.cfd == (v == 2)      # in-plane directions mix axes
        df = k1[v] * np.cos(ph1) - 0.5 * k2[v] * np.sin(ph2)
        want = np.zeros_like(f)
        L.FDOperator(gr.coef_p, gr.offset_pc, gref).apply(f, want)
        out = to_dev(np.zeros_like(f))
        gr.apply(to_dev(f), out)
        got = to_np(out)
        assert np.array_equal(got, want)
        assert np.abs(got - df).max() < tol * np.abs(df).max()


# ------------------------------------------------------- dipole correction
def test_dipole_correction_slab(cuda):
    """A neutral slab with a dipole along z (periodic in x and y, zero
    boundary along z): DipoleCorrection around FDPoissonSolver against the
    reference's wrapper around its own solver."""
    from gpaw_b200 import FDPoissonSolver
    from gpaw_b200.dipole import DipoleCorrection
    N, cell, pbc = (24, 24, 48), (5.0, 5.0, 12.0), (1, 1, 0)
    go = L.GridDescriptor(N, cell, pbc)
    gp = prod_gd(N, cell, pbc)
    x = go.get_grid_point_coordinates()
    rho = np.exp(-((x[2] - 5.0)**2) / 0.8) - np.exp(-((x[2] - 7.0)**2) / 0.8)
    rho = rho * (1.0 + 0.2 * np.cos(2 * np.pi * x[0] / 5.0))
    rho -= rho.mean()
    po = L.FDPoissonSolver(nn=3, eps=1e-20)
    po.set_grid_descriptor(go)
    want = go.zeros()
    n_o = L.dipole_fdsolve(po, 2, want, rho)
    ps = DipoleCorrection(FDPoissonSolver(nn=3, eps=1e-20), 2)
    ps.set_grid_descriptor(gp)
    phi = gp.zeros()
    n = ps.solve(phi, to_dev(rho))
    assert n == n_o
    assert max_rel(to_np(phi), want) <= RTOL_FP64
    assert abs(ps.correction) > 0


@pytest.mark.parametrize('n', [1, 2, 3, 4])
@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0), (1, 1, 0)])
def test_pot_calc_density_transfers(n, pbc, cuda):
    """FDPotentialCalculator's transfers: interpolation of a two-spin
    density to the fine grid (rescaled to the coarse integral off periodic
    grids) and restriction back, against the oracle."""
    from gpaw_b200 import GridDescriptor
    from gpaw_b200.pot_calc import FDDensityTransfers
    N = (20, 16, 24)
    cell = (4.0, 3.2, 4.8)
    gd = GridDescriptor(N, cell, pbc)
    finegd = gd.refine()
    gdo = L.GridDescriptor(N, cell, pbc)
    fgo = gdo.refine()
    rng = np.random.default_rng(n + 3 * sum(pbc))
    nt = rng.uniform(0.0, 1.0, (2,) + tuple(gdo.n_c))
    tr = FDDensityTransfers(gd, finegd, n)
    got = to_np(tr.interpolate_density(to_dev(nt)))
    ref = L.interpolate_density(gdo, fgo, nt, n)
    if all(pbc):
        assert np.array_equal(got, ref)
    else:
        assert max_rel(got, ref) <= RTOL_FP64
        assert np.allclose(gdo.integrate(nt), fgo.integrate(got),
                           rtol=1e-12, atol=0)
    back = to_np(tr.restrict(to_dev(ref)))
    back_o = np.zeros_like(nt)
    L.Transformer(fgo, gdo, n).apply(ref, back_o)
    assert np.array_equal(back, back_o)
    assert str(tr).startswith('interpolation: tri-')


def test_golden_weighted_operator(golden, cuda):
    """WeightedFDOperator (gb_wfd.cu) against the reference's WOperator:
    apply (real and complex with Bloch phases), Gauss-Seidel and Jacobi
    relaxation, diagonal element; bit for bit."""
    from gpaw_b200 import FDOperator
    from gpaw_b200.wfd_operators import WeightedFDOperator
    n = 0
    for name, c in golden.items():
        if not name.startswith('wfd_'):
            continue
        gd = prod_gd(tuple(c['N']), (3.1, 2.7, 3.4), tuple(c['pbc']))
        dtype = complex if np.iscomplexobj(c['inp']) else float
        ops = [FDOperator(c[f'coefs{i}'], c[f'offsets{i}'], gd, dtype)
               for i in range(4)]
        wop = WeightedFDOperator(ops)
        ws = [to_dev(c[f'w{i}']) for i in range(4)]
        wop.set_weights(ws)
        x = to_dev(c['inp'])
        y = x.new_zeros(x.shape)
        wop.apply(x, y, c.get('phases'))
        assert np.array_equal(to_np(y), c['out']), name
        assert wop.get_diagonal_element() == float(c['diag']), name
        wop.apply(x, x, c.get('phases'))          # in place
        assert np.array_equal(to_np(x), c['out']), name
        if dtype == float:
            for m in (1, 2):
                f = to_dev(c['f'])
                wop.relax(m, f, to_dev(c['s']), 2, 0.6)
                assert np.array_equal(to_np(f), c[f'relax{m}']), (name, m)
        n += 1
    assert n == 5


@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0), (0, 1, 1)])
def test_weighted_operator_solvation_stencils(pbc, cuda):
    """The solvation solver's operator (nn = 3 Laplacian and the three
    Gradients weighted by eps and its gradient) on a larger grid and a
    batch, against the oracle."""
    from gpaw_b200 import Gradient, Laplace
    from gpaw_b200.wfd_operators import WeightedFDOperator
    N, cell = (24, 20, 28), (4.4, 3.6, 5.0)
    gd = prod_gd(N, cell, pbc)
    gdo = L.GridDescriptor(N, cell, pbc)
    ops = [Laplace(gd, -0.25 / np.pi, 3)] + \
        [Gradient(gd, v, -0.25 / np.pi, 3) for v in range(3)]
    ops_o = [L.FDOperator(op.coef_p, op.offset_pc, gdo) for op in ops]
    rng = np.random.default_rng(sum(pbc))
    w = [rng.uniform(1.0, 80.0, tuple(gdo.n_c))] + \
        [rng.standard_normal(tuple(gdo.n_c)) for _ in range(3)]
    wop = WeightedFDOperator(ops)
    wop.set_weights([to_dev(a) for a in w])
    wop_o = L.WeightedFDOperator(ops_o)
    wop_o.set_weights(w)
    a = rng.standard_normal((3,) + tuple(gdo.n_c))
    ref = np.zeros_like(a)
    wop_o.apply(a, ref)
    x = to_dev(a)
    y = x.new_zeros(x.shape)
    wop.apply(x, y)
    assert np.array_equal(to_np(y), ref)
    assert wop.get_diagonal_element() == wop_o.get_diagonal_element()
    f = rng.standard_normal(tuple(gdo.n_c))
    s = rng.standard_normal(tuple(gdo.n_c))
    fo = f.copy()
    wop_o.relax(2, fo, s, 3, 2.0 / 3.0)
    fd = to_dev(f)
    wop.relax(2, fd, to_dev(s), 3, 2.0 / 3.0)
    assert np.array_equal(to_np(fd), fo)


@pytest.mark.parametrize('nn', [1, 2, 3, 4])
@pytest.mark.parametrize('dtype', [float, complex])
@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 1, 0)])
def test_weighted_operator_ranges(nn, dtype, pbc, cuda):
    """Weighted Laplacian + gradients of range 1..4 (the plane-marching
    kernel for ranges 1-3, and 4-6 in float64; the per-point kernel for
    complex range 4), real and complex with Bloch phases, on a grid whose
    sides are not multiples of the tile, against the oracle."""
    from gpaw_b200 import Gradient, Laplace
    from gpaw_b200.wfd_operators import WeightedFDOperator
    N, cell = (19, 21, 37), (3.3, 3.6, 6.1)
    gd = prod_gd(N, cell, pbc)
    gdo = L.GridDescriptor(N, cell, pbc)
    ops = [Laplace(gd, 0.7, nn, dtype)] + \
        [Gradient(gd, v, 0.3, nn, dtype) for v in range(3)]
    ops_o = [L.FDOperator(op.coef_p, op.offset_pc, gdo, dtype) for op in ops]
    rng = np.random.default_rng(nn + 5 * sum(pbc))
    w = [rng.uniform(1.0, 3.0, tuple(gdo.n_c))] + \
        [rng.standard_normal(tuple(gdo.n_c)) for _ in range(3)]
    wop = WeightedFDOperator(ops)
    wop.set_weights([to_dev(a) for a in w])
    wop_o = L.WeightedFDOperator(ops_o)
    wop_o.set_weights(w)
    a = rng.standard_normal((2,) + tuple(gdo.n_c))
    if dtype == complex:
        a = a + 1j * rng.standard_normal(a.shape)
    ph = gdo.phase_factor_cd(KPT) if dtype == complex else None
    ref = np.zeros_like(a)
    wop_o.apply(a, ref, ph)
    x = to_dev(a)
    y = x.new_zeros(x.shape)
    wop.apply(x, y, ph)
    assert np.array_equal(to_np(y), ref)


def test_weighted_poisson_against_oracle(cuda):
    """WeightedFDPoissonSolver (gpaw/old/solvation/poisson.py:75-124) with a
    smooth dielectric (eps 1 inside a sphere, 80 outside) against the
    oracle's restatement on the reference's WOperator and Transformer: the
    same V-cycle count and the same potential, bit for bit."""
    from gpaw_b200 import Gradient, Laplace
    from gpaw_b200.solvation import WeightedFDPoissonSolver
    N, cell = (32, 32, 32), (8.0, 8.0, 8.0)
    gdo = L.GridDescriptor(N, cell, 0)
    gdp = prod_gd(N, cell, 0)
    x = gdo.get_grid_point_coordinates() - 4.0
    g = np.exp(-(x**2).sum(0) / 3.0)
    eps = 80.0 - 79.0 * g
    grad = [79.0 * g * 2.0 * x[c] / 3.0 for c in range(3)]
    rho = np.exp(-((x[0] - 0.6)**2 + x[1]**2 + x[2]**2)) - \
        np.exp(-((x[0] + 0.6)**2 + x[1]**2 + x[2]**2))
    rho -= rho.mean()

    def stencils(g_, scale, n):
        gp = prod_gd(tuple(g_.N_c), cell, 0)
        ops = [Laplace(gp, scale, n)] + [Gradient(gp, j, scale, n)
                                         for j in range(3)]
        return [(op.coef_p, op.offset_pc) for op in ops]

    wo = L.WeightedFDPoissonSolver(stencils, nn=3, eps=1e-14, maxiter=300)
    wo.set_grid_descriptor(gdo)
    wo.set_dielectric([eps] + grad)
    wo.restrict_op_weights()
    phi_o = gdo.zeros()
    n_o = wo.solve_neutral(phi_o, rho)

    class Dielectric:
        eps_gradeps = [to_dev(a) for a in [eps] + grad]

    ps = WeightedFDPoissonSolver(nn=3, eps=1e-14, maxiter=300)
    ps.set_grid_descriptor(gdp)
    ps.set_dielectric(Dielectric())
    ps.restrict_op_weights()
    assert ps.step == wo.step
    phi = gdp.zeros()
    n = ps.solve_neutral(phi, to_dev(rho))
    assert n == n_o
    assert np.array_equal(to_np(phi), phi_o)
    assert 'weighted FD solver with dielectric' in ps.get_description()


def test_weighted_poisson_charged_against_oracle(cuda):
    """A charged system in a zero-boundary cell with a dielectric: the
    compensation charge of load_gauss (gpaw/old/solvation/poisson.py:48-72)
    equals the oracle's bit for bit; the solve agrees to the 1e-12 bar (the
    charge is summed on the device, in another order than numpy's)."""
    from gpaw_b200 import Gradient, Laplace
    from gpaw_b200.solvation import WeightedFDPoissonSolver
    N, cell = (32, 28, 36), (8.0, 7.0, 9.0)
    gdo = L.GridDescriptor(N, cell, 0)
    gdp = prod_gd(N, cell, 0)
    x = gdo.get_grid_point_coordinates() - np.array(cell)[:, None, None,
                                                             None] / 2
    g = np.exp(-(x**2).sum(0) / 2.5)
    arrays = [80.0 - 79.0 * g] + [79.0 * g * 2.0 * x[c] / 2.5
                                  for c in range(3)]
    rho = np.exp(-((x[0] - 0.3)**2 + x[1]**2 + x[2]**2) / 0.8)
    assert gdo.integrate(rho) > 0.1

    def stencils(g_, scale, n):
        gp = prod_gd(tuple(g_.N_c), cell, 0)
        ops = [Laplace(gp, scale, n)] + [Gradient(gp, j, scale, n)
                                         for j in range(3)]
        return [(op.coef_p, op.offset_pc) for op in ops]

    wo = L.WeightedFDPoissonSolver(stencils, nn=3, eps=1e-16, maxiter=400)
    wo.set_grid_descriptor(gdo)
    wo.set_dielectric(arrays)
    phi_o = gdo.zeros()
    n_o = wo.solve(phi_o, rho)

    class Dielectric:
        eps_gradeps = [to_dev(a) for a in arrays]

    ps = WeightedFDPoissonSolver(nn=3, eps=1e-16, maxiter=400)
    ps.set_grid_descriptor(gdp)
    ps.set_dielectric(Dielectric())
    phi = gdp.zeros()
    n = ps.solve(phi, to_dev(rho))
    assert np.array_equal(to_np(ps.rho_gauss), wo.rho_gauss)
    assert np.array_equal(to_np(ps.phi_gauss), wo.phi_gauss)
    assert n == n_o
    assert max_rel(to_np(phi), phi_o) <= RTOL_FP64


@pytest.mark.parametrize('corr', ['center', 'two'])
def test_moment_correction_against_oracle(corr, cuda):
    """MomentCorrectionPoissonSolver (gpaw/poisson_moment.py:60-243) around
    FDPoissonSolver on a charged, polarised zero-boundary system: the
    moments removed about the middle of the cell (L = 0..8) or about two
    centres (every point assigned to the nearer), against the oracle's
    restatement; agreement to the 1e-12 bar (the moments are device
    sums)."""
    from gpaw_b200 import FDPoissonSolver
    from gpaw_b200.poisson_moment import MomentCorrectionPoissonSolver
    N, cell = (40, 36, 44), (10.0, 9.0, 11.0)
    gdo = L.GridDescriptor(N, cell, 0)
    gdp = prod_gd(N, cell, 0)
    x = gdo.get_grid_point_coordinates()
    c0 = np.array(cell) / 2
    d1 = x - (c0 + np.array([1.0, 0.4, -0.6]))[:, None, None, None]
    d2 = x - (c0 - np.array([1.2, -0.5, 0.8]))[:, None, None, None]
    rho = np.exp(-(d1**2).sum(0) / 0.7) - 0.4 * np.exp(-(d2**2).sum(0) / 0.5)
    if corr == 'center':
        mc_p, mc_o = 9, 9
    else:
        from gpaw_b200.poisson_moment import BOHR
        ca = [(c0 + [1.0, 0.4, -0.6]) * BOHR,
              (c0 - [1.2, -0.5, 0.8]) * BOHR]
        mc_p = [{'moms': range(4), 'center': ca[0]},
                {'moms': [0, 3, 6], 'center': ca[1]}]
        mc_o = [{'moms': range(4), 'center': np.asarray(ca[0]) / BOHR},
                {'moms': [0, 3, 6],
                 'center': np.asarray(ca[1]) / BOHR}]
    po = L.MomentCorrectionPoissonSolver(L.FDPoissonSolver(nn=3, eps=1e-18),
                                         mc_o)
    po.set_grid_descriptor(gdo)
    phi_o = gdo.zeros()
    n_o = po.solve(phi_o, rho)
    pp = MomentCorrectionPoissonSolver(FDPoissonSolver(nn=3, eps=1e-18), mc_p)
    pp.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    n = pp.solve(phi, to_dev(rho))
    assert n == n_o
    assert max_rel(to_np(phi), phi_o) <= RTOL_FP64
    assert 'moment corrections' in pp.get_description()


@pytest.mark.parametrize('coarses,gpts', [(0, 48), (1, 48), (1, 64),
                                            (2, 96)])
def test_extra_vacuum_against_oracle(coarses, gpts, cuda):
    """ExtraVacuumPoissonSolver (gpaw/poisson_extravacuum.py:13-232): the
    solve on a larger grid (and, with coarses = 1, on a coarser large grid
    whose refined potential corrects the solve on the original grid)
    against the oracle's restatement: the same V-cycle counts, the
    potential to the 1e-12 bar.  With 64 and 96 points the product's
    auxiliary grid (padded by the stencils' reach) is smaller than the
    reference's, which must not change the result."""
    from gpaw_b200 import FDPoissonSolver
    from gpaw_b200.poisson_extravacuum import ExtraVacuumPoissonSolver
    N, cell = (24, 24, 24), (6.0, 6.0, 6.0)
    gdo = L.GridDescriptor(N, cell, 0)
    gdp = prod_gd(N, cell, 0)
    x = gdo.get_grid_point_coordinates() - 3.0
    rho = np.exp(-((x[0] - 0.5)**2 + x[1]**2 + x[2]**2)) - \
        np.exp(-((x[0] + 0.5)**2 + x[1]**2 + x[2]**2))
    small_o = L.FDPoissonSolver(eps=1e-18) if coarses else None
    small_p = FDPoissonSolver(eps=1e-18) if coarses else None
    evo = L.ExtraVacuumPoissonSolver((gpts,) * 3, L.FDPoissonSolver(eps=1e-18),
                                     small_o, coarses=coarses)
    evo.set_grid_descriptor(gdo)
    phi_o = gdo.zeros()
    n_o = evo.solve(phi_o, rho)
    evp = ExtraVacuumPoissonSolver((gpts,) * 3, FDPoissonSolver(eps=1e-18),
                                   small_p, coarses=coarses)
    evp.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    n = evp.solve(phi, to_dev(rho))
    assert n == n_o
    assert max_rel(to_np(phi), phi_o) <= RTOL_FP64
    assert 'ExtraVacuum' in evp.get_description()


# ----------------------------------- FDPoissonSolver's remaining options
def test_remove_moment_against_oracle(cuda):
    """FDPoissonSolver(remove_moment=4) (gpaw/poisson.py:192-208) on a
    charged, polarised density in a zero-boundary cell against the
    reference's algorithm restated with the oracle's Gaussians and
    solver: the same V-cycle count, phi to the 1e-12 bar."""
    from gpaw_b200 import FDPoissonSolver
    N, cell = (40, 36, 44), (7.0, 6.3, 7.7)
    gdo = L.GridDescriptor(N, cell, 0)
    gdp = prod_gd(N, cell, 0)
    x = gdo.get_grid_point_coordinates()
    c = np.array(cell)[:, None, None, None] / 2
    rho = 1.3 * np.exp(-((x - c + 0.6)**2).sum(0)) - \
        0.4 * np.exp(-1.5 * ((x - c - 0.8)**2).sum(0))
    po = L.FDPoissonSolver(nn=3, eps=1e-16)
    po.set_grid_descriptor(gdo)
    G = L.GaussianMP(gdo)
    rho_n = rho.copy()
    cors = [G.remove_moment(rho_n, Lm) for Lm in range(4)]
    ref = gdo.zeros()
    for cor in cors:
        ref -= cor
    n_ref = po.solve_neutral(ref, rho_n)
    for cor in cors:
        ref += cor
    ps = FDPoissonSolver(nn=3, eps=1e-16, remove_moment=4)
    ps.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    n = ps.solve(phi, to_dev(rho))
    assert n == n_ref
    assert max_rel(to_np(phi), ref) <= RTOL_FP64
    assert ps.todict()['remove_moment'] == 4


def test_charged_periodic_madelung_correction(cuda):
    """use_charged_periodic_corrections (gpaw/poisson.py:214-231): the
    potential of a charged periodic cell shifted by charge x the Madelung
    potential of the lattice (pinned to the reference's Ewald values on the
    CPU), i.e. exactly the plain solve plus that constant."""
    from gpaw_b200 import FDPoissonSolver
    from gpaw_b200.ewald import madelung
    N, cell = (32, 28, 36), (5.0, 4.4, 5.6)
    gdp = prod_gd(N, cell, 1)
    rng = np.random.default_rng(4)
    rho = to_dev(rng.standard_normal(N) + 0.3)
    out = {}
    for corr in (False, True):
        ps = FDPoissonSolver(nn=3, eps=1e-14,
                             use_charged_periodic_corrections=corr)
        ps.set_grid_descriptor(gdp)
        phi = gdp.zeros()
        out[corr] = (ps.solve(phi, rho), to_np(phi))
    q = float(gdp.integrate(rho))
    assert out[True][0] == out[False][0]
    shift = out[True][1] - out[False][1]
    want = q * madelung(np.diag(cell))
    assert np.abs(shift - want).max() <= 1e-12 * abs(want)


@pytest.mark.parametrize('electrodes', ['single', 'both'])
def test_metallic_electrodes_against_oracle(electrodes, cuda):
    """metallic_electrodes (gpaw/poisson.py:284-310) for a charged slab,
    periodic in x and y: 'both' solves the charged density as it is,
    'single' adds a dipole layer against the electrode at the top of z
    and shifts by its potential step; against the reference's branch
    restated on the oracle."""
    from gpaw_b200 import FDPoissonSolver
    N, cell, pbc = (24, 24, 48), (5.0, 5.0, 12.0), (1, 1, 0)
    gdo = L.GridDescriptor(N, cell, pbc)
    gdp = prod_gd(N, cell, pbc)
    x = gdo.get_grid_point_coordinates()
    rho = np.exp(-((x[2] - 5.0)**2) / 0.8) * (1.0 + 0.2 * np.cos(
        2 * np.pi * x[0] / 5.0))
    po = L.FDPoissonSolver(nn=3, eps=1e-16)
    po.set_grid_descriptor(gdo)
    ref = gdo.zeros()
    if electrodes == 'both':
        n_ref = po.solve_neutral(ref, rho)
    else:
        drho, dphi, corr = L.dipole_correction(2, gdo, rho,
                                               origin_c=[0, 0, N[2]])
        ref -= dphi
        n_ref = po.solve_neutral(ref, rho + drho)
        ref += dphi
        ref -= corr
    ps = FDPoissonSolver(nn=3, eps=1e-16, metallic_electrodes=electrodes)
    ps.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    n = ps.solve(phi, to_dev(rho))
    assert n == n_ref
    assert max_rel(to_np(phi), ref) <= RTOL_FP64


def test_charge_center_monopole_against_oracle(cuda):
    """use_charge_center (gpaw/poisson.py:241-262) on one GPU: the monopole
    Gaussian is put on the centre of the density's majority charge.  The
    reference's test_poisson_asym case (gpaw/test/poisson/
    test_poisson_asym.py:9-41: a unit Gaussian at (a/2, a/2, 3a/4), 20 Bohr
    zero-boundary cell, 48^3, nn = 3) gives its analytic potential to 1e-5;
    a perturbed density matches the reference's branch restated on the
    oracle (same V-cycle count, phi to the 1e-12 bar)."""
    from gpaw_b200 import FDPoissonSolver
    a, N = 20.0, (48, 48, 48)
    gdo = L.GridDescriptor(N, (a, a, a), 0)
    gdp = prod_gd(N, (a, a, a), 0)
    c0 = np.array((a / 2, a / 2, 3 * a / 4))
    G0 = L.GaussianMP(gdo, a=19., center=c0)
    ng, vg = G0.get_gauss(0), G0.get_gauss_pot(0)
    ps = FDPoissonSolver(nn=3, relax='J', use_charge_center=True)
    ps.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    ps.solve(phi, to_dev(ng), charge=1.0)
    assert (((to_np(phi) - vg)**2).sum() * gdo.dv)**0.5 < 1e-5
    # a lopsided density: the oracle restatement of the branch
    x = gdo.get_grid_point_coordinates()
    rho = ng + 0.05 * np.exp(-((x - c0[:, None, None, None] + 2.0)**2)
                             .sum(0)) - 0.01
    q_tot = gdo.integrate(rho)
    sign = np.where(rho * np.sign(q_tot) < 0, 0.0, rho * np.sign(q_tot))
    center = -(L.calculate_dipole_moment(gdo, sign) / gdo.integrate(sign))
    Gc = L.GaussianMP(gdo, a=19., center=center)
    rho_g, phi_g = Gc.get_gauss(0), Gc.get_gauss_pot(0)
    q = q_tot / np.sqrt(4 * np.pi)
    po = L.FDPoissonSolver(nn=3, relax='J')
    po.set_grid_descriptor(gdo)
    ref = gdo.zeros() - q * phi_g
    n_ref = po.solve_neutral(ref, rho - q * rho_g)
    ref += q * phi_g
    ps2 = FDPoissonSolver(nn=3, relax='J', use_charge_center=True)
    ps2.set_grid_descriptor(gdp)
    phi2 = gdp.zeros()
    n = ps2.solve(phi2, to_dev(rho))
    assert n == n_ref
    assert max_rel(to_np(phi2), ref) <= RTOL_FP64


# -------------------------------------------------- spectral Laplacian n=9
@pytest.mark.parametrize('dtype', [float, complex])
def test_ft_laplace_against_oracle(dtype, cuda):
    """Laplace(n=9) (gpaw/fd_operators.py:177-181, 399-424): a batch of
    random grids in a general periodic cell against the reference's numpy
    transform (1e-12 of the largest value), and the known answer on a plane
    wave: -|k|^2 times the wave, to rounding."""
    from gpaw_b200 import Laplace
    N, cell = (24, 20, 28), [[5.0, 0.0, 0.0], [0.8, 4.4, 0.0],
                             [0.3, -0.5, 6.1]]
    gdo = L.GridDescriptor(N, cell, 1)
    gdp = prod_gd(N, cell, 1)
    rng = np.random.default_rng(21)
    a = rng.standard_normal((3,) + N)
    if dtype is complex:
        a = a + 1j * rng.standard_normal((3,) + N)
    op = Laplace(gdp, -0.5, 9, dtype)
    out = to_dev(np.zeros_like(a))
    op.apply(to_dev(a), out)
    want = L.ft_laplace(gdo, -0.5, a)
    assert max_rel(to_np(out), want) <= 1e-12
    assert op.get_diagonal_element() == 6.0 / gdo.h_cv[0, 0]**2
    # cos(G.r) with G a reciprocal lattice vector: eigenvalue -|G|^2
    G = 2 * np.pi * np.linalg.inv(gdo.cell_cv) @ np.array([1, -2, 1])
    r = gdo.get_grid_point_coordinates()
    wave = np.cos(np.einsum('v,vxyz->xyz', G, r))
    lap = Laplace(gdp, 1.0, 9)
    got = gdp.zeros()
    lap.apply(to_dev(wave), got)
    assert np.abs(to_np(got) + (G @ G) * wave).max() <= 1e-11 * (G @ G)
