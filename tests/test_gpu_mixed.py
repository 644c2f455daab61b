"""Mixed-precision Poisson solver (FP32 V-cycles in FP64 defect correction)
against the FP64 oracle.

Bar: the relative residual ||rho - L phi|| / ||rho||, recomputed here in
FP64 by the oracle's own operator, is at most 1e-10 (x 1.01 for the
different summation order), and the potential agrees with the oracle's FP64
solution (solved to 1e-12) within 1e-7 relative (max norm); the measured
maximum error is printed."""
import numpy as np
import pytest

from oracle import gpaw_layer as L
from tests.helpers import to_dev, to_np

pytestmark = pytest.mark.gpu


def _case(N, pbc, seed):
    from gpaw_b200.workloads import BOHR, c1_density, neutralize
    h = 0.2 / BOHR
    gdo = L.GridDescriptor(N, tuple(n * h for n in N), pbc)
    rho = neutralize(c1_density(gdo, seed=seed), gdo)
    return gdo, rho


@pytest.mark.parametrize('fused', [True, False, 'tail'])
@pytest.mark.parametrize('N,pbc', [((64, 64, 64), 0), ((48, 40, 56), 0),
                                   ((48, 48, 48), 1)])
def test_mixed_reaches_1e10_and_matches_fp64(N, pbc, fused, cuda, capsys):
    """Both forms of the coarse levels (one cooperative kernel with the
    exact coarsest solve, or one kernel a pass with the Chebyshev coarsest
    solve) reach the tolerance and the FP64 solution."""
    from gpaw_b200 import GridDescriptor, MixedPoissonSolver
    gdo, rho = _case(N, pbc, seed=3)
    gdp = GridDescriptor(N, np.diag(gdo.cell_cv), pbc)
    ps = MixedPoissonSolver(nn=3, tol=1e-10, fused_coarse=fused)
    ps.set_grid_descriptor(gdp)
    phi = gdp.zeros()
    n = ps.solve_neutral(phi, to_dev(rho))
    got = to_np(phi)
    # FP64 relative residual with the oracle's operator
    op = L.Laplace(gdo, -0.25 / np.pi, 3)
    lphi = np.zeros_like(got)
    op.apply(got, lphi)
    rel = np.sqrt(((rho - lphi)**2).sum() / (rho**2).sum())
    # oracle FP64 solution to 1e-12 relative
    eps = (1e-12 * np.sqrt((rho * rho).sum()))**2 * gdo.dv
    po = L.FDPoissonSolver(nn=3, eps=eps, maxiter=2000)
    po.set_grid_descriptor(gdo)
    ref = gdo.zeros()
    po.solve_neutral(ref, rho)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    with capsys.disabled():
        print(f'\nmixed {N} pbc={pbc} fused={fused}: {n} V-cycles, '
              f'rel residual {rel:.3e} '
              f'(device {ps.rel_residual:.3e}), max rel error vs FP64 '
              f'{err:.3e}')
    assert rel <= 1.01e-10
    assert err <= 1e-7
    assert n < 40


def test_mixed_nonconvergence_raises(cuda):
    from gpaw_b200 import (GridDescriptor, MixedPoissonSolver,
                           PoissonConvergenceError)
    gdo, rho = _case((32, 32, 32), 0, seed=1)
    gdp = GridDescriptor((32, 32, 32), np.diag(gdo.cell_cv), 0)
    ps = MixedPoissonSolver(tol=1e-10, maxiter=2)
    ps.set_grid_descriptor(gdp)
    with pytest.raises(PoissonConvergenceError):
        ps.solve_neutral(gdp.zeros(), to_dev(rho))
    assert ps.niter == 2


def test_solver_pool_reuses_memory_and_results(cuda):
    """Solvers built through the library's caching allocator (gb_pool_*):
    a dropped solver's blocks are cached and handed to the next one of the
    same size classes (no new driver memory), the results are bit-identical
    to solvers built without the pool, and release empties the cache."""
    import gc
    from gpaw_b200 import GridDescriptor, MixedPoissonSolver
    from gpaw_b200._lib import (release_solver_pool, solver_pool,
                                solver_pool_stats)
    from gpaw_b200.workloads import neutral_density_device
    shapes = [(40, 56, 48), (32, 32, 64)]

    def solve(N):
        gd = GridDescriptor(N, tuple(0.34 * n for n in N), 0)
        ps = MixedPoissonSolver(nn=3, tol=1e-10, levels=4)
        ps.set_grid_descriptor(gd)
        rho = neutral_density_device(gd, 6, 3)
        phi = gd.zeros()
        n = ps.solve_neutral(phi, rho)
        return n, phi.cpu().numpy()

    plain = [solve(N) for N in shapes]
    gc.collect()
    with solver_pool():
        first = [solve(N) for N in shapes]
        gc.collect()
        live0, cached0 = solver_pool_stats()
        assert cached0 > 0
        again = [solve(N) for N in shapes]
        gc.collect()
        live1, cached1 = solver_pool_stats()
        assert cached1 == cached0          # every block came from the cache
    for a, b, c in zip(plain, first, again):
        assert a[0] == b[0] == c[0]
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[1], c[1])
    release_solver_pool()
