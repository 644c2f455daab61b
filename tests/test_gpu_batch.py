"""Batches of uneven Poisson grids: the one-graph mixed-precision batch, the
stream batch and one-by-one solves give identical potentials and V-cycle
counts; the potentials agree with the reference's FP64 solver."""
import numpy as np
import pytest

from oracle import gpaw_layer as L
from tests.helpers import to_np

pytestmark = pytest.mark.gpu


def _grids(pbc=0):
    from gpaw_b200 import GridDescriptor
    h = 0.18 / 0.52917721
    sides = [(32, 40, 24), (48, 32, 40), (24, 24, 56), (40, 48, 32),
             (56, 32, 32), (32, 24, 40)]
    return [GridDescriptor(N, tuple(n * h for n in N), pbc) for N in sides]


def _rhos(gds):
    from gpaw_b200.workloads import neutral_density_device
    return [neutral_density_device(gd, 5 + i, 200 + i)
            for i, gd in enumerate(gds)]


def test_graph_batch_equals_streams_and_single(cuda):
    from gpaw_b200 import MixedPoissonSolver
    from gpaw_b200.batch import PoissonBatch
    gds = _grids()
    rhos = _rhos(gds)
    out = {}
    for mode in ('graph', 'streams'):
        b = PoissonBatch(gds, tol=1e-10, precision='mixed',
                         graph=(mode == 'graph'), nstreams=4)
        phis = [gd.zeros() for gd in gds]
        n = b.solve(phis, rhos)
        out[mode] = (n, [to_np(p) for p in phis])
        # a second call on the same batch reuses the graph
        phis2 = [gd.zeros() for gd in gds]
        assert b.solve(phis2, rhos) == n
        for p, q in zip(phis, phis2):
            assert np.array_equal(to_np(p), to_np(q))
    assert out['graph'][0] == out['streams'][0]
    for p, q in zip(out['graph'][1], out['streams'][1]):
        assert np.array_equal(p, q)
    # one solver alone
    ps = MixedPoissonSolver(tol=1e-10, maxiter=400, fused_coarse='tail')
    ps.set_grid_descriptor(gds[2])
    phi = gds[2].zeros()
    ps.solve_neutral(phi, rhos[2])
    assert np.array_equal(to_np(phi), out['graph'][1][2])


def test_graph_batch_against_reference(cuda):
    from gpaw_b200.batch import PoissonBatch
    gds = _grids()[:3]
    rhos = _rhos(gds)
    b = PoissonBatch(gds, tol=1e-11, precision='mixed')
    phis = [gd.zeros() for gd in gds]
    b.solve(phis, rhos)
    for gd, rho, phi in zip(gds, rhos, phis):
        gref = L.GridDescriptor(tuple(gd.N_c), gd.cell_cv, tuple(gd.pbc_c))
        ps = L.FDPoissonSolver(nn=3, eps=1e-26, maxiter=2000)
        ps.set_grid_descriptor(gref)
        want = gref.zeros()
        ps.solve_neutral(want, to_np(rho))
        got = to_np(phi)
        assert np.abs(got - want).max() / np.abs(want).max() < 1e-9


def test_fp64_batch_equals_single(cuda):
    from gpaw_b200 import FDPoissonSolver
    from gpaw_b200.batch import PoissonBatch
    gds = _grids()[:4]
    rhos = _rhos(gds)
    b = PoissonBatch(gds, tol=1e-10, precision='fp64', nstreams=3)
    phis = [gd.zeros() for gd in gds]
    n = b.solve(phis, rhos)
    for i, gd in enumerate(gds):
        ps = FDPoissonSolver(nn=3, eps=b._eps[i], maxiter=400)
        ps.set_grid_descriptor(gd)
        phi = gd.zeros()
        assert ps.solve_neutral(phi, rhos[i]) == n[i]
        assert np.array_equal(to_np(phi), to_np(phis[i]))
