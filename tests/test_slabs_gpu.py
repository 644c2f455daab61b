"""Slab geometry on the GPU without a process group."""
import numpy as np
import pytest


@pytest.mark.gpu
def test_slab_transfers_on_gpu(cuda):
    """Each of three emulated ranks restricts or interpolates its own output
    planes from a replicated input (so the gather is local) with the
    library's transformer kernels on the slab geometry (no axis-0 padding,
    slabs that start on odd points, an extra plane dropped): the planes
    equal the whole-grid transformer's bit for bit."""
    from gpaw_b200 import GridDescriptor
    from gpaw_b200.domains import (DistributedTransformer, SlabDomain,
                                   gpu_local_transformer)
    from gpaw_b200.transformers import Transformer
    from tests.helpers import to_dev, to_np
    bad = []
    for pbc0 in (1, 0):
        gd = GridDescriptor((26, 12, 10), (5.2, 2.4, 2.0), (pbc0, 1, 0))
        gd2 = gd.coarsen()
        ph = gd.phase_factor_cd((0.3, -0.2, 0.0))
        for dtype in (float, complex):
            phases = ph if dtype == complex else None
            for nn in (1, 3):
                for interp in (False, True):
                    gi, go = (gd2, gd) if interp else (gd, gd2)
                    rng = np.random.default_rng(nn + 2 * pbc0)
                    a = rng.standard_normal((2,) + tuple(gi.n_c))
                    if dtype == complex:
                        a = a + 1j * rng.standard_normal(a.shape)
                    x = to_dev(a)
                    ref = go.zeros((2,), dtype)
                    Transformer(gi, go, nn, dtype).apply(x, ref, phases)
                    ref = to_np(ref)
                    for r in range(3):
                        di = SlabDomain(gi.n_c, pbc0, r, 3, True)
                        do = SlabDomain(go.n_c, pbc0, r, 3)
                        t = DistributedTransformer(gi, go, nn, dtype, di, do,
                                                   gpu_local_transformer())
                        out = x.new_zeros((2,) + do.local_shape())
                        t.apply(x, out, phases)
                        if not np.array_equal(to_np(out),
                                              ref[:, do.beg:do.end]):
                            bad.append((pbc0, dtype.__name__, nn, interp, r))
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize('pbc0', [1, 0])
def test_single_slab_vcycles_on_gpu(cuda, pbc0):
    """One rank: three V-cycles of the slab solver with the library's
    kernels leave phi equal to the native executor's V-cycles."""
    from gpaw_b200 import FDPoissonSolver, GridDescriptor
    from gpaw_b200.domains import (DistributedFDPoissonSolver,
                                   gpu_local_operator, gpu_local_transformer)
    from tests.helpers import to_dev, to_np
    gd = GridDescriptor((24, 16, 16), (6.0, 4.0, 4.4), (pbc0, 1, 0))
    rng = np.random.default_rng(17)
    rho = to_dev(rng.standard_normal(tuple(gd.n_c)))
    phi0 = rng.standard_normal(tuple(gd.n_c)) * 0.1
    ps = FDPoissonSolver(nn=3, relax='J')
    ps.set_grid_descriptor(gd)
    ps._init()
    ref = to_dev(phi0)
    ref_err = [ps.iterate2(ps.step, phi=ref, rho=rho) for _ in range(3)]
    dps = DistributedFDPoissonSolver(ps, 0, 1,
                                     gpu_local_operator(float, ref.device),
                                     gpu_local_transformer())
    phi = to_dev(phi0)
    err = [dps.iterate(phi, rho) for _ in range(3)]
    assert np.array_equal(to_np(phi), to_np(ref))
    for e, r in zip(err, ref_err):
        assert abs(e - r) <= 1e-12 * abs(r)


@pytest.mark.gpu
@pytest.mark.parametrize('pbc0', [1, 0])
def test_slab_vcycles_emulated_ranks_against_oracle(cuda, pbc0):
    """Three ranks emulated on one GPU (LocalRanks: threads exchanging the
    halo and transfer planes in memory, the same messages as over a process
    group), each running its slab of the FD Poisson V-cycle with the
    library's kernels: after three V-cycles every slab of phi equals the
    oracle's whole-grid V-cycles (the reference's C core) bit for bit, and
    the level-0 error summed over the ranks matches to rounding."""
    from gpaw_b200 import FDPoissonSolver, GridDescriptor
    from gpaw_b200.domains import (DistributedFDPoissonSolver, LocalRanks,
                                   gpu_local_operator, gpu_local_transformer)
    from oracle import gpaw_layer as L
    from tests.helpers import to_dev, to_np
    N, cell, pbc = (24, 16, 16), (6.0, 4.0, 4.4), (pbc0, 1, 0)
    gdo = L.GridDescriptor(N, cell, pbc)
    rng = np.random.default_rng(17)
    rho = rng.standard_normal(tuple(gdo.n_c))
    phi0 = rng.standard_normal(tuple(gdo.n_c)) * 0.1
    po = L.FDPoissonSolver(nn=3, relax='J')
    po.set_grid_descriptor(gdo)
    po._init()
    po.phis[0] = phi0.copy()
    po.rhos[0][:] = rho
    po.errors = []
    ref_err = [po.iterate2(po.step) for _ in range(3)]
    gd = GridDescriptor(N, cell, pbc)
    ps = FDPoissonSolver(nn=3, relax='J')
    ps.set_grid_descriptor(gd)

    def rank_body(rank, group):
        dps = DistributedFDPoissonSolver(
            ps, rank, 3, gpu_local_operator(float, gd.device),
            gpu_local_transformer(), group=group)
        dom = dps.doms[0]
        phl = to_dev(phi0[dom.beg:dom.end])
        rhl = to_dev(rho[dom.beg:dom.end])
        err = [dps.iterate(phl, rhl) for _ in range(3)]
        return dom.beg, dom.end, to_np(phl), err

    for beg, end, got, err in LocalRanks(3).run(rank_body):
        assert np.array_equal(got, po.phis[0][beg:end]), (beg, end)
        for e, r in zip(err, ref_err):
            assert abs(e - r) <= 1e-12 * abs(r)


@pytest.mark.gpu
def test_slab_solve_emulated_ranks_against_oracle(cuda):
    """The solve loop of three emulated slab ranks on one GPU (a charged
    zero-boundary grid: Gaussian monopole removal on every slab) against
    the oracle's whole-grid solve: the same V-cycle count, phi to 1e-11."""
    from gpaw_b200 import FDPoissonSolver, GridDescriptor
    from gpaw_b200.domains import (DistributedFDPoissonSolver, LocalRanks,
                                   gpu_local_operator, gpu_local_transformer)
    from oracle import gpaw_layer as L
    from tests.helpers import to_dev, to_np
    N, cell, pbc = (32, 24, 24), (6.0, 4.5, 4.5), (0, 0, 0)
    gdo = L.GridDescriptor(N, cell, pbc)
    rng = np.random.default_rng(23)
    rho = rng.standard_normal(tuple(gdo.n_c))
    po = L.FDPoissonSolver(nn=3, relax='J', eps=1e-8)
    po.set_grid_descriptor(gdo)
    ref = np.zeros(tuple(gdo.n_c))
    n_ref = po.solve(ref, rho)
    gd = GridDescriptor(N, cell, pbc)
    ps = FDPoissonSolver(nn=3, relax='J', eps=1e-8)
    ps.set_grid_descriptor(gd)

    def rank_body(rank, group):
        dps = DistributedFDPoissonSolver(
            ps, rank, 3, gpu_local_operator(float, gd.device),
            gpu_local_transformer(), group=group)
        dom = dps.doms[0]
        phl = to_dev(np.zeros(dom.local_shape()))
        n = dps.solve(phl, to_dev(rho[dom.beg:dom.end]),
                      gauss=L.gauss_l0(gdo))
        return dom.beg, dom.end, to_np(phl), n

    for beg, end, got, n in LocalRanks(3).run(rank_body):
        assert n == n_ref
        assert np.abs(got - ref[beg:end]).max() <= 1e-11 * np.abs(ref).max()
