"""Domain decomposition of one grid over gloo ranks on the host (2 to 5
ranks): slabs along axis 0 and boxes of 2-D and 3-D process grids.  The
halo exchange (Bloch phases across periodic edges), stencils, weighted
operators, restriction and interpolation, the plain and dielectric FD
Poisson V-cycles and solves, and the preconditioner, each against the
same computation on the whole grid.  The local operators here are the
oracle's CPU ones; on GPUs the boxes run the library's kernels and the
exchange goes over NCCL (one GPU per process; not run here, where a call
has one GPU)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from gpaw_b200.domains import SlabDomain, slab_bounds


def test_slab_bounds_cover_axis():
    for n0, size in ((10, 3), (7, 7), (64, 5)):
        b = slab_bounds(n0, size)
        assert b[0][0] == 0 and b[-1][1] == n0
        assert all(b[k][1] == b[k + 1][0] for k in range(size - 1))
        sizes = [e - s for s, e in b]
        assert max(sizes) - min(sizes) <= 1


def test_neighbours():
    d = SlabDomain((9, 4, 4), True, 0, 3)
    assert (d.lower, d.upper) == (2, 1)
    d = SlabDomain((9, 4, 4), False, 2, 3)
    assert (d.lower, d.upper) == (1, None)


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _OracleLocal:
    """The oracle's apply and relax on host tensors (the slab plus
    halos)."""

    def __init__(self, coef_p, offset_pc, n_c, pbc_c, dtype=complex):
        from oracle import gpaw_layer as L
        self.gd = L.GridDescriptor(_N_for(n_c, pbc_c), (1.0, 1.0, 1.0),
                                   pbc_c)
        self.dtype = dtype
        self.op = L.FDOperator(coef_p, offset_pc, self.gd, dtype, be='port')

    def apply(self, a, out, phase_cd=None):
        b = np.zeros(tuple(a.shape), self.dtype)
        self.op.apply(a.numpy().astype(self.dtype), b, phase_cd)
        out.copy_(torch.from_numpy(b))

    def relax(self, method, f, s, n, w=None):
        g = f.numpy().copy()
        self.op.relax(method, g, s.numpy(), n, w)
        f.copy_(torch.from_numpy(g))


def _N_for(n_c, pbc_c):
    return tuple(n + (0 if p else 1) for n, p in zip(n_c, pbc_c))


def _worker(rank, world, port, pbc0, q):
    import torch.distributed as dist

    from gpaw_b200.domains import DistributedFDOperator
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        pbc = (pbc0, 1, 0)
        N = (14, 10, 12)
        gd = L.GridDescriptor(N, (3.0, 2.5, 3.2), pbc)
        ph = gd.phase_factor_cd((0.3, -0.2, 0.0))
        rng = np.random.default_rng(7)
        a = rng.standard_normal(tuple(gd.n_c)) + \
            1j * rng.standard_normal(tuple(gd.n_c))
        lap = L.Laplace(gd, -0.5, 3, complex, be='port')
        ref = np.zeros_like(a)
        lap.apply(a, ref, ph)
        dom = SlabDomain(gd.n_c, pbc0, rank, world)
        op = DistributedFDOperator(lap.coef_p, lap.offset_pc, gd, dom,
                                   _OracleLocal)
        loc = torch.from_numpy(a[dom.beg:dom.end].copy())
        out = torch.zeros_like(loc)
        op.apply(loc, out, ph)
        got = out.numpy()
        q.put((rank, float(np.abs(got - ref[dom.beg:dom.end]).max()),
               float(np.abs(ref).max())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 3, 5])
@pytest.mark.parametrize('pbc0', [1, 0])
def test_slab_apply_equals_whole_grid(world, pbc0):
    """Complex apply with Bloch phases on slabs: the planes that cross the
    periodic edge take the phase with the reference's complex grouping, so
    every rank's planes equal the whole grid's exactly.  On five ranks the
    slabs of 14 planes (3 or 2 each) are thinner than the stencil's range
    R = 3 on some ranks, whose halos then come partly from ranks two
    away."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, pbc0, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err, scale in res:
        assert err == 0.0, (rank, err)


@pytest.mark.gpu
def test_single_slab_on_gpu_equals_plain_apply(cuda):
    """One rank (no process group): the slab path with the library's
    kernels on a periodic complex grid equals the plain apply to 1e-12 (the
    axis-0 halo's phase is a device complex multiply)."""
    from gpaw_b200 import GridDescriptor, Laplace
    from gpaw_b200.domains import (DistributedFDOperator, SlabDomain,
                                   gpu_local_operator)
    from tests.helpers import max_rel, to_dev, to_np
    gd = GridDescriptor((16, 12, 20), (3.0, 2.4, 4.0), True)
    ph = gd.phase_factor_cd((0.3, -0.2, 0.1))
    rng = np.random.default_rng(3)
    a = rng.standard_normal((2,) + tuple(gd.n_c)) + \
        1j * rng.standard_normal((2,) + tuple(gd.n_c))
    lap = Laplace(gd, -0.5, 3, complex)
    x = to_dev(a)
    ref = x.new_zeros(x.shape)
    lap.apply(x, ref, ph)
    dom = SlabDomain(gd.n_c, True, 0, 1)
    op = DistributedFDOperator(lap.coef_p, lap.offset_pc, gd, dom,
                               gpu_local_operator(complex, x.device))
    out = x.new_zeros(x.shape)
    op.apply(x, out, ph)
    assert max_rel(to_np(out), to_np(ref)) <= 1e-12


def _relax_worker(rank, world, port, q):
    import torch.distributed as dist

    from gpaw_b200.domains import DistributedFDOperator
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        gd = L.GridDescriptor((16, 12, 10), (4.0, 3.0, 2.5), (0, 0, 1))
        rng = np.random.default_rng(11)
        f = rng.standard_normal(tuple(gd.n_c))
        s = rng.standard_normal(tuple(gd.n_c))
        lap = L.Laplace(gd, -0.25 / np.pi, 3, be='port')
        ref = f.copy()
        lap.relax(2, ref, s, 3, 2.0 / 3.0)
        r = np.zeros_like(ref)
        lap.apply(ref, r)
        r -= s
        norm_ref = float((r * r).sum()) * gd.dv
        dom = SlabDomain(gd.n_c, False, rank, world)
        op = DistributedFDOperator(
            lap.coef_p, lap.offset_pc, gd, dom,
            lambda c, o, n, p: _OracleLocal(c, o, n, p, float))
        fl = torch.from_numpy(f[dom.beg:dom.end].copy())
        sl = torch.from_numpy(s[dom.beg:dom.end].copy())
        op.relax(2, fl, sl, 3, 2.0 / 3.0)
        norm = op.residual_norm2(fl, sl, gd.dv)
        q.put((rank, bool(np.array_equal(fl.numpy(), ref[dom.beg:dom.end])),
               norm, norm_ref))
    finally:
        dist.destroy_process_group()


def test_slab_jacobi_and_norm_equal_whole_grid():
    """Three Jacobi sweeps on three slabs (halos exchanged before each) are
    bit-identical to the sweeps on the whole grid; the residual norm summed
    over the ranks matches the whole grid's to rounding."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    world = 3
    procs = [ctx.Process(target=_relax_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, same, norm, norm_ref in res:
        assert same, rank
        assert abs(norm - norm_ref) <= 1e-12 * norm_ref


@pytest.mark.gpu
def test_single_slab_jacobi_on_gpu(cuda):
    """One rank, zero boundary along axis 0: Jacobi sweeps on the slab
    plus (zero) halos with the library's kernels equal the plain relax bit
    for bit."""
    from gpaw_b200 import GridDescriptor, Laplace
    from gpaw_b200.domains import (DistributedFDOperator, SlabDomain,
                                   gpu_local_operator)
    from tests.helpers import to_dev, to_np
    gd = GridDescriptor((20, 16, 12), (4.0, 3.2, 2.4), (0, 1, 0))
    rng = np.random.default_rng(5)
    f = rng.standard_normal(tuple(gd.n_c))
    s = rng.standard_normal(tuple(gd.n_c))
    lap = Laplace(gd, -0.25 / np.pi, 3)
    ref = to_dev(f)
    lap.relax(2, ref, to_dev(s), 3, 2.0 / 3.0)
    dom = SlabDomain(gd.n_c, False, 0, 1)
    op = DistributedFDOperator(lap.coef_p, lap.offset_pc, gd, dom,
                               gpu_local_operator(float, ref.device))
    fd = to_dev(f)
    op.relax(2, fd, to_dev(s), 3, 2.0 / 3.0)
    assert np.array_equal(to_np(fd), to_np(ref))


def _run_ranks(world, target, args=()):
    """Run ``target(rank, world, port, q, *args)`` on ``world`` spawned gloo
    ranks; every rank puts one result (or ('error', traceback)) on q."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q) + args)
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    errors = [r[1] for r in res if r[0] == 'error']
    assert not errors, errors[0]
    assert all(p.exitcode == 0 for p in procs)
    return res


class _OracleTransfer:
    """The oracle's Transformer of one rank, on host tensors."""

    def __init__(self, size_in, size_out, k, pads, npads, skip, nb, real,
                 interpolate):
        from oracle import port
        self.t = port.Transformer(size_in, size_out, k, pads, npads, skip,
                                  nb, real, None, interpolate)
        self.dtype = float if real else complex

    def apply(self, a, out, phases=None):
        b = np.zeros(tuple(out.shape), self.dtype)
        self.t.apply(a.numpy().astype(self.dtype), b, phases)
        out.copy_(torch.from_numpy(b))


def _transfer_worker(rank, world, port, q):
    import traceback

    import torch.distributed as dist

    from gpaw_b200.domains import DistributedTransformer
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        worst = []
        for pbc0 in (1, 0):
            gd = L.GridDescriptor((26, 12, 10), (5.2, 2.4, 2.0),
                                  (pbc0, 1, 0))
            gd2 = gd.coarsen()
            ph = gd.phase_factor_cd((0.3, -0.2, 0.0))
            for dtype in (float, complex):
                for nn in (1, 3):
                    for interp in (False, True):
                        gi, go = (gd2, gd) if interp else (gd, gd2)
                        for rep_in, rep_out in ((0, 0), (0, 1), (1, 0)):
                            rng = np.random.default_rng(nn + 2 * pbc0)
                            a = rng.standard_normal((2,) + tuple(gi.n_c))
                            if dtype == complex:
                                a = a + 1j * rng.standard_normal(a.shape)
                            phases = ph if dtype == complex else None
                            ref = np.zeros((2,) + tuple(go.n_c), dtype)
                            L.Transformer(gi, go, nn, dtype, be='port') \
                                .apply(a, ref, phases)
                            di = SlabDomain(gi.n_c, pbc0, rank, world,
                                            bool(rep_in))
                            do = SlabDomain(go.n_c, pbc0, rank, world,
                                            bool(rep_out))
                            t = DistributedTransformer(gi, go, nn, dtype,
                                                       di, do,
                                                       _OracleTransfer)
                            loc = torch.from_numpy(
                                a[:, di.beg:di.end].copy())
                            out = torch.zeros((2,) + do.local_shape(),
                                              dtype=loc.dtype)
                            t.apply(loc, out, phases)
                            same = np.array_equal(out.numpy(),
                                                  ref[:, do.beg:do.end])
                            worst.append(((pbc0, dtype.__name__, nn,
                                           interp, rep_in, rep_out), same))
        q.put((rank, worst))
    except Exception:
        q.put(('error', traceback.format_exc()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 3])
def test_slab_transfers_equal_whole_grid(world):
    """Restriction and interpolation (nn = 1 and 3; real, and complex with
    Bloch phases; periodic and zero axis 0; split or replicated input and
    output) on gloo ranks give each rank exactly the planes the whole-grid
    transformer gives.  26 planes over 2 or 3 ranks: slabs of odd and even
    length that start on odd and even points."""
    for rank, cases in _run_ranks(world, _transfer_worker):
        bad = [c for c, same in cases if not same]
        assert not bad, (rank, bad)


def _vcycle_worker(rank, world, port, q, pbc0):
    import traceback

    import torch.distributed as dist

    from gpaw_b200.domains import DistributedFDPoissonSolver
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        gd = L.GridDescriptor((24, 16, 16), (6.0, 4.0, 4.4), (pbc0, 1, 0))
        rng = np.random.default_rng(17)
        rho = rng.standard_normal(tuple(gd.n_c))
        phi = rng.standard_normal(tuple(gd.n_c)) * 0.1
        ps = L.FDPoissonSolver(nn=3, relax='J', be='port')
        ps.set_grid_descriptor(gd)
        ps._init()
        ps.phis[0] = phi.copy()
        ps.rhos[0][:] = rho
        ps.errors = []
        ref_err = [ps.iterate2(ps.step) for _ in range(3)]
        dps = DistributedFDPoissonSolver(
            ps, rank, world,
            lambda c, o, n, p: _OracleLocal(c, o, n, p, float),
            _OracleTransfer)
        dom = dps.doms[0]
        phl = torch.from_numpy(phi[dom.beg:dom.end].copy())
        rhl = torch.from_numpy(rho[dom.beg:dom.end].copy())
        err = [dps.iterate(phl, rhl) for _ in range(3)]
        q.put((rank, bool(np.array_equal(phl.numpy(),
                                          ps.phis[0][dom.beg:dom.end])),
               err, ref_err, dps.split_levels, dps.levels))
    except Exception:
        q.put(('error', traceback.format_exc()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 3])
@pytest.mark.parametrize('pbc0', [1, 0])
def test_slab_vcycles_equal_whole_grid(world, pbc0):
    """Three FD Poisson V-cycles (nn = 3, Jacobi, 4 levels) on slabs, with
    the thin coarse levels gathered whole on every rank, leave every rank's
    slab of phi bit-identical to the whole-grid V-cycles; the level-0
    error summed over the ranks matches to rounding."""
    res = _run_ranks(world, _vcycle_worker, (pbc0,))
    for rank, same, err, ref_err, split, levels in res:
        assert same, rank
        assert 1 <= split <= levels
        for e, r in zip(err, ref_err):
            assert abs(e - r) <= 1e-12 * abs(r)
    # some level below the finest is gathered whole in these cases
    assert any(split < levels + 1 for _, _, _, _, split, levels in res)


def _solve_worker(rank, world, port, q, case):
    import traceback

    import torch.distributed as dist

    from gpaw_b200.domains import DistributedFDPoissonSolver
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        pbc, nn = case
        gd = L.GridDescriptor((16, 12, 12), (4.0, 3.0, 3.3), pbc)
        rng = np.random.default_rng(23)
        rho = rng.standard_normal(tuple(gd.n_c))
        if any(pbc) and not all(pbc):
            rho -= rho.mean()          # mixed boundaries: neutral only
        ps = L.FDPoissonSolver(nn=nn, relax='J', eps=1e-8, be='port')
        ps.set_grid_descriptor(gd)
        ref = np.zeros(tuple(gd.n_c))
        niter_ref = ps.solve(ref, rho)
        dps = DistributedFDPoissonSolver(
            ps, rank, world,
            lambda c, o, n, p: _OracleLocal(c, o, n, p, float),
            _OracleTransfer)
        dom = dps.doms[0]
        phl = torch.zeros(dom.local_shape(), dtype=torch.float64)
        rhl = torch.from_numpy(rho[dom.beg:dom.end].copy())
        gauss = None if any(pbc) else L.gauss_l0(gd)
        niter = dps.solve(phl, rhl, gauss=gauss)
        err = float(np.abs(phl.numpy() - ref[dom.beg:dom.end]).max())
        q.put((rank, niter, niter_ref, err, float(np.abs(ref).max())))
    except Exception:
        q.put(('error', traceback.format_exc()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('case', [((1, 1, 1), 3), ((0, 1, 0), 3),
                                  ((0, 0, 0), 3), ((1, 1, 1), 'M')])
def test_slab_solve_equals_whole_grid(case):
    """The solve loop on three slabs -- a charged periodic grid (the
    background from the charge summed over the ranks), a neutral
    mixed-boundary grid, a charged zero-boundary grid (Gaussian monopole
    removal), the Mehrstellen stencil (B rho on slabs) -- takes as many
    V-cycles as the whole-grid solve and gives phi to 1e-11 (sums over
    ranks round differently)."""
    for rank, niter, niter_ref, err, scale in _run_ranks(3, _solve_worker,
                                                          (case,)):
        assert niter == niter_ref, rank
        assert err <= 1e-11 * scale, (rank, err)


def _precond_worker(rank, world, port, q, pbc0):
    import traceback

    import torch.distributed as dist

    from gpaw_b200.domains import DistributedPreconditioner
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        gd = L.GridDescriptor((24, 16, 12), (4.8, 3.2, 2.4), (pbc0, 1, 1))
        ph = gd.phase_factor_cd((0.25, -0.1, 0.2))
        rng = np.random.default_rng(29)
        res = rng.standard_normal((2,) + tuple(gd.n_c)) + \
            1j * rng.standard_normal((2,) + tuple(gd.n_c))
        kin0 = L.Laplace(gd, -0.5, 3, complex, be='port')
        pre = L.Preconditioner(gd, kin0, complex, block=2, be='port')
        ref = pre(res, ph).copy()
        dp = DistributedPreconditioner(
            pre, rank, world,
            lambda c, o, n, p: _OracleLocal(c, o, n, p, complex),
            _OracleTransfer)
        dom = dp.doms[0]
        got = dp(torch.from_numpy(res[:, dom.beg:dom.end].copy()), ph)
        q.put((rank, bool(np.array_equal(got.numpy(),
                                          ref[:, dom.beg:dom.end])),
               [d.replicated for d in dp.doms]))
    except Exception:
        q.put(('error', traceback.format_exc()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('pbc0', [1, 0])
def test_slab_preconditioner_equals_whole_grid(pbc0):
    """The three-level preconditioner on three slabs (complex, Bloch
    phases, two residuals; with a zero axis 0 the coarsest level is held
    whole on every rank) gives each rank exactly the planes of the
    whole-grid preconditioner."""
    res = _run_ranks(3, _precond_worker, (pbc0,))
    for rank, same, rep in res:
        assert same, (rank, rep)
    assert res[0][2][2] == (not pbc0)


class _OracleWeighted:
    """The oracle's WOperator of one slab plus halos, on host tensors."""

    def __init__(self, nw, weights, coef_ps, offset_ps, n_c, r, nb, real,
                 cfd):
        from oracle import port
        self.op = port.WOperator(nw, [w.numpy() for w in weights], coef_ps,
                                 offset_ps, n_c, r, nb, real, None, cfd)

    def apply(self, a, out, phases=None):
        b = np.zeros(tuple(out.shape))
        self.op.apply(a.numpy(), b, phases)
        out.copy_(torch.from_numpy(b))

    def relax(self, method, f, s, n, w=None):
        g = f.numpy().copy()
        self.op.relax(method, g, s.numpy(), n, 1.0 if w is None else w)
        f.copy_(torch.from_numpy(g))


_D1 = {1: [1 / 2], 2: [2 / 3, -1 / 12], 3: [3 / 4, -3 / 20, 1 / 60]}


def _grad_stencils(gd, scale, n):
    """The Laplacian and three central first derivatives of range n on an
    orthogonal cell, scaled, as (coefs, offsets) pairs."""
    from oracle import gpaw_layer as L
    lap = L.Laplace(gd, scale, n, be='port')
    out = [(lap.coef_p, lap.offset_pc)]
    for c in range(3):
        h = gd.cell_cv[c, c] / gd.N_c[c]
        e = np.zeros(3, int)
        e[c] = 1
        offs = [j * e for j in range(1, n + 1)] + \
            [-j * e for j in range(1, n + 1)]
        a = [scale * d / h for d in _D1[n]]
        out.append((np.array(a + [-x for x in a]), np.array(offs)))
    return out


def _weighted_worker(rank, world, port, q, pbc0, dims=None):
    import traceback

    import torch.distributed as dist

    from gpaw_b200.domains import DistributedWeightedFDPoissonSolver
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        gd = L.GridDescriptor((24, 16, 16), (6.0, 4.0, 4.0), (pbc0, 0, 0))
        x = gd.get_grid_point_coordinates() - \
            np.array([3.0, 2.0, 2.0])[:, None, None, None]
        g = np.exp(-(x**2).sum(0) / 2.0)
        arrays = [80.0 - 79.0 * g] + [79.0 * g * x[c] for c in range(3)]
        # d eps / dx_c = 79 g x_c
        rho = np.exp(-((x[0] - 0.5)**2 + x[1]**2 + x[2]**2)) - \
            np.exp(-((x[0] + 0.5)**2 + x[1]**2 + x[2]**2))
        rng = np.random.default_rng(31)
        phi = rng.standard_normal(tuple(gd.n_c)) * 0.01
        wps = L.WeightedFDPoissonSolver(_grad_stencils, nn=3, be='port')
        wps.set_grid_descriptor(gd)
        wps.set_dielectric(arrays)
        wps.restrict_op_weights()
        wps.phis[0] = phi.copy()
        wps.rhos[0][:] = rho
        wps.errors = []
        ref_err = [wps.iterate2(wps.step) for _ in range(3)]
        from gpaw_b200.domains import make_domain
        d = make_domain(gd.n_c, gd.pbc_c, rank, world, dims)

        def cut(a):
            return torch.from_numpy(np.ascontiguousarray(d.inner(a)))
        dps = DistributedWeightedFDPoissonSolver(
            wps, [cut(a) for a in arrays], rank, world, _OracleWeighted,
            _OracleTransfer, dims=dims)
        phl = cut(phi)
        rhl = cut(rho)
        err = [dps.iterate(phl, rhl) for _ in range(3)]
        same = bool(np.array_equal(phl.numpy(), d.inner(wps.phis[0])))
        # a charged system: the dielectric's compensation charge
        rho_c = rho + 0.5 * np.exp(-(x**2).sum(0)) if not pbc0 else \
            rho - rho.mean()
        wps.eps = dps.ps.eps = 1e-8
        ref_phi = np.zeros(tuple(gd.n_c))
        n_ref = wps.solve(ref_phi, rho_c)
        phc = torch.zeros(phl.shape, dtype=torch.float64)
        n = dps.solve(phc, cut(rho_c), gauss=(wps.rho_gauss, wps.phi_gauss))
        charged = (n, n_ref,
                   float(np.abs(phc.numpy() - d.inner(ref_phi)).max()),
                   float(np.abs(ref_phi).max()))
        q.put((rank, same, err, ref_err, dps.split_levels, dps.levels,
               charged))
    except Exception:
        q.put(('error', traceback.format_exc()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('pbc0,dims', [(1, None), (0, None), (1, (2, 2)),
                                       (0, (1, 3)), (0, (1, 1, 3))])
def test_slab_weighted_vcycles_equal_whole_grid(pbc0, dims):
    """The dielectric Poisson solver's V-cycles on three slabs, or on the
    boxes of a 2 x 2, 1 x 3 or 1 x 1 x 3 process grid (weights and their
    halos split, coarse weights restricted on the split grid, the
    flattened stencil offsets re-flattened for a split axis 1 or 2) leave
    phi bit-identical to the whole grid's; the level-0 error matches to
    rounding.  A charged system (the dielectric's compensation charge in a
    zero-boundary cell; the neutral part of it on a periodic axis 0) takes
    as many V-cycles as the whole-grid solve, phi to 1e-11."""
    world = 3 if dims is None else int(np.prod(dims))
    for rank, same, err, ref_err, split, levels, charged in _run_ranks(
            world, _weighted_worker, (pbc0, dims)):
        assert same, rank
        assert split <= levels
        for e, r in zip(err, ref_err):
            assert abs(e - r) <= 1e-12 * abs(r)
        n, n_ref, d, scale = charged
        assert n == n_ref, rank
        assert d <= 1e-11 * scale, (rank, d)


# --------------------------------------------------------------------------
# boxes of a P0 x P1 process grid (axes 0 and 1 split)
# --------------------------------------------------------------------------
def _pencil_worker(rank, world, port, q, dims):
    """Apply (complex with Bloch phases: the Laplacian and the Mehrstellen
    stencil, whose edge taps read halo corners), restriction and
    interpolation, and three V-cycles on the boxes of ``dims``."""
    import traceback

    import torch.distributed as dist

    from gpaw_b200.domains import (DistributedFDOperator,
                                   DistributedFDPoissonSolver,
                                   DistributedPreconditioner,
                                   DistributedTransformer, make_domain)
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        out = {}

        def box(a, dom):
            return torch.from_numpy(np.ascontiguousarray(dom.inner(a)))

        def cut(a, dom):
            return dom.inner(a)
        for pbc in ((1, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1)):
            gd = L.GridDescriptor((24, 20, 12), (4.8, 4.0, 2.4), pbc)
            ph = gd.phase_factor_cd((0.3, -0.2, 0.1))
            rng = np.random.default_rng(41)
            a = rng.standard_normal((2,) + tuple(gd.n_c)) + \
                1j * rng.standard_normal((2,) + tuple(gd.n_c))
            dom = make_domain(gd.n_c, gd.pbc_c, rank, world, dims)
            for name, op in (('lap', L.Laplace(gd, -0.5, 3, complex,
                                               be='port')),
                             ('mehr', L.LaplaceA(gd, 0.5, complex,
                                                 be='port'))):
                ref = np.zeros_like(a)
                op.apply(a, ref, ph)
                dop = DistributedFDOperator(op.coef_p, op.offset_pc, gd, dom,
                                            _OracleLocal)
                got = torch.zeros((2,) + dom.local_shape(),
                                  dtype=torch.complex128)
                dop.apply(box(a, dom), got, ph)
                out[(pbc, name)] = bool(np.array_equal(got.numpy(),
                                                       cut(ref, dom)))
            gd2 = gd.coarsen()
            for nn in (1, 3):
                for interp in (False, True):
                    gi, go = (gd2, gd) if interp else (gd, gd2)
                    x = rng.standard_normal((2,) + tuple(gi.n_c)) + \
                        1j * rng.standard_normal((2,) + tuple(gi.n_c))
                    ref = np.zeros((2,) + tuple(go.n_c), complex)
                    L.Transformer(gi, go, nn, complex, be='port') \
                        .apply(x, ref, ph)
                    di = make_domain(gi.n_c, gi.pbc_c, rank, world, dims)
                    do = make_domain(go.n_c, go.pbc_c, rank, world, dims)
                    t = DistributedTransformer(gi, go, nn, complex, di, do,
                                               _OracleTransfer)
                    got = torch.zeros((2,) + do.local_shape(),
                                      dtype=torch.complex128)
                    t.apply(box(x, di), got, ph)
                    out[(pbc, nn, interp)] = bool(
                        np.array_equal(got.numpy(), cut(ref, do)))
        # V-cycles and the preconditioner
        gd = L.GridDescriptor((24, 16, 16), (6.0, 4.0, 4.4), (0, 1, 0))
        rng = np.random.default_rng(17)
        rho = rng.standard_normal(tuple(gd.n_c))
        phi = rng.standard_normal(tuple(gd.n_c)) * 0.1
        ps = L.FDPoissonSolver(nn=3, relax='J', be='port')
        ps.set_grid_descriptor(gd)
        ps._init()
        ps.phis[0] = phi.copy()
        ps.rhos[0][:] = rho
        ps.errors = []
        [ps.iterate2(ps.step) for _ in range(3)]
        dps = DistributedFDPoissonSolver(
            ps, rank, world,
            lambda c, o, n, p: _OracleLocal(c, o, n, p, float),
            _OracleTransfer, dims=dims)
        d0 = dps.doms[0]
        phl = box(phi, d0).clone()
        rhl = box(rho, d0)
        [dps.iterate(phl, rhl) for _ in range(3)]
        out['vcycle'] = bool(np.array_equal(phl.numpy(),
                                            cut(ps.phis[0], d0)))
        from gpaw_b200.domains import gather_full
        out['gather_full'] = bool(np.array_equal(
            gather_full(phl, d0).numpy(), ps.phis[0]))
        out['split_levels'] = dps.split_levels
        gdp = L.GridDescriptor((24, 16, 12), (4.8, 3.2, 2.4), (1, 1, 1))
        php = gdp.phase_factor_cd((0.25, -0.1, 0.2))
        res = rng.standard_normal((2,) + tuple(gdp.n_c)) + \
            1j * rng.standard_normal((2,) + tuple(gdp.n_c))
        kin0 = L.Laplace(gdp, -0.5, 3, complex, be='port')
        pre = L.Preconditioner(gdp, kin0, complex, block=2, be='port')
        ref = pre(res, php).copy()
        dp = DistributedPreconditioner(
            pre, rank, world,
            lambda c, o, n, p: _OracleLocal(c, o, n, p, complex),
            _OracleTransfer, dims=dims)
        got = dp(box(res, dp.doms[0]), php)
        out['precond'] = bool(np.array_equal(got.numpy(),
                                             cut(ref, dp.doms[0])))
        q.put((rank, out))
    except Exception:
        q.put(('error', traceback.format_exc()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('dims', [(2, 2), (1, 3), (2, 1, 2)])
def test_pencils_equal_whole_grid(dims):
    """Boxes of 2 x 2, 1 x 3 and 2 x 1 x 2 process grids: complex apply
    with Bloch phases (the Laplacian, and the Mehrstellen stencil whose
    edge taps read the halo edges and corners, phased axis by axis),
    restriction and interpolation (nn = 1 and 3), three V-cycles and the
    preconditioner all give every rank exactly the whole grid's points."""
    for rank, out in _run_ranks(int(np.prod(dims)), _pencil_worker,
                                (dims,)):
        bad = [k for k, v in out.items() if v is False]
        assert not bad, (rank, bad)
        assert out['split_levels'] >= 1


def test_box_pieces_cover_each_point_once():
    """For random process grids, grid sizes, boundary flags and needed
    boxes (reaching past either edge, wider than the grid): the pieces
    cover every point of the need that lies inside the grid or across a
    periodic edge exactly once, from a rank whose box holds it (the
    receiver itself when it does), with the right number of edge
    crossings; points past a zero boundary are left out."""
    import itertools

    from gpaw_b200.domains import GridDomain, box_pieces
    rng = np.random.default_rng(5)
    for _ in range(200):
        dims = tuple(int(x) for x in rng.integers(1, 4, 3))
        n = tuple(int(x) for x in rng.integers(1, 7, 3))
        per = tuple(bool(x) for x in rng.integers(0, 2, 3))
        dom = GridDomain(n, per, 0, dims, bool(rng.integers(4) == 0))
        recv = int(rng.integers(dom.size))
        need = []
        for nc in n:
            lo = int(rng.integers(-2 * nc - 2, nc + 1))
            need.append((lo, lo + int(rng.integers(0, 3 * nc + 3))))
        hits = {}
        for owner, src, dst, ln, k in box_pieces(need, n, per, dom.boxes,
                                                 recv):
            box = dom.boxes[owner]
            for c in range(3):
                assert 0 <= src[c] and src[c] + ln[c] <= box[c][1] - box[c][0]
            for idx in itertools.product(*[range(m) for m in ln]):
                g = tuple(need[c][0] + dst[c] + idx[c] for c in range(3))
                assert g not in hits
                hits[g] = (owner, tuple(box[c][0] + src[c] + idx[c]
                                        for c in range(3)), k)
        for g in itertools.product(*[range(*nd) for nd in need]):
            kp = [divmod(g[c], n[c]) for c in range(3)]
            inside = all(per[c] or kp[c][0] == 0 for c in range(3))
            assert (g in hits) == inside
            if not inside:
                continue
            owner, q, k = hits[g]
            assert q == tuple(p for _, p in kp)
            assert k == tuple(kk for kk, _ in kp)
            if all(b <= p < e for (_, p), (b, e) in
                   zip(kp, dom.boxes[recv])):
                assert owner == recv


def test_domain_errors():
    """A process grid that does not make the rank count, a finest grid too
    thin for its stencil, and Gauss-Seidel on a split grid are refused."""
    from gpaw_b200.domains import (DistributedFDOperator,
                                   DistributedFDPoissonSolver, make_domain)
    from oracle import gpaw_layer as L
    with pytest.raises(ValueError):
        make_domain((8, 8, 8), (1, 1, 1), 0, 4, dims=(2, 3))
    gd = L.GridDescriptor((8, 8, 8), (2.0, 2.0, 2.0), (1, 1, 1))
    ps = L.FDPoissonSolver(nn=3, relax='J', be='port')
    ps.set_grid_descriptor(gd)
    with pytest.raises(ValueError):
        DistributedFDPoissonSolver(ps, 0, 4, None, None)  # 2 planes < R = 3
    ps_gs = L.FDPoissonSolver(nn=3, relax='GS', be='port')
    ps_gs.set_grid_descriptor(gd)
    with pytest.raises(NotImplementedError):
        DistributedFDPoissonSolver(ps_gs, 0, 2, None, None)
    lap = L.Laplace(gd, -0.5, 1, be='port')
    dom = make_domain(gd.n_c, gd.pbc_c, 0, 1)
    op = DistributedFDOperator(lap.coef_p, lap.offset_pc, gd, dom,
                               lambda c, o, n, p: _OracleLocal(c, o, n, p,
                                                               float))
    f = torch.zeros(dom.local_shape(), dtype=torch.float64)
    with pytest.raises(NotImplementedError):
        op.relax(1, f, f.clone(), 1)


def _asym_worker(rank, world, port, q):
    import traceback

    import torch.distributed as dist

    from gpaw_b200 import GridDescriptor
    from gpaw_b200 import multipole as M
    from gpaw_b200.domains import DistributedFDPoissonSolver
    from gpaw_b200.gauss import monopole_gaussian
    from oracle import gpaw_layer as L
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        a, N = 20.0, 48
        c0 = np.array((a / 2, a / 2, 3 * a / 4))
        gd = L.GridDescriptor((N, N, N), (a, a, a), 0)
        pgd = GridDescriptor((N, N, N), (a, a, a), False, device='cpu')
        g = M.Gaussian(pgd, a=19, center=c0)
        ng, vg = g.get_gauss(0), g.get_gauss_pot(0)
        ps = L.FDPoissonSolver(nn=3, relax='J', be='port')
        ps.set_grid_descriptor(gd)
        dps = DistributedFDPoissonSolver(
            ps, rank, world,
            lambda c, o, n, p: _OracleLocal(c, o, n, p, float),
            _OracleTransfer)
        dom = dps.doms[0]
        pot = torch.zeros(dom.local_shape(), dtype=torch.float64)
        dps.solve(pot, torch.from_numpy(np.ascontiguousarray(dom.inner(ng))),
                  charge=1.0, use_charge_center=True,
                  gauss=lambda c: monopole_gaussian(pgd, center=c))
        t = torch.tensor([float(((pot.numpy() - dom.inner(vg))**2).sum())])
        dist.all_reduce(t)
        q.put((rank, float(t[0]) * gd.dv))
    except Exception:
        q.put(('error', traceback.format_exc()))
    finally:
        dist.destroy_process_group()


def test_charge_center_solve_reference_known_answer():
    """gpaw/test/poisson/test_poisson_asym.py:9-41 on two slabs: a unit
    Gaussian centred at (a/2, a/2, 3a/4) in a 20 Bohr zero-boundary cell
    (48^3, nn = 3), solved as a charged system with the Gaussian placed on
    the centre of charge (found from sums over the ranks), gives its
    analytic potential to a residual below 1e-5."""
    from gpaw_b200 import GridDescriptor
    from gpaw_b200 import multipole as M
    from gpaw_b200.gauss import charge_center, charge_center_parts
    for rank, res2 in _run_ranks(2, _asym_worker):
        assert res2**0.5 < 1e-5, (rank, res2**0.5)
    # the centre of charge of that Gaussian is where it was put
    pgd = GridDescriptor((48, 48, 48), (20.0, 20.0, 20.0), False,
                         device='cpu')
    c0 = np.array((10.0, 10.0, 15.0))
    ng = M.Gaussian(pgd, a=19, center=c0).get_gauss(0)
    center = charge_center(pgd, *charge_center_parts(pgd, ng, 1.0))
    assert np.abs(center - c0).max() < 1e-6
    with pytest.raises(RuntimeError):      # within 7 spacings of a face
        ng = M.Gaussian(pgd, a=19, center=np.array((10.0, 10.0, 1.5)))
        charge_center(pgd, *charge_center_parts(pgd, ng.get_gauss(0),
                                                1.0))


def test_local_ranks_vcycles_equal_whole_grid():
    """The in-process rank emulation (LocalRanks) runs the slab V-cycles of
    three ranks as threads with the oracle's local operators: every slab of
    phi equals the whole-grid V-cycles bit for bit, as over gloo."""
    from gpaw_b200.domains import DistributedFDPoissonSolver, LocalRanks
    from oracle import gpaw_layer as L
    gd = L.GridDescriptor((24, 16, 16), (6.0, 4.0, 4.4), (1, 1, 0))
    rng = np.random.default_rng(17)
    rho = rng.standard_normal(tuple(gd.n_c))
    phi = rng.standard_normal(tuple(gd.n_c)) * 0.1
    ps = L.FDPoissonSolver(nn=3, relax='J', be='port')
    ps.set_grid_descriptor(gd)
    ps._init()
    ps.phis[0] = phi.copy()
    ps.rhos[0][:] = rho
    ps.errors = []
    ref_err = [ps.iterate2(ps.step) for _ in range(2)]

    def body(rank, group):
        dps = DistributedFDPoissonSolver(
            ps, rank, 3, lambda c, o, n, p: _OracleLocal(c, o, n, p, float),
            _OracleTransfer, group=group)
        dom = dps.doms[0]
        phl = torch.from_numpy(phi[dom.beg:dom.end].copy())
        rhl = torch.from_numpy(rho[dom.beg:dom.end].copy())
        err = [dps.iterate(phl, rhl) for _ in range(2)]
        return dom.beg, dom.end, phl.numpy(), err

    for beg, end, got, err in LocalRanks(3).run(body):
        assert np.array_equal(got, ps.phis[0][beg:end])
        for e, r in zip(err, ref_err):
            assert abs(e - r) <= 1e-12 * abs(r)
