"""Slab decomposition of one grid along axis 0 over gloo ranks on the host
(world sizes 2 and 3): the halo exchange, with the Bloch phase of axis 0
across a periodic edge, and a stencil applied slab by slab equal to the
same stencil on the whole grid.  The local operator here is the oracle's
CPU apply; on GPUs the slabs run the library's kernels and the exchange
goes over NCCL (one GPU per process; not run here, where a call has one
GPU)."""
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


@pytest.mark.parametrize('world', [2, 3])
@pytest.mark.parametrize('pbc0', [1, 0])
def test_slab_apply_equals_whole_grid(world, pbc0):
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
        assert err <= 1e-12 * scale, (rank, err)


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
