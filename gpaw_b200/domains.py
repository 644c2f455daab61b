"""One grid split into slabs along axis 0 over the ranks of a process group
(the single-axis case of the reference's domain decomposition,
gpaw/old/domain.py and the halo exchange of c/bc.cpp:146-258).

Every rank owns a contiguous run of axis-0 planes.  Before a stencil is
applied, each rank receives the R planes on either side of its slab from
its neighbours (send/recv on the process group: NCCL across GPUs, gloo on
the host); across a periodic axis 0 the first and last ranks are
neighbours, and planes that cross that edge carry the Bloch phase of axis 0
(phase_cd[0][0] for planes from past the high edge, [0][1] from past the
low edge), as the reference's halo fill multiplies them.  The stencil then
runs on the local slab plus its halos as a grid whose axis 0 has a zero
boundary (only the halo planes' own outputs see that boundary, and they
are dropped), with the global grid's boundary conditions on axes 1 and 2.
"""
from __future__ import annotations

import numpy as np


def slab_bounds(n0, size):
    """(begin, end) of each rank's planes: sizes differ by at most one."""
    q, r = divmod(int(n0), int(size))
    beg = [k * q + min(k, r) for k in range(size)]
    end = [b + q + (k < r) for k, b in enumerate(beg)]
    return list(zip(beg, end))


class SlabDomain:
    """Rank ``rank`` of ``size`` owning planes [beg, end) of axis 0."""

    def __init__(self, n_c, periodic0, rank, size):
        self.n_c = tuple(int(x) for x in n_c)
        self.periodic0 = bool(periodic0)
        self.rank, self.size = int(rank), int(size)
        self.beg, self.end = slab_bounds(self.n_c[0], self.size)[self.rank]
        self.m0 = self.end - self.beg
        self.lower = self.rank - 1 if self.rank > 0 else \
            (self.size - 1 if self.periodic0 else None)
        self.upper = self.rank + 1 if self.rank < self.size - 1 else \
            (0 if self.periodic0 else None)

    def local_shape(self):
        return (self.m0,) + self.n_c[1:]


def exchange_halos(a, R, dom, phase_cd=None, group=None):
    """Local slab a (..., m0, n1, n2) -> (..., m0 + 2R, n1, n2) with the
    neighbours' planes (zeros past a zero boundary).  Works on torch
    tensors on any device the process group can send from."""
    import torch
    import torch.distributed as dist
    if dom.m0 < R:
        raise ValueError('every slab needs at least R = %d planes' % R)
    shape = a.shape[:-3] + (dom.m0 + 2 * R,) + a.shape[-2:]
    ext = a.new_zeros(shape)
    ext[..., R:R + dom.m0, :, :] = a
    lo_send = a[..., :R, :, :].contiguous()
    hi_send = a[..., dom.m0 - R:, :, :].contiguous()
    lo_recv = torch.zeros_like(lo_send)
    hi_recv = torch.zeros_like(hi_send)
    if dom.size == 1:
        if dom.periodic0:
            lo_recv.copy_(hi_send)
            hi_recv.copy_(lo_send)
    else:
        # sends: top planes up (tag 0), bottom planes down (tag 1); receives
        # in the matching order, so that two ranks that are each other's
        # upper and lower neighbour (two ranks, periodic) pair the messages
        # correctly on backends that match by order as well as by tag
        reqs = []
        if dom.upper is not None:
            reqs.append(dist.isend(hi_send, dom.upper, group, tag=0))
        if dom.lower is not None:
            reqs.append(dist.isend(lo_send, dom.lower, group, tag=1))
        if dom.lower is not None:
            reqs.append(dist.irecv(lo_recv, dom.lower, group, tag=0))
        if dom.upper is not None:
            reqs.append(dist.irecv(hi_recv, dom.upper, group, tag=1))
        for req in reqs:
            req.wait()
    if phase_cd is not None and a.is_complex():
        ph = np.asarray(phase_cd)
        if dom.rank == 0 and dom.periodic0:
            lo_recv = lo_recv * complex(ph[0][1])
        if dom.rank == dom.size - 1 and dom.periodic0:
            hi_recv = hi_recv * complex(ph[0][0])
    if dom.lower is not None:
        ext[..., :R, :, :] = lo_recv
    if dom.upper is not None:
        ext[..., R + dom.m0:, :, :] = hi_recv
    return ext


class DistributedFDOperator:
    """A stencil (coef_p, offset_pc) applied to a grid split in slabs.
    ``make_local(coef_p, offset_pc, n_c, pbc_c)`` builds the operator of
    one slab plus halos (``n_c`` points, zero boundary along axis 0): on a
    GPU an FDOperator of gpaw_b200; any object with
    ``apply(in, out, phase_cd)``."""

    def __init__(self, coef_p, offset_pc, gd, dom, make_local, group=None):
        offset_pc = np.asarray(offset_pc, int)
        self.R = int(np.abs(offset_pc[:, 0]).max()) if len(offset_pc) else 0
        self.dom, self.group = dom, group
        n_ext = (dom.m0 + 2 * self.R,) + tuple(int(x) for x in gd.n_c[1:])
        pbc = (False,) + tuple(bool(p) for p in gd.pbc_c[1:])
        self.local = make_local(coef_p, offset_pc, n_ext, pbc)

    def apply(self, a, out, phase_cd=None):
        R = self.R
        ext = exchange_halos(a, R, self.dom, phase_cd, self.group) if R \
            else a
        tmp = ext.new_zeros(ext.shape)
        ph = None
        if phase_cd is not None:
            ph = np.array(phase_cd, complex)
            ph[0] = 1.0              # axis 0 phases travelled with the halos
        self.local.apply(ext, tmp, ph)
        out[...] = tmp[..., R:R + self.dom.m0, :, :]

    def relax(self, relax_method, f, s, n, w=None):
        """Weighted Jacobi (method 2) on the split grid: before every sweep
        the halos of f are exchanged, the slab plus halos is swept once,
        and its interior kept -- the same sweeps as on the whole grid.
        Gauss-Seidel's lexicographic order does not split across slabs."""
        if relax_method != 2:
            raise NotImplementedError('only weighted Jacobi (2) runs on '
                                      'slabs')
        R = self.R
        s_ext = s.new_zeros(s.shape[:-3] + (self.dom.m0 + 2 * R,) +
                            s.shape[-2:])
        s_ext[..., R:R + self.dom.m0, :, :] = s
        for _ in range(n):
            ext = exchange_halos(f, R, self.dom, None, self.group)
            self.local.relax(2, ext, s_ext, 1, w)
            f[...] = ext[..., R:R + self.dom.m0, :, :]

    def residual_norm2(self, phi, rho, dv=1.0):
        """sum over the whole grid of (L phi - rho)^2 * dv, summed over the
        ranks (all ranks get it)."""
        import torch.distributed as dist
        r = phi.new_zeros(phi.shape)
        self.apply(phi, r)
        r -= rho
        t = (r * r).sum().reshape(1) * dv
        if self.dom.size > 1:
            dist.all_reduce(t, group=self.group)
        return float(t.item())


def gpu_local_operator(dtype=float, device=None):
    """``make_local`` for DistributedFDOperator on a GPU: an FDOperator of
    this library on the slab-plus-halo grid (the stencil is given, so the
    grid's cell does not matter)."""
    def make(coef_p, offset_pc, n_c, pbc_c):
        from .fd_operators import FDOperator
        from .grid_descriptor import GridDescriptor
        N = tuple(n + (0 if p else 1) for n, p in zip(n_c, pbc_c))
        gd = GridDescriptor(N, (1.0, 1.0, 1.0), pbc_c, device=device)
        return FDOperator(coef_p, offset_pc, gd, dtype)
    return make
