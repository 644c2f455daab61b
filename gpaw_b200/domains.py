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

Restriction and interpolation gather the input planes each rank's output
reaches (``gather_planes``), and the FD Poisson V-cycle runs on slabs down
to the levels too thin to split, which every rank then holds whole.

Axes 1 and 2 can be split too (``GridDomain``: boxes of a P0 x P1 x P2
process grid); the same gathers then run over boxes (``gather_box``),
points past several periodic edges taking the phases axis by axis in
order.
"""
from __future__ import annotations

import collections
import functools
import threading

import numpy as np


# --------------------------------------------------------------------------
# transports: a torch.distributed group, or ranks emulated in one process
# --------------------------------------------------------------------------
class LocalRanks:
    """Stand-in for a process group: ``size`` ranks run as threads of one
    process and exchange tensors through in-memory mailboxes, with the
    same messages in the same order as over torch.distributed.  It lets a
    decomposition run on one device (all ranks' slabs on one GPU), for
    tests and debugging: ``LocalRanks(3).run(lambda rank, group: ...)``.

    Point-to-point messages are matched by (source, destination, tag) and
    a per-pair sequence number, so successive collectives do not mix; sums
    over the ranks add the ranks' tensors in rank order (deterministic).
    GPU work stays ordered because every thread enqueues on the device's
    default stream."""

    def __init__(self, size):
        self.size = int(size)
        self._cv = threading.Condition()
        self._mail = {}
        self._barrier = threading.Barrier(self.size)
        self._slots = [None] * self.size
        self._local = threading.local()

    # per-thread state: the rank and its message counters
    def _rank(self):
        return self._local.rank

    def _next(self, key):
        cnt = self._local.counts
        cnt[key] += 1
        return cnt[key]

    def exchange(self, sends, recvs):
        """sends: [(dst, tag, tensor)], recvs: [(src, tag, buffer)];
        returns when every buffer is filled."""
        me = self._rank()
        with self._cv:
            for dst, tag, t in sends:
                key = ('s', me, dst, tag)
                # a copy taken now: the sender goes on writing its arrays
                self._mail[(me, dst, tag, self._next(key))] = t.clone()
            self._cv.notify_all()
        for src, tag, buf in recvs:
            k = (src, me, tag, self._next(('r', src, me, tag)))
            with self._cv:
                ok = self._cv.wait_for(lambda: k in self._mail, timeout=120)
                if not ok:
                    raise RuntimeError(f'LocalRanks: rank {me} got no message '
                                       f'{k} in 120 s')
                t = self._mail.pop(k)
            buf.copy_(t)

    def all_reduce_sum(self, t):
        me = self._rank()
        self._slots[me] = t.clone()
        self._barrier.wait(timeout=120)
        total = self._slots[0].clone()
        for r in range(1, self.size):
            total += self._slots[r]
        self._barrier.wait(timeout=120)
        t.copy_(total)

    def run(self, fn):
        """fn(rank, group) on every rank, each in its own thread; returns
        the list of results in rank order and re-raises the first error."""
        results = [None] * self.size
        errors = []

        def body(rank):
            self._local.rank = rank
            self._local.counts = collections.Counter()
            try:
                results[rank] = fn(rank, self)
            except BaseException as e:   # noqa: BLE001 (reported below)
                errors.append(e)
                self._barrier.abort()
                with self._cv:
                    self._cv.notify_all()

        threads = [threading.Thread(target=body, args=(r,))
                   for r in range(self.size)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        if errors:
            raise errors[0]
        return results


def _all_reduce_sum(t, group):
    if isinstance(group, LocalRanks):
        group.all_reduce_sum(t)
    else:
        import torch.distributed as dist
        dist.all_reduce(t, group=group)


def slab_bounds(n0, size):
    """(begin, end) of each rank's planes: sizes differ by at most one."""
    q, r = divmod(int(n0), int(size))
    beg = [k * q + min(k, r) for k in range(size)]
    end = [b + q + (k < r) for k, b in enumerate(beg)]
    return list(zip(beg, end))


class GridDomain:
    """Rank ``rank`` of a P0 x P1 x P2 process grid (rank = (r0 P1 + r1) P2
    + r2; ``dims`` of two entries means P2 = 1) owning the box [beg, end)
    x [beg1, end1) x [beg2, end2).  ``replicated``: every rank holds the
    whole grid (the coarse levels of a split V-cycle); halos then come
    from the rank's own points and nothing is sent.  Axis 0 is always
    treated as split; axis 2 when P2 > 1, axis 1 when P1 > 1 or P2 > 1."""

    def __init__(self, n_c, pbc_c, rank, dims, replicated=False):
        self.n_c = tuple(int(x) for x in n_c)
        pbc = [bool(p) for p in pbc_c] + [False] * (3 - len(pbc_c))
        self.periodic = tuple(pbc)
        self.periodic0 = self.periodic[0]
        d = [int(x) for x in dims] + [1] * (3 - len(dims))
        self.dims = tuple(d)
        self.rank = int(rank)
        self.size = d[0] * d[1] * d[2]
        self.replicated = bool(replicated)
        if self.replicated:
            self.boxes = [tuple((0, n) for n in self.n_c)] * self.size
        else:
            b = [slab_bounds(n, p) for n, p in zip(self.n_c, d)]
            self.boxes = [(b[0][r // (d[1] * d[2])],
                           b[1][(r // d[2]) % d[1]], b[2][r % d[2]])
                          for r in range(self.size)]
        self.bounds = [bx[0] for bx in self.boxes]
        ((self.beg, self.end), (self.beg1, self.end1),
         (self.beg2, self.end2)) = self.boxes[self.rank]
        self.m0 = self.end - self.beg
        self.m1 = self.end1 - self.beg1
        self.m2 = self.end2 - self.beg2
        # axes whose halos the gathers fill: axis 0, and every axis up to
        # the last split one -- an unsplit axis 1 before a split axis 2 is
        # gathered too, so that points past several periodic edges take
        # their phases axis by axis in order, as the whole grid's fill
        # multiplies them
        self.split = (True, d[1] > 1 or d[2] > 1, d[2] > 1)
        self.split1 = self.split[1]

    def local_shape(self):
        return (self.m0, self.m1, self.m2)

    def inner(self, a):
        """This rank's box of a whole-grid array (leading axes kept)."""
        return a[..., self.beg:self.end, self.beg1:self.end1,
                 self.beg2:self.end2]

    def thinnest(self):
        """Fewest points of a rank's box along each split axis, as a box of
        an unreplicated split would have."""
        return tuple(min(e - b for b, e in slab_bounds(n, p))
                     for n, p, sp in zip(self.n_c, self.dims, self.split)
                     if sp)


class SlabDomain(GridDomain):
    """Rank ``rank`` of ``size`` owning planes [beg, end) of axis 0: the
    P0 x 1 x 1 grid, with the neighbouring ranks along axis 0."""

    def __init__(self, n_c, periodic0, rank, size, replicated=False):
        super().__init__(n_c, (periodic0, False, False), rank, (size, 1, 1),
                         replicated)
        if self.replicated:
            # the rank's own planes across a periodic edge
            self.lower = self.upper = self.rank if self.periodic0 else None
            return
        self.lower = self.rank - 1 if self.rank > 0 else \
            (self.size - 1 if self.periodic0 else None)
        self.upper = self.rank + 1 if self.rank < self.size - 1 else \
            (0 if self.periodic0 else None)


def make_domain(n_c, pbc_c, rank, size, dims=None, replicated=False):
    """A SlabDomain of ``size`` ranks, or the GridDomain of the process
    grid ``dims`` (P0, P1) or (P0, P1, P2)."""
    if dims is None or int(np.prod([int(x) for x in dims[1:]])) == 1:
        return SlabDomain(n_c, bool(pbc_c[0]), rank, size, replicated)
    if int(np.prod([int(x) for x in dims])) != int(size):
        raise ValueError('dims %s do not make %d ranks' % (dims, size))
    return GridDomain(n_c, tuple(bool(p) for p in pbc_c), rank, dims,
                      replicated)


def exchange_halos(a, R, dom, phase_cd=None, group=None):
    """Collective: local box a (..., m0, m1, m2) -> the box grown by R_c
    points on either side along every split axis c (``R`` is one number
    for all, or one per axis; unsplit axes grow by nothing), the points
    coming from the ranks that hold them: zeros past a zero boundary;
    points that crossed a periodic edge times the Bloch phase when
    ``phase_cd`` is given (phase_cd[c][1] per crossing of the low edge of
    axis c, [c][0] of the high edge; axis 0 first, then 1, then 2, as the
    reference's halo fill of edges and corners multiplies them).  One
    gather_box: the sends and receives go as one batch, ordered alike on
    both sides, so two ranks that are each other's upper and lower
    neighbour cannot wait on each other; boxes thinner than the halo take
    points from ranks further away.  Works on torch tensors on any device
    the process group can send from."""
    Rc = [int(R)] * 3 if np.isscalar(R) else \
        [int(x) for x in R] + [0] * (3 - len(R))
    Rc = [r if sp else 0 for r, sp in zip(Rc, dom.split)]
    needs = [tuple((b - r, e + r) for (b, e), r in zip(box, Rc))
             for box in dom.boxes]
    return gather_box(a, needs, dom.boxes, dom.rank, dom.n_c,
                      dom.periodic, phase_cd, group)


class DistributedFDOperator:
    """A stencil (coef_p, offset_pc) applied to a grid split in slabs (or
    boxes of a process grid).  ``make_local(coef_p, offset_pc, n_c,
    pbc_c)`` builds the operator of one box plus halos (``n_c`` points,
    zero boundary along the split axes): on a GPU an FDOperator of
    gpaw_b200; any object with ``apply(in, out, phase_cd)``."""

    def __init__(self, coef_p, offset_pc, gd, dom, make_local, group=None):
        offset_pc = np.asarray(offset_pc, int)
        reach = np.abs(offset_pc).max(0) if len(offset_pc) else (0, 0, 0)
        self.Rc = tuple(int(r) if sp else 0
                        for r, sp in zip(reach, dom.split))
        self.R, self.R1 = self.Rc[0], self.Rc[1]
        self.dom, self.group = dom, group
        n_ext = tuple(m + 2 * r if sp else int(n) for m, r, sp, n in
                      zip(dom.local_shape(), self.Rc, dom.split, gd.n_c))
        pbc = tuple(False if sp else bool(p)
                    for sp, p in zip(dom.split, gd.pbc_c))
        self.local = make_local(coef_p, offset_pc, n_ext, pbc)

    def _halos(self, a, phase_cd=None):
        return exchange_halos(a, self.Rc, self.dom, phase_cd, self.group)

    def _inner(self, ext):
        sl = tuple(slice(r, r + m)
                   for r, m in zip(self.Rc, self.dom.local_shape()))
        return ext[(Ellipsis,) + sl]

    def apply(self, a, out, phase_cd=None):
        ext = self._halos(a, phase_cd)
        tmp = ext.new_zeros(ext.shape)
        ph = None
        if phase_cd is not None:
            ph = np.array(phase_cd, complex)
            for c, sp in enumerate(self.dom.split):
                if sp:               # split axes' phases travelled with
                    ph[c] = 1.0      # the halos
        self.local.apply(ext, tmp, ph)
        out[...] = self._inner(tmp)

    def relax(self, relax_method, f, s, n, w=None):
        """Weighted Jacobi (method 2) on the split grid: before every sweep
        the halos of f are exchanged, the box plus halos is swept once,
        and its interior kept -- the same sweeps as on the whole grid.
        Gauss-Seidel's lexicographic order does not split across ranks."""
        if relax_method != 2:
            raise NotImplementedError('only weighted Jacobi (2) runs on '
                                      'slabs')
        s_ext = s.new_zeros(s.shape[:-3] + tuple(
            m + 2 * r for m, r in zip(self.dom.local_shape(), self.Rc)))
        self._inner(s_ext)[...] = s
        for _ in range(n):
            ext = self._halos(f)
            self.local.relax(2, ext, s_ext, 1, w)
            f[...] = self._inner(ext)

    def residual_norm2(self, phi, rho, dv=1.0):
        """sum over the whole grid of (L phi - rho)^2 * dv, summed over the
        ranks (all ranks get it)."""
        r = phi.new_zeros(phi.shape)
        self.apply(phi, r)
        r -= rho
        t = (r * r).sum().reshape(1) * dv
        if self.dom.size > 1:
            _all_reduce_sum(t, self.group)
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


def gpu_local_transformer(device=None):
    """``make_local`` for DistributedTransformer on a GPU: a Transformer
    object of this library with the given geometry."""
    def make(size_in, size_out, k, pads, npads, skip, neighbors, real,
             interpolate):
        from . import cgpaw
        return cgpaw.Transformer(size_in, size_out, k, pads, npads, skip,
                                 neighbors, real, None, interpolate)
    return make


# --------------------------------------------------------------------------
# any run of planes from the ranks that hold them
# --------------------------------------------------------------------------
def _segments(lo, hi, n, periodic, cuts):
    """[lo, hi) of one axis (indices past either edge wrap round a periodic
    axis and are zeros past a zero boundary) as runs (dst, p, length, wraps)
    that cross neither a wrap edge nor any rank's box boundary (``cuts``):
    global points p.. go to dst.. of the receiver's buffer; ``wraps`` counts
    the crossings of the periodic edge (negative: the low one)."""
    segs = []
    g = lo
    while g < hi:
        k, p = divmod(g, n)
        if k and not periodic:
            if g < 0:
                g = min(0, hi)
                continue
            break
        nxt = min([c for c in cuts if c > p] + [n])
        take = min(nxt - p, hi - g)
        segs.append((g - lo, p, take, k))
        g += take
    return segs


def _owner(point, boxes, recv):
    """The rank that sends ``point`` (one index per gathered axis) to rank
    ``recv``: recv itself when it holds it (replicated levels), else the
    first rank whose box does."""
    for r in [recv] + list(range(len(boxes))):
        if all(b <= p < e for p, (b, e) in zip(point, boxes[r])):
            return r
    raise ValueError('point %s is held by no rank' % (point,))


def box_pieces(need, n_c, periodic_c, boxes, recv):
    """The box ``need`` = ((lo0, hi0), (lo1, hi1), ...) of the gathered
    axes as pieces (owner, src, dst, lengths, wraps), one entry per axis:
    points src.. of the owner's box go to dst.. of the receiver's buffer,
    having crossed the periodic edges wraps times.  Every rank computes
    every receiver's list the same way, so senders and receivers agree on
    the pieces and their order."""
    import itertools
    na = len(need)
    cuts = [sorted({x for b in boxes for x in b[c]}) for c in range(na)]
    segs = [_segments(need[c][0], need[c][1], n_c[c], periodic_c[c],
                      cuts[c]) for c in range(na)]
    pieces = []
    for combo in itertools.product(*segs):
        point = tuple(sg[1] for sg in combo)
        owner = _owner(point, boxes, recv)
        pieces.append((owner,
                       tuple(sg[1] - boxes[owner][c][0]
                             for c, sg in enumerate(combo)),
                       tuple(sg[0] for sg in combo),
                       tuple(sg[2] for sg in combo),
                       tuple(sg[3] for sg in combo)))
    return pieces


def _phase_mul(t, ph):
    """ph * t in place, each product rounded on its own and summed as
    (a c - b d) + i (a d + b c), the grouping of the reference's complex
    halo multiply (c/bmgs/translate.cpp:28)."""
    import torch
    a, b = float(ph.real), float(ph.imag)
    r = torch.view_as_real(t)
    c, d = r[..., 0].clone(), r[..., 1].clone()
    r[..., 0] = c * a - d * b
    r[..., 1] = d * a + c * b


def _tup(x):
    """Nested lists of bounds as nested tuples of ints (hashable)."""
    if isinstance(x, (list, tuple, np.ndarray)):
        return tuple(_tup(y) for y in x)
    return int(x)


@functools.lru_cache(maxsize=512)
def _gather_plan(needs, boxes, rank, n_c, periodic_c):
    """This rank's part of a gather, computed once per layout: entries
    (kind, peer, tag, source slices, destination slices, wraps) with kind
    'copy' (from its own box), 'recv' or 'send', in the order both sides
    derive from box_pieces."""
    plan = []
    for r, need in enumerate(needs):
        for idx, (owner, src, dst, ln, k) in enumerate(
                box_pieces(need, n_c, periodic_c, boxes, r)):
            sl = (Ellipsis,) + tuple(slice(x, x + m)
                                     for x, m in zip(src, ln))
            dl = (Ellipsis,) + tuple(slice(x, x + m)
                                     for x, m in zip(dst, ln))
            if r == rank and owner == rank:
                plan.append(('copy', rank, idx, sl, dl, k))
            elif r == rank:
                plan.append(('recv', owner, idx, None, dl, k))
            elif owner == rank:
                plan.append(('send', r, idx, sl, None, k))
    return tuple(plan)


def gather_box(a, needs, boxes, rank, n_c, periodic_c, phase_cd=None,
               group=None):
    """Collective: every rank gets the points ``needs[rank]`` = ((lo0,
    hi0), (lo1, hi1), (lo2, hi2)) of a grid of ``n_c`` points from
    whichever ranks hold them (``boxes[r]``: the box rank r holds in
    ``a``).  Returns (..., hi0 - lo0, hi1 - lo1, hi2 - lo2): zeros past a
    zero boundary; for complex data with ``phase_cd``, points that crossed
    the periodic edge of axis c upwards times phase_cd[c][0] per crossing,
    downwards times phase_cd[c][1], axis 0 first, then 1, then 2, as the
    reference's halo fill multiplies them (c/bc.cpp:146-258).  The
    messages are one batch of point-to-point sends and receives, ordered
    alike on both sides.  Over NCCL, run one collective on the group (a
    barrier) before the first gather, so that every rank has set up its
    communicator when the first batch starts."""
    import torch
    plan = _gather_plan(_tup(needs), _tup(boxes), int(rank),
                        tuple(int(n) for n in n_c),
                        tuple(bool(p) for p in periodic_c))
    out = a.new_zeros(a.shape[:-3] +
                      tuple(hi - lo for lo, hi in needs[rank]))
    sends, recvs, recvd = [], [], []
    for kind, peer, idx, sl, dl, k in plan:
        if kind == 'copy':
            out[dl] = a[sl]
            recvd.append((dl, k, None))
        elif kind == 'recv':
            buf = torch.empty_like(out[dl])
            recvs.append((peer, idx, buf))
            recvd.append((dl, k, buf))
        else:
            sends.append((peer, idx, a[sl].contiguous()))
    if isinstance(group, LocalRanks):
        group.exchange(sends, recvs)
    elif sends or recvs:
        import torch.distributed as dist
        # the same order of operations as before: the plan's order
        ops = []
        si, ri = iter(sends), iter(recvs)
        for kind, peer, idx, sl, dl, k in plan:
            if kind == 'recv':
                _, tag, buf = next(ri)
                ops.append(dist.P2POp(dist.irecv, buf, peer, group, tag=tag))
            elif kind == 'send':
                _, tag, t = next(si)
                ops.append(dist.P2POp(dist.isend, t, peer, group, tag=tag))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    ph = None if phase_cd is None else np.asarray(phase_cd)
    for dl, k, buf in recvd:
        view = out[dl]
        if buf is not None:
            view.copy_(buf)
        if ph is None or not a.is_complex():
            continue
        for c in range(3):
            if k[c]:
                f = ph[c][0] if k[c] > 0 else ph[c][1]
                for _ in range(abs(k[c])):
                    _phase_mul(view, complex(f))
    return out


def gather_planes(a, needs, n0, periodic0, bounds, rank, phase_cd=None,
                  group=None):
    """Collective: gather_box along axis 0 alone -- every rank gets the
    global planes [lo, hi) that ``needs[rank]`` names from the ranks whose
    planes ``bounds`` lists."""
    n1, n2 = a.shape[-2:]
    return gather_box(a, [(tuple(nd), (0, n1), (0, n2)) for nd in needs],
                      [(tuple(b), (0, n1), (0, n2)) for b in bounds], rank,
                      (n0, n1, n2), (periodic0, False, False), phase_cd,
                      group)


def gather_full(a, dom, group=None):
    """Collective: the whole of a split grid on every rank."""
    return gather_box(a, [tuple((0, n) for n in dom.n_c)] * dom.size,
                      dom.boxes, dom.rank, dom.n_c, dom.periodic, None,
                      group)


# --------------------------------------------------------------------------
# restriction and interpolation between split grids
# --------------------------------------------------------------------------
class DistributedTransformer:
    """Restriction or interpolation (gpaw/transformers.py:18-94) from a grid
    on slabs (or boxes) ``dom_in`` to one on ``dom_out`` of the same shape
    of process grid (either may be replicated).  Each rank gathers the
    input points that its output points reach along the split axes (the
    stencil's K - 1 = 2 nn - 1 fine points either side of a coarse point's
    centre 2 J, or the nn coarse points either side of a fine midpoint) and
    runs one transformer on them: the split axes get no padding of their
    own (the gathered points are the padding) and the others keep the whole
    grid's geometry (transformer_geometry).  Every
    output point is computed from the same values in the same order as on
    the whole grid, so the results are identical.

    ``make_local(size_in, size_out, k, pads, npads, skip, neighbors, real,
    interpolate)`` builds the transformer of one rank (on a GPU:
    gpu_local_transformer)."""

    def __init__(self, gdin, gdout, nn, dtype, dom_in, dom_out, make_local,
                 group=None):
        from .transformers import transformer_geometry
        pad, npad, skip, self.interpolate = transformer_geometry(gdin, gdout,
                                                                 nn)
        self.dom_in, self.dom_out, self.group = dom_in, dom_out, group
        self.K = K = 2 * int(nn)
        self.dtype = dtype
        axes = tuple(c for c in range(3) if dom_out.split[c])
        self.axes = axes
        self.needs, self.keep = [], []
        mine = None
        for r in range(dom_out.size):
            geo = {c: self._axis(dom_out.boxes[r][c], int(gdin.beg_c[c]),
                                 int(gdout.beg_c[c]), K) for c in axes}
            if any(g is None for g in geo.values()):
                self.needs.append(((0, 0),) * 3)
                self.keep.append(None)
                continue
            self.needs.append(tuple(geo[c][:2] if c in geo else
                                    (0, int(gdin.n_c[c])) for c in range(3)))
            self.keep.append(tuple(e - b for b, e in dom_out.boxes[r]))
            if r == dom_out.rank:
                mine = geo
        self.local = None
        if mine is not None:
            pads = np.array(pad, np.int64).reshape(3, 2)
            npads = np.array(npad, np.int64).reshape(3, 2)
            skips = np.array(skip, np.int64).reshape(3, 2)
            nb = np.array(gdin.neighbor_cd, np.int64).reshape(3, 2).copy()
            size_in = [int(x) for x in gdin.n_c]
            size_out = [int(x) for x in gdout.n_c]
            for c, (lo, hi, mcalc, s0) in mine.items():
                pads[c] = npads[c] = 0
                skips[c] = (s0, 0)
                nb[c] = -1
                size_in[c] = hi - lo
                size_out[c] = mcalc
            self.size_in, self.size_out = tuple(size_in), tuple(size_out)
            self.local = make_local(
                np.array(size_in, np.int64), np.array(size_out, np.int64),
                K, pads, npads, skips, nb, dtype == float, self.interpolate)

    def _axis(self, box, bi, bo, K):
        """(lo, hi, mcalc, s0) along one split axis for the output points
        [ob, oe): the input points [lo, hi) they reach, the outputs the
        local transformer computes and its skip of the first one; None
        for an empty box."""
        ob, oe = box
        if oe <= ob:
            return None
        if not self.interpolate:
            # coarse global J is centred on fine global 2 J
            lo = 2 * (ob + bo) - bi - (K - 1)
            hi = 2 * (oe - 1 + bo) - bi + K
            return lo, hi, oe - ob, 0
        # fine global G: even 2 J copies coarse J, odd 2 J + 1 reads coarse
        # J - nn + 1 .. J + nn; the first output is dropped when the box
        # starts on an odd point, and one extra fine point is computed (and
        # dropped) so that whole coarse points are processed
        g0 = ob + bo
        s0 = g0 % 2
        mf = oe - ob
        mcalc = mf + (mf + s0) % 2
        n = (mcalc + s0) // 2
        lo = (g0 - s0) // 2 - bi - K // 2 + 1
        return lo, lo + n + K - 1, mcalc, s0

    def apply(self, a, out, phases=None):
        """Collective: ``a`` holds this rank's input box, ``out`` gets its
        output box."""
        di = self.dom_in
        ext = gather_box(a, self.needs, di.boxes, di.rank, di.n_c,
                         di.periodic, phases, self.group)
        if self.local is None:
            return out
        m = self.keep[self.dom_out.rank]
        if tuple(self.size_out) == m:
            self.local.apply(ext, out, phases)
        else:
            tmp = out.new_zeros(out.shape[:-3] + self.size_out)
            self.local.apply(ext, tmp, phases)
            out[...] = tmp[..., :m[0], :m[1], :m[2]]
        return out


# --------------------------------------------------------------------------
# the FD Poisson V-cycle on slabs
# --------------------------------------------------------------------------
def _level_domains(gds, ranges, rank, size, dims, min_planes):
    """The domain of every level: split (slabs, or boxes of the process
    grid ``dims``) while each rank's extent along every split axis is at
    least max(min_planes, R) points, whole on every rank below."""
    doms = []
    split = True
    for level, (gd, R) in enumerate(zip(gds, ranges)):
        dom = make_domain(gd.n_c, gd.pbc_c, rank, size, dims)
        need = max(int(min_planes), int(R))
        split = split and min(dom.thinnest()) >= need
        if level == 0 and not split:
            raise ValueError('every rank needs at least %d points of the '
                             'finest grid along each split axis' % need)
        if not split:
            dom = make_domain(gd.n_c, gd.pbc_c, rank, size, dims,
                              replicated=True)
        doms.append(dom)
    return doms


class DistributedFDPoissonSolver:
    """The V-cycle of FDPoissonSolver.iterate2 (gpaw/poisson.py:500-537) on
    a grid split in slabs.  ``ps`` is a solver on the whole grid after
    set_grid_descriptor: its levels, stencils, sweep counts and weights are
    used (the coarsest level smooths 8 + 8, :451-472).  Levels stay split
    while every slab of the level holds at least max(min_planes, R) planes
    (R: the level's stencil range); the level below the last split one is
    gathered whole on every rank, which run the rest of the V-cycle alike
    and keep their own slab of the correction.  Relaxation is weighted
    Jacobi (Gauss-Seidel's lexicographic order does not split).

    ``make_op`` / ``make_tr`` build the slab-local operators and
    transformers (gpu_local_operator / gpu_local_transformer on a GPU)."""

    def __init__(self, ps, rank, size, make_op, make_tr, group=None,
                 min_planes=2, dims=None):
        if ps.relax_method != 2:
            raise NotImplementedError('only weighted Jacobi runs on slabs')
        self.ps, self.group = ps, group
        self.rank, self.size = int(rank), int(size)
        self.levels = ps.levels
        self.pre = list(ps.presmooths)
        self.post = list(ps.postsmooths)
        self.pre[self.levels] = 8
        self.post[self.levels] = 8
        self.weights = list(ps.weights)
        self.relax_method = 2
        self.gd = ps.gd
        gds = [op.gd for op in ps.operators]
        self.doms = _level_domains(gds, [self._op_range(op)
                                         for op in ps.operators],
                                   rank, size, dims, min_planes)
        self.split_levels = sum(not d.replicated for d in self.doms)
        self.B = None
        self.restrictors, self.interpolators = [], []
        for level in range(self.levels):
            r, i = ps.restrictors[level], ps.interpolators[level]
            self.restrictors.append(DistributedTransformer(
                gds[level], gds[level + 1], r.nn, float, self.doms[level],
                self.doms[level + 1], make_tr, group))
            self.interpolators.append(DistributedTransformer(
                gds[level + 1], gds[level], i.nn, float,
                self.doms[level + 1], self.doms[level], make_tr, group))
        self._arrays = None
        self._build_ops(make_op, gds)

    @staticmethod
    def _op_range(op):
        """Points the level's stencil reaches along an axis."""
        return int(np.abs(np.asarray(op.offset_pc, int)).max())

    def _build_ops(self, make_op, gds):
        ps, group = self.ps, self.group
        self.ops = [DistributedFDOperator(op.coef_p, op.offset_pc, gd, dom,
                                          make_op, group)
                    for op, gd, dom in zip(ps.operators, gds, self.doms)]
        # Mehrstellen (nn = 'M'): rho is replaced by B rho before solving
        B = getattr(ps, 'B', None)
        if B is not None:
            self.B = DistributedFDOperator(B.coef_p, B.offset_pc, gds[0],
                                           self.doms[0], make_op, group)

    def _alloc(self, like):
        if self._arrays is not None and self._arrays[0].device == \
                like.device:
            return
        self.phis = [None]
        self.rhos = [None]
        self.residuals = []
        for level, dom in enumerate(self.doms):
            z = like.new_zeros(dom.local_shape())
            self.residuals.append(z)
            if level:
                self.phis.append(like.new_zeros(dom.local_shape()))
                self.rhos.append(like.new_zeros(dom.local_shape()))
        self._arrays = self.residuals

    def iterate(self, phi, rho):
        """Collective: one V-cycle on this rank's slabs of phi (updated in
        place) and rho; returns the level-0 error sum(r^2) dv over the
        whole grid (every rank gets it)."""
        self._alloc(phi)
        self.phis[0] = phi
        self.rhos[0] = rho
        return self._cycle(0)

    def _sum(self, t):
        t = t.sum().reshape(1)
        if self.size > 1:
            _all_reduce_sum(t, self.group)
        return float(t.item())

    def solve_neutral(self, phi, rho, eps=None, maxiter=None):
        """Collective: gpaw/poisson.py:474-498 on slabs -- V-cycles until
        the level-0 error is at most ``eps`` (the whole-grid solver's by
        default), then, on a fully periodic grid, the mean of phi over the
        whole grid removed.  Returns the number of V-cycles; raises
        PoissonConvergenceError at ``maxiter``."""
        from ._lib import PoissonConvergenceError
        eps = self.ps.eps if eps is None else eps
        maxiter = self.ps.maxiter if maxiter is None else maxiter
        if self.B is not None:
            rhob = rho.new_zeros(rho.shape)
            self.B.apply(rho, rhob)
            rho = rhob
        niter = 1
        while self.iterate(phi, rho) > eps and niter < maxiter:
            niter += 1
        if niter == maxiter:
            raise PoissonConvergenceError(
                'Poisson solver did not converge in %d iterations!'
                % maxiter)
        if bool(np.all(self.gd.pbc_c)):
            phi -= self._sum(phi) / float(np.prod(self.gd.n_c))
        self.niter = niter
        return niter

    def solve(self, phi, rho, charge=None, maxcharge=1e-6,
              zero_initial_phi=False, gauss=None, use_charge_center=None):
        """Collective: gpaw/poisson.py:182-283 on slabs.  Neutral systems
        and charged fully periodic ones (the homogeneous background of the
        whole grid's charge is subtracted from rho); charged systems in a
        non-periodic cell through a Gaussian carrying the charge, solved
        neutral, its potential added back.  ``gauss``: the whole grid's
        (rho_gauss, phi_gauss), or a function of the Gaussian's centre
        returning them; by default gauss.monopole_gaussian of the grid
        (each rank keeps its own box of them).  ``use_charge_center``
        (default: the whole-grid solver's setting) centres the Gaussian on
        the majority charge, from sums over the ranks (:248-262)."""
        actual_charge = self._sum(rho) * float(self.gd.dv)
        background = actual_charge / float(self.gd.dv) / \
            float(np.prod(self.gd.n_c))
        if charge is None:
            charge = actual_charge
        pbc = np.asarray(self.gd.pbc_c, bool)
        if abs(charge) <= maxcharge:
            return self.solve_neutral(phi, rho - background)
        if pbc.all():
            if zero_initial_phi:
                phi.zero_()
            return self.solve_neutral(phi, rho - background)
        if pbc.any():
            raise NotImplementedError(
                'charged system with mixed boundary conditions')
        import torch
        dom = self.doms[0]
        if use_charge_center is None:
            use_charge_center = getattr(self.ps, 'use_charge_center', False)
        center = None
        if use_charge_center:
            from .gauss import charge_center, charge_center_parts
            rhog_c, total = charge_center_parts(
                self.gd, rho, actual_charge, (dom.beg, dom.beg1, dom.beg2))
            t = torch.tensor(list(rhog_c) + [total], dtype=torch.float64,
                             device=rho.device)
            if self.size > 1:
                _all_reduce_sum(t, self.group)
            t = t.cpu().numpy()
            center = charge_center(self.gd, t[:3], float(t[3]))
        if gauss is None:
            from .gauss import monopole_gaussian
            gauss = monopole_gaussian(self.gd, center=center)
        elif callable(gauss):
            gauss = gauss(center)
        rg, pg = [torch.as_tensor(np.ascontiguousarray(
            dom.inner(np.asarray(g)))).to(phi.device) for g in gauss]
        q = actual_charge / np.sqrt(4 * np.pi)
        rho_neutral = rho - q * rg
        if zero_initial_phi:
            phi.zero_()
        else:
            phi -= q * pg
        niter = self.solve_neutral(phi, rho_neutral)
        phi += q * pg
        return niter

    def _cycle(self, level):
        op = self.ops[level]
        residual = self.residuals[level]
        if level < self.levels:
            op.relax(2, self.phis[level], self.rhos[level],
                     self.pre[level], self.weights[level])
            op.apply(self.phis[level], residual)
            residual -= self.rhos[level]
            self.restrictors[level].apply(residual, self.rhos[level + 1])
            self.phis[level + 1].zero_()
            self._cycle(level + 1)
            self.interpolators[level].apply(self.phis[level + 1], residual)
            self.phis[level] -= residual
        op.relax(2, self.phis[level], self.rhos[level], self.post[level],
                 self.weights[level])
        if level == 0:
            return op.residual_norm2(self.phis[0], self.rhos[0],
                                     float(self.gd.dv))


# --------------------------------------------------------------------------
# weighted operators and the dielectric Poisson solver on slabs
# --------------------------------------------------------------------------
class DistributedWeightedOperator(DistributedFDOperator):
    """A WeightedFDOperator (gpaw/wfd_operators.py) on a grid split in
    slabs: sum_i w_i(x) L_i with this rank's slabs of the weights.  The
    weights' halo planes are exchanged once, here; apply and the Jacobi
    sweeps exchange the operand's halos as DistributedFDOperator does.
    The stencils' flattened offsets depend only on the padded extents of
    axes 1 and 2, which a slab shares with the whole grid, so they are
    used unchanged; on boxes with a split axis 1 or 2 they are re-flattened
    for the box's extents.  ``make_local(nweights, weights, coef_ps, offset_ps,
    n_c, r, neighbors, real, cfd)`` builds the WOperator of one slab plus
    halos (on a GPU: gpu_local_woperator)."""

    def __init__(self, wop, weights, dom, make_local, group=None):
        R = int(wop.mp)
        self.Rc = tuple(R if sp else 0 for sp in dom.split)
        self.R, self.R1 = self.Rc[0], self.Rc[1]
        self.dom, self.group = dom, group
        n_c = [int(x) for x in wop.gd.n_c]
        n_ext = [m + 2 * r if sp else n for m, r, sp, n in
                 zip(dom.local_shape(), self.Rc, dom.split, n_c)]
        nb = np.array(wop.gd.neighbor_cd, np.int64).reshape(3, 2).copy()
        for c, sp in enumerate(dom.split):
            if sp:
                nb[c] = -1
        offset_ps = wop.offset_ps
        if dom.split[1] or dom.split[2]:
            offset_ps = [_reflatten(o, n_c[1] + 2 * R, n_c[2] + 2 * R,
                                    n_ext[1] + 2 * R, n_ext[2] + 2 * R)
                         for o in offset_ps]
        self.weights_ext = [exchange_halos(w, self.Rc, dom, None, group)
                            for w in weights]
        self.local = make_local(wop.nweights, self.weights_ext, wop.coef_ps,
                                offset_ps, np.array(n_ext, np.int64), R,
                                nb, wop.dtype == float, wop.cfd)


def _reflatten(offsets, M1, M2, M1_new, M2_new):
    """Flattened stencil offsets (o0 M1 + o1) M2 + o2 of a grid padded to
    M1 x M2 points on axes 1 and 2, re-flattened for extents M1_new x
    M2_new (every |o1|, |o2| is at most the padding, below half of M1 and
    M2, so the split is unique)."""
    out = []
    for o in np.asarray(offsets, np.int64):
        o = int(o)
        o2 = (o + M2 // 2) % M2 - M2 // 2
        rest = (o - o2) // M2
        o1 = (rest + M1 // 2) % M1 - M1 // 2
        o0 = (rest - o1) // M1
        out.append((o0 * M1_new + o1) * M2_new + o2)
    return np.array(out, np.int64)


def gpu_local_woperator():
    """``make_local`` for DistributedWeightedOperator on a GPU: a WOperator
    of this library."""
    def make(nweights, weights, coef_ps, offset_ps, n_c, r, neighbors, real,
             cfd):
        from . import cgpaw
        return cgpaw.WOperator(nweights, weights, coef_ps, offset_ps, n_c, r,
                               neighbors, real, None, cfd)
    return make


class DistributedWeightedFDPoissonSolver(DistributedFDPoissonSolver):
    """The dielectric Poisson solver's V-cycle
    (gpaw/old/solvation/poisson.py:75-124) on slabs: level 0 weighted by
    this rank's slabs of eps and its gradient (``eps_gradeps``), every
    coarser level by the restrictions of the finer level's weights
    (restrict_op_weights, :100-106) through the slab transformers.
    ``ps`` is the whole-grid WeightedFDPoissonSolver after
    set_grid_descriptor; ``make_op`` builds weighted slab operators."""

    def __init__(self, ps, eps_gradeps, rank, size, make_op, make_tr,
                 group=None, min_planes=2, dims=None):
        self._eps_gradeps = list(eps_gradeps)
        super().__init__(ps, rank, size, make_op, make_tr, group,
                         min_planes, dims)

    @staticmethod
    def _op_range(op):
        return int(op.mp)

    def solve(self, phi, rho, charge=None, maxcharge=1e-6,
              zero_initial_phi=False, gauss=None):
        """Collective: :87-98 on slabs.  Periodic systems must be neutral;
        a charged one in a non-periodic cell needs the dielectric's
        compensation charge and its potential on the whole grid,
        ``gauss=(rho_gauss, phi_gauss)`` (WeightedFDPoissonSolver.
        load_gauss), of which each rank keeps its slab."""
        actual_charge = self._sum(rho) * float(self.gd.dv)
        pbc = np.asarray(self.gd.pbc_c, bool)
        if pbc.all() and abs(actual_charge) > maxcharge:
            raise NotImplementedError(
                'charged periodic systems are not implemented')
        q = actual_charge if charge is None else charge
        if abs(q) > maxcharge and not pbc.any() and gauss is None:
            raise ValueError('a charged system in a dielectric needs '
                             'gauss=(rho_gauss, phi_gauss) of the whole '
                             'grid')
        return super().solve(phi, rho, charge, maxcharge, zero_initial_phi,
                             gauss)

    def _build_ops(self, make_op, gds):
        weights = self._eps_gradeps
        self.ops = []
        for level, (op, dom) in enumerate(zip(self.ps.operators,
                                              self.doms)):
            self.ops.append(DistributedWeightedOperator(op, weights, dom,
                                                        make_op, self.group))
            if level < self.levels:
                nxt = [w.new_zeros(self.doms[level + 1].local_shape())
                       for w in weights]
                for w, c in zip(weights, nxt):
                    self.restrictors[level].apply(w, c)
                weights = nxt


# --------------------------------------------------------------------------
# the multigrid preconditioner on slabs
# --------------------------------------------------------------------------
class DistributedPreconditioner:
    """The three-level preconditioner of gpaw/preconditioner.py:9-73 (the
    sequence of c/fd_preconditioner.cpp:106-351, scalar factors 4 step and
    16 step) on a grid split in slabs.  ``pre`` is a Preconditioner on the
    whole grid: its kinetic operators, step and transformer orders are
    used.  Levels 1 and 2 stay split while every slab holds at least
    ``min_planes`` planes, else every rank holds them whole.
    ``make_op`` / ``make_tr`` build the slab-local operators and
    transformers for the preconditioner's dtype."""

    def __init__(self, pre, rank, size, make_op, make_tr, group=None,
                 min_planes=2, dims=None):
        # the kinetic operator of each level: the product's Preconditioner
        # keeps them in its level list, the oracle's as kin0..kin2
        if hasattr(pre, 'levels'):
            kins = [lv.kin for lv in pre.levels]
        else:
            kins = [pre.kin0, pre.kin1, pre.kin2]
        gds = [k.gd for k in kins]
        self.step = float(pre.step)
        self.group = group
        dtype = getattr(kins[1], 'dtype', float)
        ranges = [int(np.abs(np.asarray(k.offset_pc, int)).max())
                  for k in kins]
        self.doms = _level_domains(gds, ranges, rank, size, dims,
                                   min_planes)
        self.kin = [DistributedFDOperator(k.coef_p, k.offset_pc, gd, dom,
                                          make_op, group)
                    for k, gd, dom in zip(kins, gds, self.doms)]
        d0, d1, d2 = self.doms

        # the preconditioner's transfers are all of order 2 (nn = 1)
        def tr(gi, go, di, do):
            return DistributedTransformer(gi, go, 1, dtype, di, do,
                                          make_tr, group)
        self.rest0 = tr(gds[0], gds[1], d0, d1)
        self.rest1 = tr(gds[1], gds[2], d1, d2)
        self.intp2 = tr(gds[2], gds[1], d2, d1)
        self.intp1 = tr(gds[1], gds[0], d1, d0)

    def __call__(self, residuals, phases=None, out=None):
        """Collective: the preconditioned residuals of this rank's slab
        (leading batch axes allowed); ``out`` if given receives them."""
        lead = residuals.shape[:-3]
        s4, s16 = 4 * self.step, 16 * self.step

        def z(level):
            return residuals.new_zeros(lead + self.doms[level].local_shape())
        r1, d1, q1 = z(1), z(1), z(1)
        r2, q2 = z(2), z(2)
        d0 = out if out is not None else z(0)
        q0 = z(0)
        self.rest0.apply(-residuals, r1, phases)
        d1.copy_(s4 * r1)
        self.kin[1].apply(d1, q1, phases)
        q1 -= r1
        self.rest1.apply(q1, r2, phases)
        d2 = s16 * r2
        self.kin[2].apply(d2, q2, phases)
        q2 -= r2
        d2 -= s16 * q2
        self.intp2.apply(d2, q1, phases)
        d1 -= q1
        self.kin[1].apply(d1, q1, phases)
        q1 -= r1
        d1 -= s4 * q1
        d1.neg_()
        self.intp1.apply(d1, d0, phases)
        self.kin[0].apply(d0, q0, phases)
        q0 -= residuals
        d0 -= self.step * q0
        d0.neg_()
        return d0
