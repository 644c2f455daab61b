"""CPU restatement (numpy) of the reference's C objects on the FD hot path.

TEST INFRASTRUCTURE ONLY.  This module is an oracle: tests, ``smoke()`` and
the CPU-baseline leg of ``bench.py`` use it to check the CUDA path.  The
``gpaw_b200`` package never imports it.

It exposes the same three entry points, with the same argument order, as the
reference's compiled extension (c/_gpaw.h:182,185,194):

* ``Operator(coefs, offsets, size, range, neighbors, real, comm, cfd)``
  (c/operators.cpp:379-420) with ``apply``, ``relax``,
  ``get_diagonal_element``;
* ``Transformer(size_in, size_out, k, pads, npads, skip, neighbors, real,
  comm, interpolate)`` (c/transformers.cpp:196-246) with ``apply``;
* ``fd_precond(...)`` (c/fd_preconditioner.cpp:106-351).

Every floating-point expression keeps the reference's operation order and
grouping so that results are bit-identical to the compiled reference built
without FMA contraction (x86-64 -O2).  Single-domain only: a neighbour equal
to rank 0 means a periodic copy, -1 means a zero boundary
(c/bc.cpp:82-104).
"""
from __future__ import annotations

import numpy as np

COPY_DATA = -2   # c/bc.h:77
DO_NOTHING = -3  # c/bc.h:78


# --------------------------------------------------------------------------
# Boundary conditions: padded buffer fill (c/bc.cpp:17-143, 146-258)
# --------------------------------------------------------------------------
class BoundaryConditions:
    """Single-domain restatement of ``bc_init`` (c/bc.cpp:17-143)."""

    def __init__(self, size1, padding, npadding, neighbors, real, cfd):
        self.size1 = [int(x) for x in size1]
        padding = np.asarray(padding).reshape(3, 2)
        npadding = np.asarray(npadding).reshape(3, 2)
        neighbors = np.asarray(neighbors).reshape(3, 2)
        self.padding = padding
        self.size2 = [self.size1[i] + int(padding[i, 0]) + int(padding[i, 1])
                      for i in range(3)]
        self.real = bool(real)
        self.cfd = bool(cfd)
        # Slab geometry per (axis, side): start/size in the padded buffer.
        start = [int(padding[i, 0]) for i in range(3)]
        size = list(self.size1)
        self.sendstart = np.zeros((3, 2, 3), int)
        self.sendsize = np.zeros((3, 2, 3), int)
        self.recvstart = np.zeros((3, 2, 3), int)
        self.sendproc = np.full((3, 2), DO_NOTHING, int)
        for i in range(3):
            for d in range(2):
                ds = int(npadding[i, d])
                dr = int(padding[i, d])
                self.sendstart[i, d] = start
                self.sendsize[i, d] = size
                self.recvstart[i, d] = start
                if d == 0:
                    self.sendstart[i, d, i] = dr
                    self.recvstart[i, d, i] = 0
                else:
                    self.sendstart[i, d, i] = (int(padding[i, 0]) +
                                               self.size1[i] - ds)
                    self.recvstart[i, d, i] = (int(padding[i, 0]) +
                                               self.size1[i])
                self.sendsize[i, d, i] = ds
                p = int(neighbors[i, d])
                if p == 0 and ds > 0:       # own rank: periodic copy
                    self.sendproc[i, d] = COPY_DATA
                elif p > 0:
                    raise NotImplementedError('single domain only')
            if not self.cfd:
                # c/bc.cpp:108-112: later axes copy the full padded extent
                # along this axis, so edges and corners get filled.
                start[i] = 0
                size[i] = self.size2[i]

    def unpack(self, a, phases=None):
        """Return the padded buffer of one grid (c/bc.cpp:146-258).

        ``phases`` is the (3, 2) complex array of Bloch factors, only read
        for complex data (``bmgs_translatemz``, c/bmgs/translate.cpp:28).
        """
        dtype = float if self.real else complex
        buf = np.zeros(self.size2, dtype)
        p = self.padding
        n = self.size1
        # memset + paste (c/bc.cpp:159-173)
        buf[p[0, 0]:p[0, 0] + n[0], p[1, 0]:p[1, 0] + n[1],
            p[2, 0]:p[2, 0] + n[2]] = a
        for i in range(3):
            for d in range(2):
                if self.sendproc[i, d] != COPY_DATA:
                    continue
                src = tuple(slice(s, s + z) for s, z in
                            zip(self.sendstart[i, d], self.sendsize[i, d]))
                dst0 = self.recvstart[i, 1 - d]
                dst = tuple(slice(s, s + z) for s, z in
                            zip(dst0, self.sendsize[i, d]))
                if self.real:
                    buf[dst] = buf[src]                     # translate.cpp:8
                else:
                    buf[dst] = _cmul(phases[i][d], buf[src])  # :28
        return buf


def _cmul(ph, z):
    """phase * z with the grouping of libgcc's complex multiply:
    (a c - b d) + i (a d + b c), each product rounded separately."""
    ph = complex(ph)
    a, b = ph.real, ph.imag
    c, d = z.real, z.imag
    out = np.empty(z.shape, complex)
    out.real = a * c - b * d
    out.imag = a * d + b * c
    return out


# --------------------------------------------------------------------------
# Operator (c/operators.cpp, c/bmgs/fd.cpp, c/bmgs/relax.cpp)
# --------------------------------------------------------------------------
class Operator:
    """Restatement of the reference ``Operator`` object
    (c/operators.cpp:379-420; stencil struct c/bmgs/stencils.cpp:11-26)."""

    def __init__(self, coefs, offsets, size, r, neighbors, real, comm, cfd,
                 use_gpu=0):
        assert comm is None
        self.coefs = np.ascontiguousarray(coefs, float)
        self.offsets = np.ascontiguousarray(offsets, np.int64)
        self.n = [int(x) for x in size]
        self.r = int(r)
        pad = np.full((3, 2), self.r, int)
        self.bc = BoundaryConditions(self.n, pad, pad, neighbors, real, cfd)
        n0, n1, n2 = self.n
        M = [x + 2 * self.r for x in self.n]
        # flat index of every interior point in the padded buffer
        i0, i1, i2 = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2),
                                 indexing='ij')
        self._idx = (((i0 + self.r) * M[1] + i1 + self.r) * M[2] +
                     i2 + self.r).ravel()

    def _fd(self, buf):
        """bmgs_fd / bmgs_fdz (c/bmgs/fd.cpp:9-33): x += a[i+off]*coef in
        coefficient order, starting from 0.0."""
        flat = buf.ravel()
        x = np.zeros(self._idx.shape, buf.dtype)
        for c in range(len(self.coefs)):
            x = x + flat[self._idx + self.offsets[c]] * self.coefs[c]
        return x.reshape(self.n)

    def apply(self, inp, out, phases=None):
        """Operator_apply (c/operators.cpp:245-316), one grid at a time."""
        nin = inp.shape[0] if inp.ndim == 4 else 1
        src = inp.reshape((nin,) + tuple(self.n))
        dst = out.reshape((nin,) + tuple(self.n))
        for m in range(nin):
            dst[m] = self._fd(self.bc.unpack(src[m], phases))

    def relax(self, method, f, s, nrelax, w=1.0):
        """Operator_relax (c/operators.cpp:50-92) + bmgs_relax
        (c/bmgs/relax.cpp:8-66).  Real data only."""
        if w is None:
            w = 1.0
        for _ in range(nrelax):
            buf = self.bc.unpack(f, None)
            flat = buf.ravel()
            if method == 1:
                self._gauss_seidel(flat, f, s)
                continue
            x = np.zeros(self._idx.shape, float)
            for c in range(1, len(self.coefs)):
                x = x + flat[self._idx + self.offsets[c]] * self.coefs[c]
            b = f.ravel()
            b[:] = (1.0 - w) * b + w * (s.ravel() - x) / self.coefs[0]

    def _gauss_seidel(self, flat, f, s):
        """Lexicographic Gauss-Seidel (c/bmgs/relax.cpp:12-40), evaluated
        wavefront by wavefront: points whose every earlier-in-order neighbour
        is already updated are computed together.  The result equals the
        sequential loop exactly because no point reads a point of its own
        wavefront."""
        coef = 1.0 / self.coefs[0]
        n0, n1, n2 = self.n
        mp = max(self.r, 1)
        beta = 2 * mp + 1
        alpha = (beta + 1) * mp + 1
        i0, i1, i2 = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2),
                                 indexing='ij')
        t = (alpha * i0 + beta * i1 + i2).ravel()
        order = np.argsort(t, kind='stable')
        ts = t[order]
        bounds = np.flatnonzero(np.diff(ts)) + 1
        groups = np.split(order, bounds)
        b = f.ravel()
        src = s.ravel()
        for g in groups:
            j = self._idx[g]
            x = np.zeros(len(g))
            for c in range(1, len(self.coefs)):
                x = x + flat[j + self.offsets[c]] * self.coefs[c]
            x = (src[g] - x) * coef
            b[g] = x
            flat[j] = x

    def get_diagonal_element(self):
        """c/operators.cpp:319-332: the coefficient at offset 0."""
        d = 0.0
        for c, o in zip(self.coefs, self.offsets):
            if o == 0:
                d = c
        return d


class WOperator:
    """Restatement of the reference ``WOperator`` object
    (c/woperators.cpp:416-460): A = sum_i w_i(x) L_i with per-point
    weights; apply = bmgs_wfd / bmgs_wfdz (c/bmgs/wfd.cpp:10-40), relax =
    bmgs_wrelax (c/bmgs/wrelax.cpp:8-95).  ``weights`` are kept by
    reference, as the reference keeps its array pointers."""

    def __init__(self, nweights, weights, coefs, offsets, size, r, neighbors,
                 real, comm, cfd):
        assert comm is None
        self.nw = int(nweights)
        self.weights = list(weights)
        self.coefs = [np.ascontiguousarray(c, float) for c in coefs]
        self.offsets = [np.ascontiguousarray(o, np.int64) for o in offsets]
        self.n = [int(x) for x in size]
        self.r = int(r)
        pad = np.full((3, 2), self.r, int)
        self.bc = BoundaryConditions(self.n, pad, pad, neighbors, real, cfd)
        n0, n1, n2 = self.n
        M = [x + 2 * self.r for x in self.n]
        i0, i1, i2 = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2),
                                 indexing='ij')
        self._idx = (((i0 + self.r) * M[1] + i1 + self.r) * M[2] +
                     i2 + self.r).ravel()

    def apply(self, inp, out, phases=None):
        """WOperator_apply (c/woperators.cpp:318-370): every grid of the
        batch with the same weights."""
        nin = inp.shape[0] if inp.ndim == 4 else 1
        src = inp.reshape((nin,) + tuple(self.n))
        dst = out.reshape((nin,) + tuple(self.n))
        for m in range(nin):
            flat = self.bc.unpack(src[m], phases).ravel()
            x = np.zeros(self._idx.shape, flat.dtype)
            for iw in range(self.nw):
                tmp = np.zeros(self._idx.shape, flat.dtype)
                for c in range(len(self.coefs[iw])):
                    tmp = tmp + flat[self._idx + self.offsets[iw][c]] * \
                        self.coefs[iw][c]
                tmp = tmp * np.asarray(self.weights[iw]).ravel()
                x = x + tmp
            dst[m] = x.reshape(self.n)

    def _terms(self, flat, j, sel):
        """Off-diagonal sum and diagonal of the points ``sel`` (padded
        indices j), in bmgs_wrelax's order."""
        x = np.zeros(len(j))
        coef = np.zeros(len(j))
        for iw in range(self.nw):
            weight = np.asarray(self.weights[iw]).ravel()[sel]
            tmp = np.zeros(len(j))
            for c in range(1, len(self.coefs[iw])):
                tmp = tmp + flat[j + self.offsets[iw][c]] * self.coefs[iw][c]
            tmp = tmp * weight
            x = x + tmp
            coef = coef + weight * self.coefs[iw][0]
        return x, coef

    def relax(self, method, f, s, nrelax, w=1.0):
        """WOperator_relax (c/woperators.cpp:53-96)."""
        if w is None:
            w = 1.0
        allpts = np.arange(len(self._idx))
        for _ in range(nrelax):
            flat = self.bc.unpack(f, None).ravel()
            b = f.ravel()
            if method == 1:
                n0, n1, n2 = self.n
                mp = max(self.r, 1)
                beta = 2 * mp + 1
                alpha = (beta + 1) * mp + 1
                i0, i1, i2 = np.meshgrid(np.arange(n0), np.arange(n1),
                                         np.arange(n2), indexing='ij')
                t = (alpha * i0 + beta * i1 + i2).ravel()
                order = np.argsort(t, kind='stable')
                ts = t[order]
                groups = np.split(order, np.flatnonzero(np.diff(ts)) + 1)
                for g in groups:
                    j = self._idx[g]
                    x, coef = self._terms(flat, j, g)
                    x = (s.ravel()[g] - x) / coef
                    b[g] = x
                    flat[j] = x
                continue
            x, coef = self._terms(flat, self._idx, allpts)
            b[:] = (1.0 - w) * b + w * (s.ravel() - x) / coef

    def get_diagonal_element(self):
        """c/woperators.cpp:372-398."""
        coef = np.zeros(int(np.prod(self.n)))
        for iw in range(self.nw):
            coef = coef + np.asarray(self.weights[iw]).ravel() * \
                self.coefs[iw][0]
        return float(max(0.0, np.abs(coef).max()))


# --------------------------------------------------------------------------
# Transformer (c/transformers.cpp, c/bmgs/restrict.cpp, interpolate.cpp)
# --------------------------------------------------------------------------
def lagrange_midpoint_weights(k):
    """Weights of the order-k Lagrange interpolant at a midpoint, for the
    symmetric pairs at distance 1/2, 3/2, ... (in units of the coarse
    spacing).  Exact binary fractions; they equal the constants of
    c/bmgs/restrict.cpp:37-57 and c/bmgs/interpolate.cpp:29-40."""
    from fractions import Fraction
    nodes = [Fraction(2 * j - k + 1, 2) for j in range(k)]   # ±1/2, ±3/2 ..
    w = []
    for j in range(k // 2, k):
        num = Fraction(1)
        for m in range(k):
            if m != j:
                num *= (0 - nodes[m]) / (nodes[j] - nodes[m])
        w.append(num)
    return [float(x) for x in w]


def _rst1d(a, K, w):
    """RST1D (c/bmgs/restrict.cpp:18-60): restrict along the last axis of a
    (m, n) view; output (nout, m) is transposed."""
    m, n = a.shape
    nout = (n - K * 2 + 3) // 2
    base = K - 1 + 2 * np.arange(nout)
    x = a[:, base]
    for j, wj in enumerate(w):
        o = 2 * j + 1
        t = wj * (a[:, base + o] + a[:, base - o])
        x = x + t
    return (0.5 * x).T.copy()


def _ip1d(a, K, w, n, skip):
    """IP1D (c/bmgs/interpolate.cpp:10-46) along the last axis of an (m, L)
    view; ``n`` coarse points processed; output (nout, m) transposed."""
    m = a.shape[0]
    base = K // 2 - 1 + np.arange(n)
    even = a[:, base]
    odd = None
    for j, wj in enumerate(w):
        t = wj * (a[:, base - j] + a[:, base + 1 + j])
        odd = t if odd is None else odd + t
    out = np.empty((m, 2 * n), a.dtype)
    out[:, 0::2] = even
    out[:, 1::2] = odd
    lo = 1 if skip[0] else 0
    hi = 2 * n - (1 if skip[1] else 0)
    return out[:, lo:hi].T.copy()


class Transformer:
    """Restatement of the reference ``Transformer`` object
    (c/transformers.cpp:196-246)."""

    def __init__(self, size_in, size_out, k, pads, npads, skip, neighbors,
                 real, comm, interpolate, use_gpu=0):
        assert comm is None
        self.k = int(k)
        self.interpolate = bool(interpolate)
        self.size_in = [int(x) for x in size_in]
        self.size_out = [int(x) for x in size_out]
        self.skip = np.asarray(skip, int).reshape(3, 2)
        self.real = bool(real)
        # transformers always fill edges and corners (cfd=0,
        # c/transformers.cpp:230)
        self.bc = BoundaryConditions(self.size_in, pads, npads, neighbors,
                                     real, cfd=0)
        self.w = lagrange_midpoint_weights(self.k)

    def _one(self, a, phases):
        buf = self.bc.unpack(a, phases)
        s = buf.shape
        K, w = self.k, self.w
        if not self.interpolate:
            # bmgs_restrict (c/bmgs/restrict.cpp:137-156)
            e = 2 * K - 3
            nb = [(s[i] - e) // 2 for i in range(3)]
            t = _rst1d(buf.reshape(s[0] * s[1], s[2]), K, w)
            t = _rst1d(t.reshape(nb[2] * s[0], s[1]), K, w)
            t = _rst1d(t.reshape(nb[1] * nb[2], s[0]), K, w)
            return t.reshape(nb[0], nb[1], nb[2])
        # bmgs_interpolate (c/bmgs/interpolate.cpp:70-99)
        e = K - 1
        sk = self.skip
        n2 = s[2] - e + sk[2, 1]
        t = _ip1d(buf.reshape(s[0] * s[1], s[2]), K, w, n2, sk[2])
        o2 = t.shape[0]
        n1 = s[1] - e + sk[1, 1]
        t = _ip1d(t.reshape(o2 * s[0], s[1]), K, w, n1, sk[1])
        o1 = t.shape[0]
        n0 = s[0] - e + sk[0, 1]
        t = _ip1d(t.reshape(o1 * o2, s[0]), K, w, n0, sk[0])
        return t.reshape(t.shape[0], o1, o2)

    def apply(self, inp, out, phases=None):
        nin = inp.shape[0] if inp.ndim == 4 else 1
        src = inp.reshape((nin,) + tuple(self.size_in))
        dst = out.reshape((nin,) + tuple(self.size_out))
        for m in range(nin):
            dst[m] = self._one(src[m], phases)


# --------------------------------------------------------------------------
# fd_precond (c/fd_preconditioner.cpp:106-351)
# --------------------------------------------------------------------------
def fd_precond(rest0, rest1, intp1, intp2, kin0, kin1, kin2,
               d0, q0, r1, d1, q1, r2, d2, q2,
               residuals, nresiduals, step, phases=None):
    """Three-level V-cycle, same sequence and same scalar factors as the
    reference (4 * step and 16 * step formed in double)."""
    if residuals.ndim == 3:
        residuals = residuals[None]
        nresiduals = nresiduals[None]
    s4 = 4 * step
    s16 = 16 * step
    rest0.apply(nresiduals, r1, phases)
    d1[:] = s4 * r1
    kin1.apply(d1, q1, phases)
    q1 -= r1
    rest1.apply(q1, r2, phases)
    d2[:] = s16 * r2
    kin2.apply(d2, q2, phases)
    q2 -= r2
    d2 -= s16 * q2
    intp2.apply(d2, q1, phases)
    d1 -= q1
    kin1.apply(d1, q1, phases)
    q1 -= r1
    d1 -= s4 * q1
    d1[:] = -d1
    intp1.apply(d1, d0, phases)
    kin0.apply(d0, q0, phases)
    q0 -= residuals
    d0 -= step * q0
    d0[:] = -d0
