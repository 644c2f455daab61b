"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own C core (built from its sources by
``make -C oracle``) through the restatement of its Python layer in
``oracle/gpaw_layer.py`` on small seeded inputs, and stores inputs and
outputs in ``golden.npz``.  Re-run after changing a case:

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import gpaw_layer as L  # noqa: E402

KPT = (0.25, 0.0, 0.1)


def cases():
    """(name, builder) pairs; every builder returns a dict of arrays."""
    out = []
    # FD apply: nn = 1..6, real/complex, periodic / zero / mixed
    for nn in range(1, 7):
        for bc in ('p', 'z', 'm'):
            for dt in ('f', 'c'):
                out.append((f'fd_nn{nn}_{bc}_{dt}', ('fd', nn, bc, dt)))
    # non-orthorhombic cell (cfd = 0 stencil)
    for dt in ('f', 'c'):
        out.append((f'fd_hex_{dt}', ('fdhex', 2, 'p', dt)))
    # relax
    for m in (1, 2):
        for bc in ('p', 'z'):
            out.append((f'relax_m{m}_{bc}', ('relax', m, bc, 'f')))
    # transformers
    for nn in range(1, 4):
        for bc in ('p', 'z', 'm'):
            for dt in ('f', 'c'):
                out.append((f'tr_nn{nn}_{bc}_{dt}', ('tr', nn, bc, dt)))
    # order 8 needs larger grids (interpolator guard, gpaw/transformers.py:50)
    for bc, dt in (('p', 'f'), ('z', 'f'), ('p', 'c')):
        out.append((f'tr_nn4_{bc}_{dt}', ('tr', 4, bc, dt)))
    # preconditioner
    for bc in ('p', 'z'):
        for dt in ('f', 'c'):
            out.append((f'pc_{bc}_{dt}', ('pc', 3, bc, dt)))
    # Poisson
    for bc in ('p', 'z'):
        out.append((f'ps_{bc}', ('ps', 3, bc, 'f')))
    # FD Hamiltonian local part (appended last: earlier cases keep their
    # random draws)
    for nn, bc, dt in ((3, 'p', 'c'), (3, 'z', 'f'), (2, 'm', 'c'),
                       (1, 'p', 'f')):
        out.append((f'ham_nn{nn}_{bc}_{dt}', ('ham', nn, bc, dt)))
    # Mehrstellen operators and the nn='M' Poisson solver (appended last)
    for bc, dt in (('p', 'f'), ('z', 'f'), ('m', 'c')):
        out.append((f'mst_{bc}_{dt}', ('mst', 0, bc, dt)))
    for bc in ('p', 'z'):
        out.append((f'psM_{bc}', ('psM', 0, bc, 'f')))
    # weighted operator (Laplacian + three gradients, per-point weights;
    # appended last)
    for bc, dt in (('p', 'f'), ('z', 'f'), ('m', 'f'), ('p', 'c'), ('m', 'c')):
        out.append((f'wfd_{bc}_{dt}', ('wfd', 2, bc, dt)))
    return out


def wfd_stencils(gd, nn):
    """(coefs, offsets_pc) of a Laplacian and the three axis gradients
    (4th order, no centre point) used by the weighted-operator cases."""
    lap = L.Laplace(gd, 0.4, nn)
    ops = [(lap.coef_p, lap.offset_pc)]
    h = np.diag(gd.h_cv)
    for c in range(3):
        e = np.zeros(3, int)
        e[c] = 1
        ops.append((np.array([2 / 3, -1 / 12, -2 / 3, 1 / 12]) / h[c],
                    np.array([e, 2 * e, -e, -2 * e])))
    return ops


def pbc_of(bc):
    return {'p': (1, 1, 1), 'z': (0, 0, 0), 'm': (1, 0, 1)}[bc]


def build(kind, nn, bc, dt, rng):
    dtype = float if dt == 'f' else complex
    pbc = pbc_of(bc)
    d = {}

    def rand(shape):
        a = rng.standard_normal(shape)
        if dtype == complex:
            a = a + 1j * rng.standard_normal(shape)
        return a

    if kind in ('fd', 'fdhex'):
        N = (8, 7, 9) if kind == 'fd' else (8, 8, 6)
        cell = (3.1, 2.9, 3.5) if kind == 'fd' else \
            [(3.0, 0, 0), (1.5, 3.0 * 3**0.5 / 2, 0), (0, 0, 3.2)]
        gd = L.GridDescriptor(N, cell, pbc)
        op = L.Laplace(gd, -0.5, nn, dtype, be='ref')
        a = rand((1,) + tuple(gd.n_c))
        ph = gd.phase_factor_cd(KPT) if dtype == complex else None
        b = np.zeros_like(a)
        op.apply(a, b, ph)
        d.update(N=np.array(N), cell=np.array(cell, float), pbc=np.array(pbc),
                 inp=a, out=b, coefs=op.coef_p, offsets=op.offset_pc)
        if ph is not None:
            d['phases'] = ph
    elif kind == 'relax':
        gd = L.GridDescriptor((8, 7, 9), (3.0, 2.6, 3.3), pbc)
        op = L.Laplace(gd, -0.25 / np.pi, 3, be='ref')
        f = rand(tuple(gd.n_c))
        s = rand(tuple(gd.n_c))
        g = f.copy()
        op.relax(nn, g, s, 3, 2.0 / 3.0)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), f=f, s=s, out=g)
    elif kind == 'tr':
        N = {1: (12, 10, 8), 2: (12, 10, 8), 3: (16, 14, 8), 4: (20, 18, 8)}[nn]
        gd = L.GridDescriptor(N, (3.0, 3.4, 3.9), pbc)
        gd2 = gd.coarsen()
        ph = gd.phase_factor_cd(KPT) if dtype == complex else None
        a = rand((1,) + tuple(gd.n_c))
        r = L.Transformer(gd, gd2, nn, dtype, be='ref').apply(a, phases=ph)
        c = rand((1,) + tuple(gd2.n_c))
        i = L.Transformer(gd2, gd, nn, dtype, be='ref').apply(c, phases=ph)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), fine=a,
                 restricted=r, coarse=c, interpolated=i)
        if ph is not None:
            d['phases'] = ph
    elif kind == 'pc':
        gd = L.GridDescriptor((8, 8, 12), (3.0, 3.0, 4.5), pbc)
        kin = L.Laplace(gd, -0.5, nn, dtype, be='ref')
        pc = L.Preconditioner(gd, kin, dtype, block=2, be='ref')
        R = rand((3,) + tuple(gd.n_c))
        ph = gd.phase_factor_cd(KPT) if dtype == complex else None
        o = np.zeros_like(R)
        pc(R, ph, out=o)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), res=R, out=o)
        if ph is not None:
            d['phases'] = ph
    elif kind == 'ham':
        gd = L.GridDescriptor((10, 9, 12), (3.0, 2.8, 3.6), pbc)
        ham = L.FDHamiltonian(gd, nn, dtype, be='ref')
        psit = rand((3,) + tuple(gd.n_c))
        vt = rng.standard_normal(tuple(gd.n_c))
        ph = gd.phase_factor_cd(KPT) if dtype == complex else None
        out = np.zeros_like(psit)
        ham.apply_local_potential(vt, psit, out, ph)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), psit=psit, vt=vt,
                 out=out)
        if ph is not None:
            d['phases'] = ph
    elif kind == 'mst':
        gd = L.GridDescriptor((10, 12, 9), (3.0, 3.3, 2.8), pbc)
        a = rand((2,) + tuple(gd.n_c))
        ph = gd.phase_factor_cd(KPT) if dtype == complex else None
        oa = np.zeros_like(a)
        ob = np.zeros_like(a)
        L.LaplaceA(gd, 0.3, dtype, be='ref').apply(a, oa, ph)
        L.LaplaceB(gd, dtype, be='ref').apply(a, ob, ph)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), inp=a, outA=oa,
                 outB=ob)
        if ph is not None:
            d['phases'] = ph
    elif kind == 'psM':
        gd = L.GridDescriptor((16, 16, 8), (4.0, 4.0, 2.0), pbc)
        x = gd.get_grid_point_coordinates()
        rho = np.exp(-((x[0] - 2) ** 2 + (x[1] - 1.9) ** 2 +
                       (x[2] - 1.1) ** 2) / 0.6) - \
            np.exp(-((x[0] - 1.6) ** 2 + (x[1] - 2.3) ** 2 +
                     (x[2] - 0.9) ** 2) / 0.6)
        rho = rho - rho.mean()
        ps = L.FDPoissonSolver(nn='M', eps=1e-18, be='ref')
        ps.set_grid_descriptor(gd)
        phi = gd.zeros()
        niter = ps.solve(phi, rho)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), rho=rho, phi=phi,
                 niter=np.array(niter), errors=np.array(ps.errors))
    elif kind == 'wfd':
        gd = L.GridDescriptor((9, 8, 10), (3.1, 2.7, 3.4), pbc)
        st = wfd_stencils(gd, nn)
        ops = [L.FDOperator(c, o, gd, dtype, be='ref') for c, o in st]
        wop = L.WeightedFDOperator(ops, be='ref')
        w = [rng.uniform(1.0, 2.0, tuple(gd.n_c))] + \
            [rng.standard_normal(tuple(gd.n_c)) for _ in range(3)]
        wop.set_weights(w)
        a = rand((2,) + tuple(gd.n_c))
        ph = gd.phase_factor_cd(KPT) if dtype == complex else None
        b = np.zeros_like(a)
        wop.apply(a, b, ph)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), inp=a, out=b,
                 diag=np.array(wop.get_diagonal_element()))
        for i, (c, o) in enumerate(st):
            d[f'coefs{i}'] = np.asarray(c, float)
            d[f'offsets{i}'] = np.asarray(o, int)
            d[f'w{i}'] = w[i]
        if ph is not None:
            d['phases'] = ph
        if dtype == float:
            f = rng.standard_normal(tuple(gd.n_c))
            src = rng.standard_normal(tuple(gd.n_c))
            for m in (1, 2):
                g = f.copy()
                wop.relax(m, g, src, 2, 0.6)
                d[f'relax{m}'] = g
            d.update(f=f, s=src)
    elif kind == 'ps':
        gd = L.GridDescriptor((16, 8, 16), (4.0, 2.0, 4.0), pbc)
        x = gd.get_grid_point_coordinates()
        rho = np.exp(-((x[0] - 2) ** 2 + (x[1] - 0.9) ** 2 +
                       (x[2] - 2.1) ** 2) / 0.5) - \
            np.exp(-((x[0] - 1.5) ** 2 + (x[1] - 1.1) ** 2 +
                     (x[2] - 2.1) ** 2) / 0.5)
        rho = rho - rho.mean()
        ps = L.FDPoissonSolver(nn=nn, eps=1e-18, be='ref')
        ps.set_grid_descriptor(gd)
        phi = gd.zeros()
        niter = ps.solve(phi, rho)
        d.update(N=np.array(gd.N_c), pbc=np.array(pbc), rho=rho, phi=phi,
                 niter=np.array(niter), errors=np.array(ps.errors))
    return d


def main():
    if L._REF is None:
        raise SystemExit('reference core not built: make -C oracle')
    rng = np.random.default_rng(20261203)
    data = {}
    for name, (kind, nn, bc, dt) in cases():
        for k, v in build(kind, nn, bc, dt, rng).items():
            data[f'{name}/{k}'] = v
    path = os.path.join(HERE, 'golden.npz')
    np.savez_compressed(path, **data)
    print(path, os.path.getsize(path), 'bytes', len(cases()), 'cases')


if __name__ == '__main__':
    main()
