"""Complex128 kernels whose input planes arrive by TMA tensor copies
(restriction, interpolation and the plane-marching stencil kernel;
GPAW_B200_TMA=0 selects the per-thread cp.async staging):
both paths against the oracle, bit for bit, on grids that exercise the
window edges (periodic wrap with Bloch phases on every axis, zero and mixed
boundaries, odd sizes, tiles cut by the grid's edge, batches) and the
fallback for tiles with more wrapped cells than the TMA kernel deals out."""
import os

import numpy as np
import pytest

from oracle import gpaw_layer as L
from tests.helpers import to_dev, to_np

pytestmark = pytest.mark.gpu

CASES = [
    # N, pbc, nn, batch
    ((96, 96, 96), (1, 1, 1), 3, 2),
    ((40, 36, 44), (1, 1, 1), 3, 3),
    ((40, 36, 44), (0, 0, 0), 3, 2),
    ((40, 36, 44), (1, 0, 1), 2, 2),
    ((34, 50, 26), (0, 1, 1), 1, 1),
    ((24, 24, 24), (1, 1, 1), 4, 2),
    ((16, 12, 20), (1, 1, 1), 3, 2),   # small: falls back to cp.async
    ((70, 20, 66), (1, 1, 0), 3, 1),
]


def _interp(gdp, nn, c, ph, tma):
    from gpaw_b200 import Transformer
    old = os.environ.get('GPAW_B200_TMA_INTERP')
    os.environ['GPAW_B200_TMA_INTERP'] = '1' if tma else '0'
    try:
        t = Transformer(gdp.coarsen(), gdp, nn, complex)
        return to_np(t.apply(to_dev(c), phases=ph))
    finally:
        if old is None:
            del os.environ['GPAW_B200_TMA_INTERP']
        else:
            os.environ['GPAW_B200_TMA_INTERP'] = old


def _restrict(gdp, nn, a, ph, tma):
    from gpaw_b200 import Transformer
    old = os.environ.get('GPAW_B200_TMA')
    os.environ['GPAW_B200_TMA'] = '1' if tma else '0'
    try:
        t = Transformer(gdp, gdp.coarsen(), nn, complex)
        return to_np(t.apply(to_dev(a), phases=ph))
    finally:
        if old is None:
            del os.environ['GPAW_B200_TMA']
        else:
            os.environ['GPAW_B200_TMA'] = old


@pytest.mark.parametrize('N,pbc,nn,nb', CASES)
def test_transfers_tma_against_oracle(N, pbc, nn, nb, cuda):
    from gpaw_b200 import GridDescriptor, _lib
    cell = tuple(0.2 * n for n in N)
    gdp = GridDescriptor(N, cell, pbc)
    gdo = L.GridDescriptor(N, cell, pbc)
    rng = np.random.default_rng(sum(N) + nn)
    a = rng.standard_normal((nb,) + tuple(gdo.n_c)) + \
        1j * rng.standard_normal((nb,) + tuple(gdo.n_c))
    ph = gdo.phase_factor_cd((0.25, -0.3, 0.1))
    ref = L.Transformer(gdo, gdo.coarsen(), nn, complex).apply(a, phases=ph)
    got_tma = _restrict(gdp, nn, a, ph, True)
    got_cp = _restrict(gdp, nn, a, ph, False)
    assert np.array_equal(got_tma, ref)
    assert np.array_equal(got_cp, ref)
    gc = gdo.coarsen()
    c = rng.standard_normal((nb,) + tuple(gc.n_c)) + \
        1j * rng.standard_normal((nb,) + tuple(gc.n_c))
    ref = L.Transformer(gc, gdo, nn, complex).apply(c, phases=ph)
    assert np.array_equal(_interp(gdp, nn, c, ph, True), ref)
    assert np.array_equal(_interp(gdp, nn, c, ph, False), ref)
    code = _lib.C.c_int(-1)
    _lib.check(_lib.load().gb_device_fault(_lib.C.byref(code)))
    assert code.value == 0


APPLY_CASES = [
    # N, pbc, nn, batch
    ((96, 96, 96), (1, 1, 1), 3, 2),
    ((40, 36, 44), (1, 1, 1), 3, 2),
    ((40, 36, 44), (0, 0, 0), 3, 2),
    ((33, 17, 70), (1, 0, 1), 2, 3),
    ((21, 50, 26), (0, 1, 1), 1, 1),
    ((24, 24, 24), (1, 1, 1), 6, 2),
    ((12, 6, 9), (1, 1, 1), 3, 2),     # smaller than a tile and its halo
    ((70, 20, 66), (1, 1, 0), 4, 1),
]


def _with_tma(flag, fn):
    old = os.environ.get('GPAW_B200_TMA')
    os.environ['GPAW_B200_TMA'] = '1' if flag else '0'
    try:
        return fn()
    finally:
        if old is None:
            del os.environ['GPAW_B200_TMA']
        else:
            os.environ['GPAW_B200_TMA'] = old


@pytest.mark.parametrize('N,pbc,nn,nb', APPLY_CASES)
def test_apply_tma_against_oracle(N, pbc, nn, nb, cuda):
    """The complex stencil apply, its fused potential term and the
    preconditioner step (the plane-marching kernel's complex modes) with
    TMA tiles and with cp.async tiles against the oracle."""
    from gpaw_b200 import FDHamiltonian, GridDescriptor, Laplace
    cell = tuple(0.2 * n for n in N)
    gdp = GridDescriptor(N, cell, pbc)
    gdo = L.GridDescriptor(N, cell, pbc)
    rng = np.random.default_rng(sum(N) * nn)
    shape = (nb,) + tuple(gdo.n_c)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ph = gdo.phase_factor_cd((0.25, -0.3, 0.1))
    ref = np.zeros_like(a)
    L.Laplace(gdo, -0.5, nn, complex).apply(a, ref, ph)
    op = Laplace(gdp, -0.5, nn, complex)
    x = to_dev(a)
    for flag in (True, False):
        y = x.new_zeros(x.shape)
        _with_tma(flag, lambda: op.apply(x, y, ph))
        assert np.array_equal(to_np(y), ref), flag
    if nn == 3:
        vt = rng.standard_normal(tuple(gdo.n_c))
        refh = np.zeros_like(a)
        L.FDHamiltonian(gdo, 3, complex).apply_local_potential(vt, a, refh, ph)
        ham = FDHamiltonian(gdp, kin_stencil=3, dtype=complex)
        for flag in (True, False):
            y = x.new_zeros(x.shape)
            _with_tma(flag, lambda: ham.apply_local_potential(to_dev(vt), x, y,
                                                             ph))
            assert np.array_equal(to_np(y), refh), flag
    from gpaw_b200 import _lib
    code = _lib.C.c_int(-1)
    _lib.check(_lib.load().gb_device_fault(_lib.C.byref(code)))
    assert code.value == 0


@pytest.mark.parametrize('pbc', [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
def test_preconditioner_tma_against_oracle(pbc, cuda):
    from gpaw_b200 import GridDescriptor, Laplace, Preconditioner
    N, cell = (48, 40, 56), (5.0, 4.2, 5.8)
    gdp = GridDescriptor(N, cell, pbc)
    gdo = L.GridDescriptor(N, cell, pbc)
    rng = np.random.default_rng(3)
    R = rng.standard_normal((3,) + tuple(gdo.n_c)) + \
        1j * rng.standard_normal((3,) + tuple(gdo.n_c))
    ph = gdo.phase_factor_cd((0.25, -0.3, 0.1))
    ref = np.zeros_like(R)
    L.Preconditioner(gdo, L.Laplace(gdo, -0.5, 3, complex), complex,
                     block=3)(R, ph, out=ref)
    pc = Preconditioner(gdp, Laplace(gdp, -0.5, 3, complex), complex, block=3)
    for flag in (True, False):
        out = to_dev(np.zeros_like(R))
        _with_tma(flag, lambda: pc(to_dev(R), ph, out=out))
        assert np.array_equal(to_np(out), ref), flag
