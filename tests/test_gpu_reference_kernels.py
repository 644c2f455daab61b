"""The reference's own GPU kernels (c/gpu/kernels, built for sm_100a from
its sources into oracle/_ref by `make -C oracle gpu`; bench.py times them
beside this library's) give this library's results: the complex stencil
with Bloch phases, restriction and interpolation of order 6 (the stencil
variants), and the order-2 transfers (the reference's optimised kernels),
within the FP64 bar.  Skipped where that library was not built."""
import ctypes as C
import os

import numpy as np
import pytest

from tests.helpers import RTOL_FP64, max_rel, to_dev, to_np

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, 'oracle', '_ref', 'libgpaw_ref_gpu.so')


def _lib():
    if not os.path.exists(LIB):
        pytest.skip('reference GPU kernels not built')
    lib = C.CDLL(LIB)
    vp, lp, dp = C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_double)
    lib.refgpu_operator_new.restype = vp
    lib.refgpu_operator_new.argtypes = [dp, lp, C.c_int, C.c_int, lp, lp,
                                        C.c_int]
    lib.refgpu_operator_apply.argtypes = [vp, vp, vp, C.c_int, dp]
    lib.refgpu_transformer_new.restype = vp
    lib.refgpu_transformer_new.argtypes = [lp, lp, C.c_int, lp, lp, lp, lp,
                                           C.c_int, C.c_int]
    lib.refgpu_transformer_apply.argtypes = [vp, vp, vp, C.c_int, dp]
    return lib


def _l(a):
    a = np.ascontiguousarray(np.asarray(a).ravel(), np.int64)
    return a, a.ctypes.data_as(C.POINTER(C.c_long))


def _d(a):
    a = np.ascontiguousarray(np.asarray(a, float).ravel())
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.mark.parametrize('pbc,dtype', [((1, 1, 1), complex), ((0, 0, 0), float)])
@pytest.mark.parametrize('nn', [1, 3])
def test_reference_gpu_kernels_match(pbc, dtype, nn, cuda):
    import torch
    from gpaw_b200 import GridDescriptor, Laplace, Transformer
    lib = _lib()
    N = (24, 20, 28)
    gd = GridDescriptor(N, (4.0, 3.4, 4.6), pbc)
    real = int(dtype == float)
    rng = np.random.default_rng(nn)
    a = rng.standard_normal((3,) + tuple(gd.n_c))
    if not real:
        a = a + 1j * rng.standard_normal(a.shape)
    ph = gd.phase_factor_cd((0.25, -0.3, 0.1)) if not real else None
    phv, ph_p = _d(np.column_stack([np.asarray(ph).real.ravel(),
                                    np.asarray(ph).imag.ravel()])) \
        if not real else (None, None)
    x = to_dev(a)
    keep = []
    op = Laplace(gd, -0.5, nn, dtype)
    co, cp = _d(op.coef_p)
    of, opp = _l(op.offset_p)
    sz, szp = _l(gd.n_c)
    ne, nep = _l(gd.neighbor_cd)
    keep += [co, of, sz, ne, phv]
    h = lib.refgpu_operator_new(cp, opp, len(op.coef_p), int(op.mp), szp,
                                nep, real)
    ref = torch.empty_like(x)
    assert lib.refgpu_operator_apply(h, C.c_void_p(x.data_ptr()),
                                     C.c_void_p(ref.data_ptr()), 3,
                                     ph_p) == 0
    got = torch.empty_like(x)
    op.apply(x, got, ph)
    torch.cuda.synchronize()
    assert max_rel(to_np(ref), to_np(got)) <= RTOL_FP64
    for gi, go in ((gd, gd.coarsen()), (gd.coarsen(), gd)):
        t = Transformer(gi, go, nn, dtype)
        si, sip = _l(gi.n_c)
        so, sop = _l(go.n_c)
        pa, pap = _l(t.pad_cd)
        npd, npp = _l(t.neighborpad_cd)
        sk, skp = _l(t.skip_cd)
        nb, nbp = _l(gi.neighbor_cd)
        keep += [si, so, pa, npd, sk, nb]
        ht = lib.refgpu_transformer_new(sip, sop, 2 * nn, pap, npp, skp, nbp,
                                        real, int(t.interpolate))
        inp = x if gi is gd else t_in
        out_ref = torch.empty((3,) + tuple(go.n_c), dtype=x.dtype,
                              device=x.device)
        assert lib.refgpu_transformer_apply(
            ht, C.c_void_p(inp.data_ptr()), C.c_void_p(out_ref.data_ptr()),
            3, ph_p) == 0
        out = t.apply(inp, phases=ph)
        torch.cuda.synchronize()
        assert max_rel(to_np(out_ref), to_np(out)) <= RTOL_FP64, \
            ('interpolate' if t.interpolate else 'restrict')
        t_in = out
