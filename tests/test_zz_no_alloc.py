"""gb_operator_relax_noalloc: the relaxation entry point that allocates no
device memory (its scratch grid is a fixed device array), for callers that
cannot let the library call cudaMalloc.

Checked through the C ABI against gb_operator_relax on two calls in a row
(the shared array keeps the first call's contents when the second starts).
This file is collected last, so that a run stopping at the first failure has
run every other test already."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import RTOL_FP64, max_rel, to_dev, to_np

pytestmark = pytest.mark.gpu


def _relax_both(op, method, f0, s0, nrelax, w):
    import torch
    from gpaw_b200 import _lib
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    a, b = to_dev(f0), to_dev(f0)
    s = to_dev(s0)
    _lib.check(lib.gb_operator_relax(op._h, method, C.c_void_p(a.data_ptr()),
                                     C.c_void_p(s.data_ptr()), nrelax, w,
                                     stream))
    _lib.check(lib.gb_operator_relax_noalloc(
        op._h, method, C.c_void_p(b.data_ptr()), C.c_void_p(s.data_ptr()),
        nrelax, w, stream))
    return to_np(a), to_np(b)


@pytest.mark.parametrize('method,pbc', [(2, 0), (2, 1), (1, 1), (1, 0)])
def test_noalloc_matches_relax_twice(method, pbc, cuda):
    from gpaw_b200 import GridDescriptor, Laplace
    gd = GridDescriptor((40, 36, 34), (6.0, 5.5, 5.0), pbc)
    op = Laplace(gd, -0.25 / np.pi, 3).operator
    rng = np.random.default_rng(42 + method)
    for call in range(2):
        f = rng.standard_normal(tuple(gd.n_c))
        s = rng.standard_normal(f.shape)
        ref, got = _relax_both(op, method, f, s, 3 if call == 0 else 2,
                               2.0 / 3.0)
        assert max_rel(got, ref) <= RTOL_FP64
        assert np.array_equal(got, ref)


def test_noalloc_rejects_large_grid(cuda):
    import torch
    from gpaw_b200 import GridDescriptor, Laplace, _lib
    gd = GridDescriptor((130, 130, 130), 20.0, 1)   # 2.2 M points > limit
    op = Laplace(gd, 1.0, 1).operator
    f = torch.zeros(tuple(gd.n_c), dtype=torch.float64, device='cuda')
    rc = _lib.load().gb_operator_relax_noalloc(
        op._h, 2, C.c_void_p(f.data_ptr()), C.c_void_p(f.data_ptr()), 1, 1.0,
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    with pytest.raises(ValueError, match='more than the'):
        _lib.check(rc)
