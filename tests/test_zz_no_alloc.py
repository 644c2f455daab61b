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


@pytest.mark.parametrize('method', [2, 1])
def test_noalloc_general_cell_twice(method, cuda):
    """A non-orthogonal cell: the stencil is not axis-aligned, so the Jacobi
    sweeps take the generic kernel and Gauss-Seidel the wider wavefront
    spacing; both through the allocation-free entry point."""
    from gpaw_b200 import GridDescriptor, Laplace
    cell = [(3.0, 0, 0), (1.5, 3.0 * 3**0.5 / 2, 0), (0, 0, 3.2)]
    gd = GridDescriptor((18, 18, 16), cell, (1, 1, 0))
    op = Laplace(gd, -0.25 / np.pi, 3)
    assert not op.cfd
    rng = np.random.default_rng(7 + method)
    for call in range(2):
        f = rng.standard_normal(tuple(gd.n_c))
        s = rng.standard_normal(f.shape)
        ref, got = _relax_both(op.operator, method, f, s, 2 + call, 0.6)
        assert np.array_equal(got, ref)


_FIRST_CALL_IN_CAPTURE = r"""
import ctypes as C, sys, torch
sys.path.insert(0, sys.argv[1])
from gpaw_b200 import GridDescriptor, Laplace, _lib
gd = GridDescriptor((20, 20, 20), 4.0, 0)
op = Laplace(gd, -0.25 / 3.141592653589793, 3).operator
f = torch.zeros(tuple(gd.n_c), dtype=torch.float64, device='cuda')
s = torch.ones_like(f)
lib = _lib.load()
side = torch.cuda.Stream()
torch.cuda.synchronize()
g = torch.cuda.CUDAGraph()
with torch.cuda.stream(side):
    with torch.cuda.graph(g, stream=side):
        rc = lib.gb_operator_relax_noalloc(
            op._h, 2, C.c_void_p(f.data_ptr()), C.c_void_p(s.data_ptr()), 2,
            1.0, C.c_void_p(side.cuda_stream))
        msg = lib.gb_last_error().decode()
print(rc, msg)
"""


def test_noalloc_first_call_inside_capture_is_refused(cuda):
    """In a fresh process, a first call made inside a stream capture is
    refused (GB_EINVAL) with a message naming the rule, instead of a CUDA
    error from the address look-up."""
    import os
    import subprocess
    import sys
    from gpaw_b200 import _lib
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, '-c', _FIRST_CALL_IN_CAPTURE, root],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    rc, msg = out.stdout.strip().splitlines()[-1].split(' ', 1)
    assert int(rc) == _lib.GB_EINVAL
    assert 'stream capture' in msg


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
