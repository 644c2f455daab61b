"""ctypes binding of the gpaw_b200 C ABI (include/gpaw_b200.h).

The shared library is built in-tree by ``python -m gpaw_b200.build``.  There
is no fallback: if the library is missing or CUDA is unavailable, every call
raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_lib', 'libgpaw_b200.so')

GB_OK, GB_EINVAL, GB_ECUDA, GB_ENOCONV = 0, 1, 2, 3
GB_F64, GB_C128 = 0, 1

_p = C.c_void_p
_i64p = C.POINTER(C.c_int64)
_dp = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    'gb_version': (C.c_int, []),
    'gb_last_error': (C.c_char_p, []),
    'gb_operator_new': (C.c_int, [_dp, _i64p, C.c_int, _i64p, C.c_int, _i64p,
                                  C.c_int, C.c_int, C.POINTER(_p)]),
    'gb_operator_free': (None, [_p]),
    'gb_operator_apply': (C.c_int, [_p, _p, _p, C.c_int64, C.c_int, _dp, _p]),
    'gb_operator_set_chunk': (C.c_int, [_p, C.c_int]),
    'gb_transformer_set_chunk': (C.c_int, [_p, C.c_int]),
    'gb_operator_apply_potential': (C.c_int, [_p, _p, _p, C.c_int64, C.c_int,
                                              _dp, _p, _p]),
    'gb_operator_relax': (C.c_int, [_p, C.c_int, _p, _p, C.c_int, C.c_double,
                                    _p]),
    'gb_operator_relax_noalloc': (C.c_int, [_p, C.c_int, _p, _p, C.c_int,
                                            C.c_double, _p]),
    'gb_operator_residual': (C.c_int, [_p, _p, _p, _p, C.c_int64, C.c_int,
                                       _dp, C.c_double, _p, _p]),
    'gb_operator_get_diagonal_element': (C.c_double, [_p]),
    'gb_trace_begin': (C.c_int, [C.c_int]),
    'gb_device_fault': (C.c_int, [C.POINTER(C.c_int)]),
    'gb_pool_set': (C.c_int, [C.c_int, C.c_size_t]),
    'gb_pool_release': (C.c_int, []),
    'gb_pool_stats': (C.c_int, [C.POINTER(C.c_size_t),
                                C.POINTER(C.c_size_t)]),
    'gb_mixed_vcycle_eager': (C.c_int, [_p, _p, _p, _p]),
    'gb_mixed_set_fused_coarse': (C.c_int, [_p, C.c_int]),
    'gb_trace_end': (C.c_int, [C.c_int, C.POINTER(C.c_float),
                               C.POINTER(C.c_char_p), C.POINTER(C.c_int)]),
    'gb_operator_reserve': (C.c_int, [_p, C.c_int64, C.c_int]),
    'gb_transformer_new': (C.c_int, [_i64p, _i64p, C.c_int, _i64p, _i64p,
                                     _i64p, _i64p, C.c_int, C.c_int,
                                     C.POINTER(_p)]),
    'gb_transformer_free': (None, [_p]),
    'gb_transformer_apply': (C.c_int, [_p, _p, _p, C.c_int64, C.c_int, _dp,
                                       _p]),
    'gb_fd_precond': (C.c_int, [_p] * 7 + [_p] * 8 + [_p, _p, C.c_int64,
                                                       C.c_int, C.c_double,
                                                       _dp, _p]),
    'gb_poisson_new': (C.c_int, [C.c_int, C.POINTER(_p), C.POINTER(_p),
                                 C.POINTER(_p), C.POINTER(C.c_int),
                                 C.POINTER(C.c_int), _dp, C.c_int,
                                 C.c_double, C.POINTER(_p)]),
    'gb_poisson_free': (None, [_p]),
    'gb_poisson_fused_levels': (C.c_int, [_p]),
    'gb_woperator_new': (C.c_int, [C.c_int, _p, _p, _p, _p, _p, C.c_int, _p,
                                   C.c_int, C.c_int, _p]),
    'gb_woperator_free': (None, [_p]),
    'gb_woperator_apply': (C.c_int, [_p, _p, _p, C.c_int64, C.c_int, _p, _p]),
    'gb_woperator_relax': (C.c_int, [_p, C.c_int, _p, _p, C.c_int, C.c_double,
                                     _p]),
    'gb_woperator_get_diagonal_element': (C.c_int, [_p, _p, _p]),
    'gb_mixed_new': (C.c_int, [C.c_int, _p, C.POINTER(_p), C.POINTER(_p),
                               C.POINTER(_p), _dp, C.c_double, C.c_int,
                               C.POINTER(_p)]),
    'gb_mixed_free': (None, [_p]),
    'gb_mixed_batch_new': (C.c_int, [C.c_int, C.POINTER(_p), C.c_double,
                                     C.c_int, C.POINTER(_p)]),
    'gb_mixed_batch_free': (None, [_p]),
    'gb_mixed_batch_solve_async': (C.c_int, [_p, C.POINTER(_p),
                                             C.POINTER(_p), _p]),
    'gb_mixed_batch_result': (C.c_int, [_p, C.POINTER(C.c_int), _dp]),
    'gb_mixed_solve_async': (C.c_int, [_p, _p, _p, C.c_double, C.c_int, _p]),
    'gb_mixed_prepare': (C.c_int, [_p]),
    'gb_mixed_result': (C.c_int, [_p, C.POINTER(C.c_int), _dp]),
    'gb_poisson_solve_neutral_async': (C.c_int, [_p, _p, _p, C.c_double,
                                                 C.c_int, _p]),
    'gb_poisson_result': (C.c_int, [_p, C.POINTER(C.c_int), _dp]),
    'gb_mixed_solve': (C.c_int, [_p, _p, _p, C.c_double, C.c_int,
                                 C.POINTER(C.c_int), _dp, _p]),
    'gb_poisson_iterate': (C.c_int, [_p, _p, _p, _dp, _p]),
    'gb_poisson_solve_neutral': (C.c_int, [_p, _p, _p, C.c_double, C.c_int,
                                           C.POINTER(C.c_int), _dp, _p]),
}

_lib = None


class PoissonConvergenceError(RuntimeError):
    """Raised when the V-cycle loop reaches maxiter (gpaw/poisson.py:487)."""


def load():
    """Load the library (once) and bind every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f'gpaw_b200 CUDA library not built ({LIB_PATH}); run '
            '`python -m gpaw_b200.build`')
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc):
    """Map a C-ABI status to the reference's exception types."""
    if rc == GB_OK:
        return
    msg = load().gb_last_error().decode(errors='replace')
    if rc == GB_EINVAL:
        raise ValueError(msg)
    if rc == GB_ENOCONV:
        raise PoissonConvergenceError(msg)
    raise RuntimeError(msg)


class KernelTrace:
    """Per-kernel device times of composite calls (gb_fd_precond), through
    the library's kernel trace:

        with KernelTrace() as tr:
            precond(R, None, out=out)
        tr.intervals   # [(label, ms), ...] in launch order
    """

    def __init__(self, capacity=4096):
        self.capacity = int(capacity)
        self.intervals = []

    def __enter__(self):
        check(load().gb_trace_begin(self.capacity))
        return self

    def __exit__(self, *exc):
        n = self.capacity
        ms = (C.c_float * n)()
        labels = (C.c_char_p * n)()
        count = C.c_int(0)
        check(load().gb_trace_end(n, ms, labels, C.byref(count)))
        self.intervals = [(labels[i].decode(), float(ms[i]))
                          for i in range(min(count.value, n))]
        return False


def set_solver_pool(on=True, cache_limit=16 << 30):
    """Switch the library's caching allocator of solver objects on or off
    (gb_pool_set).  With it on, drop a solver only when none of its work
    is in flight."""
    check(load().gb_pool_set(int(bool(on)), int(cache_limit)))


class solver_pool:
    """Context manager: the solver-object pool on inside, its previous
    state (off by default) restored on exit.  Objects built inside may be
    dropped later; drop them only when none of their work is in flight."""

    _depth = 0

    def __init__(self, cache_limit=16 << 30):
        self.cache_limit = int(cache_limit)

    def __enter__(self):
        if solver_pool._depth == 0:
            set_solver_pool(True, self.cache_limit)
        solver_pool._depth += 1
        return self

    def __exit__(self, *exc):
        solver_pool._depth -= 1
        if solver_pool._depth == 0:
            set_solver_pool(False)
        return False


def solver_pool_stats():
    """(bytes handed out, bytes cached) of the solver-object pool."""
    live, cached = C.c_size_t(0), C.c_size_t(0)
    check(load().gb_pool_stats(C.byref(live), C.byref(cached)))
    return live.value, cached.value


def release_solver_pool():
    """Return every cached block of the pool to the driver."""
    check(load().gb_pool_release())


def i64(a):
    a = np.ascontiguousarray(np.asarray(a).ravel(), np.int64)
    return a, a.ctypes.data_as(_i64p)


def f64(a):
    a = np.ascontiguousarray(np.asarray(a, float).ravel())
    return a, a.ctypes.data_as(_dp)


def phases_arg(phases):
    """(3, 2) complex phase_cd -> 12 doubles, or NULL."""
    if phases is None:
        return None, None
    ph = np.ascontiguousarray(np.asarray(phases, complex).reshape(3, 2))
    buf = ph.view(float).ravel().copy()
    return buf, buf.ctypes.data_as(_dp)
