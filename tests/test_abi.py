"""The C-ABI library loads without a GPU and exports every entry point that
include/gpaw_b200.h declares, with a binding for each in gpaw_b200._lib."""
import ctypes
import os
import re

import pytest

from gpaw_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, 'include')):
        if not fn.endswith('.h'):
            continue
        text = open(os.path.join(ROOT, 'include', fn)).read()
        text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
        names |= set(re.findall(r'\b(gb_[a-z0-9_]+)\s*\(', text))
    return names


def test_header_declares_entry_points():
    names = declared()
    assert {'gb_operator_new', 'gb_operator_apply', 'gb_operator_relax',
            'gb_transformer_new', 'gb_transformer_apply', 'gb_fd_precond',
            'gb_poisson_new', 'gb_poisson_solve_neutral'} <= names


def test_library_exports_all_symbols():
    lib = _lib.load()
    for name in sorted(declared()):
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name


def test_library_hides_internal_symbols():
    import subprocess
    out = subprocess.run(['nm', '-D', '--defined-only', _lib.LIB_PATH],
                         capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if ' T ' in l}
    gb = {s for s in exported if s.startswith('gb_')}
    assert gb == declared()


def test_errors_map_to_reference_exceptions():
    lib = _lib.load()
    h = ctypes.c_void_p()
    import numpy as np
    coefs, cp = _lib.f64([1.0])
    offs, op = _lib.i64([0])
    size, sp = _lib.i64([4, 4, 4])
    nb, nbp = _lib.i64([[1, 1], [-1, -1], [-1, -1]])
    rc = lib.gb_operator_new(cp, op, 1, sp, 1, nbp, 1, 1, ctypes.byref(h))
    with pytest.raises(ValueError, match='domain decomposition'):
        _lib.check(rc)


def _wop_new(lib, nweights=1, offsets=((0, 1, -1),), range_=1,
             neighbors=((0, 0), (-1, -1), (-1, -1))):
    """gb_woperator_new on host-side dummy weight pointers (construction
    touches no device memory)."""
    import numpy as np
    n = len(offsets)
    keep = []
    C = (ctypes.c_void_p * n)
    cs, os_ = [], []
    for o in offsets:
        ca, cp = _lib.f64([1.0] * len(o))
        oa, op = _lib.i64(o)
        keep += [ca, oa]
        cs.append(ctypes.cast(cp, ctypes.c_void_p))
        os_.append(ctypes.cast(op, ctypes.c_void_p))
    dummy = np.zeros(8)
    W = C(*([dummy.ctypes.data] * n))
    NC = (ctypes.c_int * n)(*[len(o) for o in offsets])
    size, sp = _lib.i64([6, 5, 7])
    nb, nbp = _lib.i64(neighbors)
    h = ctypes.c_void_p()
    rc = lib.gb_woperator_new(nweights, W, C(*cs), C(*os_), NC, sp, range_,
                              nbp, 1, 1, ctypes.byref(h))
    if rc == 0:
        lib.gb_woperator_free(h)
    return rc


def test_woperator_argument_checks():
    """WOperator construction rejects what the reference's WeightedFDOperator
    asserts or cannot run: no operators, an operator whose first offset is
    not the centre, offsets beyond the range, more than one domain."""
    lib = _lib.load()
    assert _wop_new(lib) == 0
    with pytest.raises(ValueError, match='weights'):
        _lib.check(_wop_new(lib, nweights=0))
    with pytest.raises(ValueError, match='offset 0'):
        _lib.check(_wop_new(lib, offsets=((1, 0, -1),)))
    with pytest.raises(ValueError, match='does not fit'):
        _lib.check(_wop_new(lib, offsets=((0, 200),)))
    with pytest.raises(ValueError, match='single-domain'):
        _lib.check(_wop_new(lib, neighbors=((1, 1), (-1, -1), (-1, -1))))
    assert lib.gb_poisson_fused_levels(None) == 0
