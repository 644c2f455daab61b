"""C-object layer with the reference extension's signatures.

Mirrors the three hot-path objects of ``gpaw.cgpaw`` (c/_gpaw.h:182-194):

* ``Operator``    — NewOperatorObject, c/operators.cpp:379-420
* ``Transformer`` — NewTransformerObject, c/transformers.cpp:196-246
* ``fd_precond``  — c/fd_preconditioner.cpp:106-351

Array arguments are torch CUDA tensors (or, for the ``*_gpu`` methods, raw
device pointers, as the reference's ``apply_gpu`` takes ``in.data.ptr``).
Every call is enqueued on torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import GB_C128, GB_F64, check, f64, i64, phases_arg


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dtype_code(dtype):
    if dtype in (float, np.float64, torch.float64, np.dtype('float64')):
        return GB_F64
    if dtype in (complex, np.complex128, torch.complex128,
                 np.dtype('complex128')):
        return GB_C128
    raise TypeError(f'unsupported dtype {dtype}')


def _check_tensor(a, name):
    if not isinstance(a, torch.Tensor):
        raise TypeError(f'{name}: expected a torch CUDA tensor, got {type(a)}')
    if not a.is_cuda:
        raise TypeError(f'{name}: tensor must live on a CUDA device')
    if not a.is_contiguous():
        raise TypeError(f'{name}: tensor must be C-contiguous')


def _nin(shape):
    return int(shape[0]) if len(shape) == 4 else 1


class Operator:
    """Stencil object: ``Operator(coefs, offsets, size, range, neighbors,
    real, comm, cfd, use_gpu=1)``."""

    def __init__(self, coefs, offsets, size, range, neighbors, real, comm,
                 cfd, use_gpu=1):
        if comm is not None:
            raise NotImplementedError('domain decomposition (comm) is not '
                                      'supported: one grid per GPU')
        lib = _lib.load()
        coefs_a, coefs_p = f64(coefs)
        offs_a, offs_p = i64(offsets)
        if len(coefs_a) != len(offs_a):
            raise TypeError('coefs and offsets differ in length')
        size_a, size_p = i64(size)
        nb_a, nb_p = i64(neighbors)
        h = C.c_void_p()
        check(lib.gb_operator_new(coefs_p, offs_p, len(coefs_a), size_p,
                                  int(range), nb_p, int(bool(real)),
                                  int(bool(cfd)), C.byref(h)))
        self._h = h
        self._lib = lib
        self.size = tuple(int(x) for x in size_a)
        self.real = bool(real)

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value:
            self._lib.gb_operator_free(h)
            self._h = None

    # -- reference GPU entry points (raw device pointers) ------------------
    def apply_gpu(self, in_ptr, out_ptr, shape, dtype, phases=None):
        """Operator_apply_gpu (c/gpu/operators.cpp:344-385)."""
        ph, ph_p = phases_arg(phases)
        check(self._lib.gb_operator_apply(
            self._h, C.c_void_p(in_ptr), C.c_void_p(out_ptr), _nin(shape),
            _dtype_code(dtype), ph_p, _stream()))

    def relax_gpu(self, relax_method, f_ptr, s_ptr, nrelax, w=1.0):
        """Operator_relax_gpu (c/gpu/operators.cpp:200-221)."""
        check(self._lib.gb_operator_relax(
            self._h, int(relax_method), C.c_void_p(f_ptr), C.c_void_p(s_ptr),
            int(nrelax), float(1.0 if w is None else w), _stream()))

    # -- tensor conveniences ------------------------------------------------
    def apply(self, input, output, phases=None):
        _check_tensor(input, 'input')
        _check_tensor(output, 'output')
        if input.shape != output.shape or input.dtype != output.dtype:
            raise TypeError('input and output differ in shape or dtype')
        if tuple(input.shape[-3:]) != self.size:
            raise TypeError(f'grid shape {tuple(input.shape[-3:])} != '
                            f'{self.size}')
        self.apply_gpu(input.data_ptr(), output.data_ptr(),
                       tuple(input.shape), input.dtype, phases)

    def apply_potential(self, input, output, v, phases=None):
        """output = L input + input * v (v: float64 grid shared by the
        batch) in one pass; FDHamiltonian.apply_local_potential's
        arithmetic (gpaw/new/fd/hamiltonian.py:23-32)."""
        _check_tensor(input, 'input')
        _check_tensor(output, 'output')
        _check_tensor(v, 'v')
        if input.shape != output.shape or input.dtype != output.dtype:
            raise TypeError('input and output differ in shape or dtype')
        if tuple(input.shape[-3:]) != self.size or \
                tuple(v.shape) != self.size:
            raise TypeError('apply_potential: grid shapes do not match')
        if v.dtype != torch.float64:
            raise TypeError('apply_potential: v must be float64')
        ph, ph_p = phases_arg(phases)
        check(self._lib.gb_operator_apply_potential(
            self._h, C.c_void_p(input.data_ptr()),
            C.c_void_p(output.data_ptr()), _nin(input.shape),
            _dtype_code(input.dtype), ph_p, C.c_void_p(v.data_ptr()),
            _stream()))

    def relax(self, relax_method, f, s, nrelax, w=1.0):
        _check_tensor(f, 'f')
        _check_tensor(s, 's')
        if tuple(f.shape) != self.size or tuple(s.shape) != self.size:
            raise TypeError('relax: arrays must have the grid shape')
        if f.dtype != torch.float64 or s.dtype != torch.float64:
            raise TypeError('relax: float64 arrays only')
        self.relax_gpu(relax_method, f.data_ptr(), s.data_ptr(), nrelax, w)

    def residual(self, phi, rho, r=None, phases=None, scale=None, norm2=None):
        """r = L(phi) - rho; optional per-grid scale * sum |r|^2 into
        ``norm2`` (a float64 CUDA tensor of length nin)."""
        _check_tensor(phi, 'phi')
        _check_tensor(rho, 'rho')
        nin = _nin(phi.shape)
        ph, ph_p = phases_arg(phases)
        check(self._lib.gb_operator_residual(
            self._h, C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()),
            C.c_void_p(r.data_ptr() if r is not None else None), nin,
            _dtype_code(phi.dtype), ph_p, float(scale or 1.0),
            C.c_void_p(norm2.data_ptr() if norm2 is not None else None),
            _stream()))

    def reserve(self, nin, dtype):
        check(self._lib.gb_operator_reserve(self._h, int(nin),
                                            _dtype_code(dtype)))

    def get_diagonal_element(self):
        return self._lib.gb_operator_get_diagonal_element(self._h)

    def set_chunk(self, chunk):
        """Axis-0 planes per CTA of the plane-marching kernels (0 = the
        automatic rule); results do not depend on it."""
        check(self._lib.gb_operator_set_chunk(self._h, int(chunk)))

    def get_async_sizes(self):
        # c/operators.cpp:335-345 without GPAW_ASYNC
        return (0, 1, 1)


class WOperator:
    """Weighted stencil object: ``WOperator(nweights, weights, coefs,
    offsets, size, range, neighbors, real, comm, cfd)``
    (NewWOperatorObject, c/woperators.cpp:416-460).  ``weights``: float64
    CUDA tensors of the grid shape, one per operator, kept by reference as
    the reference keeps its arrays."""

    def __init__(self, nweights, weights, coefs, offsets, size, range,
                 neighbors, real, comm, cfd):
        if comm is not None:
            raise NotImplementedError('domain decomposition (comm) is not '
                                      'supported: one grid per GPU')
        nweights = int(nweights)
        if not (len(weights) == len(coefs) == len(offsets) == nweights):
            raise TypeError('weights, coefs and offsets need nweights items')
        lib = _lib.load()
        size_a, size_p = i64(size)
        nb_a, nb_p = i64(neighbors)
        for w in weights:
            _check_tensor(w, 'weight')
            if w.dtype != torch.float64 or \
                    tuple(w.shape) != tuple(int(x) for x in size_a):
                raise TypeError('weights must be float64 grids of the '
                                'operator size')
        cs = [f64(c) for c in coefs]
        os_ = [i64(o) for o in offsets]
        for (ca, _), (oa, _) in zip(cs, os_):
            if len(ca) != len(oa):
                raise TypeError('coefs and offsets differ in length')
        W = (C.c_void_p * nweights)(*[w.data_ptr() for w in weights])
        CP = (C.c_void_p * nweights)(*[C.cast(p, C.c_void_p) for _, p in cs])
        OP = (C.c_void_p * nweights)(*[C.cast(p, C.c_void_p) for _, p in os_])
        NC = (C.c_int * nweights)(*[len(a) for a, _ in cs])
        h = C.c_void_p()
        check(lib.gb_woperator_new(nweights, W, CP, OP, NC, size_p,
                                   int(range), nb_p, int(bool(real)),
                                   int(bool(cfd)), C.byref(h)))
        self._h = h
        self._lib = lib
        self._keep = (weights, cs, os_)
        self.size = tuple(int(x) for x in size_a)
        self.real = bool(real)

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value:
            self._lib.gb_woperator_free(h)
            self._h = None

    def apply(self, input, output, phases=None):
        """WOperator_apply (c/woperators.cpp:318-370)."""
        _check_tensor(input, 'input')
        _check_tensor(output, 'output')
        if input.shape != output.shape or input.dtype != output.dtype:
            raise TypeError('input and output differ in shape or dtype')
        if tuple(input.shape[-3:]) != self.size:
            raise TypeError(f'grid shape {tuple(input.shape[-3:])} != '
                            f'{self.size}')
        ph, ph_p = phases_arg(phases)
        check(self._lib.gb_woperator_apply(
            self._h, C.c_void_p(input.data_ptr()),
            C.c_void_p(output.data_ptr()), _nin(input.shape),
            _dtype_code(input.dtype), ph_p, _stream()))

    def relax(self, relax_method, f, s, nrelax, w=1.0):
        """WOperator_relax (c/woperators.cpp:53-96)."""
        _check_tensor(f, 'f')
        _check_tensor(s, 's')
        if tuple(f.shape) != self.size or tuple(s.shape) != self.size:
            raise TypeError('relax: arrays must have the grid shape')
        if f.dtype != torch.float64 or s.dtype != torch.float64:
            raise TypeError('relax: float64 arrays only')
        check(self._lib.gb_woperator_relax(
            self._h, int(relax_method), C.c_void_p(f.data_ptr()),
            C.c_void_p(s.data_ptr()), int(nrelax),
            float(1.0 if w is None else w), _stream()))

    def get_diagonal_element(self):
        """c/woperators.cpp:372-398 (synchronises the stream)."""
        d = C.c_double(0.0)
        check(self._lib.gb_woperator_get_diagonal_element(
            self._h, C.byref(d), _stream()))
        return d.value

    def get_async_sizes(self):
        # c/woperators.cpp:400-410 without GPAW_ASYNC
        return (0, 1, 1)


class Transformer:
    """``Transformer(size_in, size_out, k, pads, npads, skip, neighbors,
    real, comm, interpolate, use_gpu=1)``."""

    def __init__(self, size_in, size_out, k, paddings, npaddings, skip,
                 neighbors, real, comm, interpolate, use_gpu=1):
        if comm is not None:
            raise NotImplementedError('domain decomposition (comm) is not '
                                      'supported: one grid per GPU')
        lib = _lib.load()
        a = [i64(x) for x in (size_in, size_out, paddings, npaddings, skip,
                              neighbors)]
        h = C.c_void_p()
        check(lib.gb_transformer_new(a[0][1], a[1][1], int(k), a[2][1],
                                     a[3][1], a[4][1], a[5][1],
                                     int(bool(real)), int(bool(interpolate)),
                                     C.byref(h)))
        self._h = h
        self._lib = lib
        self.size_in = tuple(int(x) for x in a[0][0])
        self.size_out = tuple(int(x) for x in a[1][0])
        self.interpolate = bool(interpolate)

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value:
            self._lib.gb_transformer_free(h)
            self._h = None

    def apply_gpu(self, in_ptr, out_ptr, shape, dtype, phases=None):
        """Transformer_apply_gpu (c/gpu/transformers.cpp:189-226)."""
        ph, ph_p = phases_arg(phases)
        check(self._lib.gb_transformer_apply(
            self._h, C.c_void_p(in_ptr), C.c_void_p(out_ptr), _nin(shape),
            _dtype_code(dtype), ph_p, _stream()))

    def apply(self, input, output, phases=None):
        _check_tensor(input, 'input')
        _check_tensor(output, 'output')
        if tuple(input.shape[-3:]) != self.size_in or \
                tuple(output.shape[-3:]) != self.size_out:
            raise TypeError('transformer: grid shapes do not match')
        if input.shape[:-3] != output.shape[:-3] or \
                input.dtype != output.dtype:
            raise TypeError('transformer: batch shape or dtype mismatch')
        self.apply_gpu(input.data_ptr(), output.data_ptr(),
                       tuple(input.shape), input.dtype, phases)

    def set_chunk(self, chunk):
        """Output planes of axis 0 per CTA (0 = the automatic rule)."""
        check(self._lib.gb_transformer_set_chunk(self._h, int(chunk)))

    def get_async_sizes(self):
        return (0, 1)


def fd_precond(rest0, rest1, intp1, intp2, kin0, kin1, kin2,
               d0, q0, r1, d1, q1, r2, d2, q2, residuals, nresiduals, step,
               phases=None):
    """c/fd_preconditioner.cpp:106-351 on the GPU; writes d0.

    ``nresiduals`` may be None (the negation is then done on load)."""
    if residuals.dim() not in (3, 4):
        raise TypeError('Bad array dimension.')
    for name, a in (('d0', d0), ('q0', q0), ('r1', r1), ('d1', d1),
                    ('q1', q1), ('r2', r2), ('d2', d2), ('q2', q2)):
        _check_tensor(a, name)
        if a.dim() != 4:
            raise TypeError('Work arrays do not have 4 dimensions.')
    _check_tensor(residuals, 'residuals')
    nin = _nin(residuals.shape)
    if d0.shape[0] != nin or d1.shape[0] != nin or d2.shape[0] != nin:
        raise TypeError('Number of input grids does not match with work '
                        'arrays.')
    if d0.shape != q0.shape:
        raise TypeError('Arrays d0 and q0 do not have the same shape.')
    if not (d1.shape == r1.shape == q1.shape):
        raise TypeError('Arrays d1, q1, r1 do not have the same shape.')
    if not (d2.shape == r2.shape == q2.shape):
        raise TypeError('Arrays d2, q2, r2 do not have the same shape.')
    if nresiduals is not None and nresiduals.shape != residuals.shape:
        raise TypeError('Arrays residuals and nresiduals do not have the '
                        'same shape.')
    lib = _lib.load()
    ph, ph_p = phases_arg(phases)
    ptr = [C.c_void_p(a.data_ptr()) for a in (d0, q0, r1, d1, q1, r2, d2,
                                             q2)]
    check(lib.gb_fd_precond(
        rest0._h, rest1._h, intp1._h, intp2._h, kin0._h, kin1._h, kin2._h,
        *ptr, C.c_void_p(residuals.data_ptr()),
        C.c_void_p(nresiduals.data_ptr() if nresiduals is not None
                   else None),
        nin, _dtype_code(residuals.dtype), float(step), ph_p, _stream()))
