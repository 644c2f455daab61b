"""Autotuner for the plane-marching kernels' z-block depth.

Every stencil and transfer kernel cuts axis 0 of the grid into chunks, one
chunk per CTA (tiles of 32 x 16 points in axes 1-2 for the stencils, 16 x 16
or 8 x 32 output points for the transfers).  Short chunks give more CTAs
(better load balance, shorter tail) but re-read 2nn halo planes per chunk;
long chunks stream more planes per CTA.  The best depth depends on the grid,
the batch size, the element type and the stencil order, so it is picked by
timing: each candidate depth runs on the caller's own arrays (CUDA events on
the current stream, after one untimed launch), the fastest is set on the
object, and the choice is remembered per (kind, grid, batch, dtype, order)
in a cache that can be saved as JSON and loaded by later runs.

Outputs do not depend on the depth (every point is computed the same way in
any chunk), so tuning never changes a result.
"""
from __future__ import annotations

import json
import math
import os

import torch

_CACHE: dict = {}


def candidates(n0: int) -> list:
    """0 (the automatic rule) and depths n0, n0/2, n0/4, ... down to 4."""
    out = [0]
    d = n0
    while d >= 4:
        if d not in out:
            out.append(d)
        d = math.ceil(d / 2) if d > 4 else 0
    return out


def _key(kind, shape, dtype, order):
    return f'{kind}|{"x".join(str(int(s)) for s in shape)}|{dtype}|{order}'


def _time(fn, reps):
    fn()                                   # untimed: loads, warms caches
    st = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _tune(obj, key, n0, fn, reps, cands):
    if key in _CACHE:
        obj.set_chunk(_CACHE[key])
        return _CACHE[key], None
    times = {}
    for c in (cands if cands is not None else candidates(n0)):
        obj.set_chunk(c)
        times[c] = _time(fn, reps)
    best = min(times, key=times.get)
    obj.set_chunk(best)
    _CACHE[key] = best
    return best, times


def tune_operator(op, in_xg, out_xg, phase_cd=None, reps=3, cands=None):
    """Pick the z-block depth of ``op`` (an FDOperator) for ``op.apply(
    in_xg, out_xg, phase_cd)`` on these arrays.  Returns (depth, {depth:
    ms}) -- the timings are None when the depth came from the cache."""
    key = _key('apply', tuple(in_xg.shape), in_xg.dtype, op.npoints)
    return _tune(op, key, int(op.gd.n_c[0]),
                 lambda: op.apply(in_xg, out_xg, phase_cd), reps, cands)


def tune_transformer(tr, input, output, phases=None, reps=3, cands=None):
    """Pick the depth of a Transformer for ``tr.apply(input, output,
    phases)`` on these arrays."""
    kind = 'interpolate' if tr.interpolate else 'restrict'
    key = _key(kind, tuple(input.shape), input.dtype, tr.nn)
    n0 = int(output.shape[-3])
    return _tune(tr, key, n0, lambda: tr.apply(input, output, phases),
                 reps, cands)


def save(path):
    """Write the cache as JSON."""
    with open(path, 'w') as f:
        json.dump(_CACHE, f, indent=1, sort_keys=True)


def load(path):
    """Merge a JSON cache written by save(); missing file is not an error."""
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        data = json.load(f)
    _CACHE.update({k: int(v) for k, v in data.items()})
    return len(data)


def clear():
    _CACHE.clear()
