"""Grid transformers: restriction and interpolation between grids whose
point counts differ by 2 (drop-in for gpaw/transformers.py)."""
from __future__ import annotations

import numpy as np

from . import cgpaw


def transformer_geometry(gdin, gdout, nn):
    """Halo pads, neighbour pads and skip flags (gpaw/transformers.py:27-55).

    Restriction when gdin has twice gdout's points, interpolation when it
    has half.  Returns (pad_cd, neighborpad_cd, skip_cd, interpolate)."""
    pad_cd = np.empty((3, 2), int)
    neighborpad_cd = np.empty((3, 2), int)
    skip_cd = np.zeros((3, 2), int)
    if (gdin.N_c == 2 * gdout.N_c).all():
        pad_cd[:, 0] = 2 * nn - 1 - 2 * gdout.beg_c + gdin.beg_c
        pad_cd[:, 1] = 2 * nn - 2 + 2 * gdout.end_c - gdin.end_c
        neighborpad_cd[:, 0] = 2 * nn - 2 + 2 * gdout.beg_c - gdin.beg_c
        neighborpad_cd[:, 1] = 2 * nn - 1 - 2 * gdout.end_c + gdin.end_c
        interpolate = False
    else:
        assert (gdout.N_c == 2 * gdin.N_c).all()
        pad_cd[:, 0] = nn - 1 - gdout.beg_c // 2 + gdin.beg_c
        pad_cd[:, 1] = nn + gdout.end_c // 2 - gdin.end_c
        neighborpad_cd[:, 0] = nn + gdout.beg_c // 2 - gdin.beg_c
        neighborpad_cd[:, 1] = nn - 1 - gdout.end_c // 2 + gdin.end_c
        skip_cd[:, 0] = gdout.beg_c % 2
        skip_cd[:, 1] = gdout.end_c % 2
        interpolate = True
        inpoints = (gdin.n_c[0] + 2 * nn - 1) * (gdin.n_c[1] + 2 * nn - 1)
        outpoints = gdout.n_c[0] * gdout.n_c[1]
        if inpoints > outpoints:
            points = ' x '.join([str(N) for N in gdin.N_c])
            raise ValueError('Cannot construct interpolator.  Grid %s '
                             'may be too small' % points)
    assert (pad_cd.ravel() >= 0).all()
    return pad_cd, neighborpad_cd, skip_cd, interpolate


class _Transformer:
    def __init__(self, gdin, gdout, nn=1, dtype=float, xp=None):
        self.gdin = gdin
        self.gdout = gdout
        self.nn = nn
        assert 1 <= nn <= 4
        assert dtype in [float, complex]
        self.dtype = dtype
        self.xp = xp
        pad, npad, skip, self.interpolate = transformer_geometry(gdin, gdout,
                                                                 nn)
        self.pad_cd = pad
        self.neighborpad_cd = npad
        self.skip_cd = skip
        self.ngpin = tuple(int(x) for x in gdin.n_c)
        self.ngpout = tuple(int(x) for x in gdout.n_c)
        self.transformer = cgpaw.Transformer(gdin.n_c, gdout.n_c, 2 * nn,
                                             pad, npad, skip,
                                             gdin.neighbor_cd,
                                             dtype == float, None,
                                             self.interpolate)

    def apply(self, input, output=None, phases=None):
        """gpaw/transformers.py:79-91: returns ``output``."""
        if output is None:
            output = self.gdout.empty(tuple(input.shape[:-3]),
                                      dtype=self.dtype)
        self.transformer.apply(input, output, phases)
        return output

    def set_chunk(self, chunk):
        """Output planes of axis 0 per CTA; 0 = automatic.  See
        gpaw_b200.autotune."""
        self.transformer.set_chunk(chunk)

    def get_async_sizes(self):
        return self.transformer.get_async_sizes()


def Transformer(gdin, gdout, nn=1, dtype=float, xp=None):
    """Factory of gpaw/transformers.py:121-134 (nn = 9 copies the input)."""
    if nn != 9:
        return _Transformer(gdin, gdout, nn, dtype, xp)

    class T:
        nn = 1

        def apply(self, input, output, phases=None):
            output[:] = input
            return output

    return T()
