"""Autotuner of the z-block depth: candidate lists and the cache on the
CPU; on the GPU, every depth gives bit-identical results and the tuner
picks one of its candidates."""
import numpy as np
import pytest

from gpaw_b200 import autotune


def test_candidates():
    assert autotune.candidates(96) == [0, 96, 48, 24, 12, 6]
    assert autotune.candidates(7) == [0, 7, 4]
    assert autotune.candidates(3) == [0]


def test_cache_roundtrip(tmp_path):
    autotune.clear()
    autotune._CACHE['apply|2x8x8x8|torch.float64|19'] = 4
    p = tmp_path / 'tune.json'
    autotune.save(str(p))
    autotune.clear()
    assert autotune.load(str(p)) == 1
    assert autotune._CACHE == {'apply|2x8x8x8|torch.float64|19': 4}
    assert autotune.load(str(tmp_path / 'missing.json')) == 0
    autotune.clear()


@pytest.mark.gpu
@pytest.mark.parametrize('nn', [1, 3, 6])
@pytest.mark.parametrize('dtype', [float, complex])
def test_depth_does_not_change_results(nn, dtype, cuda):
    from oracle import gpaw_layer as L
    from gpaw_b200 import GridDescriptor, Laplace, Transformer
    from tests.helpers import to_dev, to_np
    rng = np.random.default_rng(40 + nn)
    N, pbc, cell = (38, 22, 34), (1, 0, 1), (5.0, 3.0, 4.4)
    gd = GridDescriptor(N, cell, pbc)
    gref = L.GridDescriptor(N, cell, pbc)
    a = rng.standard_normal((2,) + tuple(gd.n_c))
    if dtype == complex:
        a = a + 1j * rng.standard_normal(a.shape)
    ph = gref.phase_factor_cd((0.25, 0.0, 0.1)) if dtype == complex else None
    want = np.zeros_like(a)
    L.Laplace(gref, -0.5, nn, dtype).apply(a, want, ph)
    op = Laplace(gd, -0.5, nn, dtype)
    x = to_dev(a)
    for depth in (1, 2, 3, 5, 7, 16, 0):
        op.set_chunk(depth)
        y = x.new_zeros(x.shape)
        op.apply(x, y, ph)
        assert np.array_equal(to_np(y), want), depth
    if nn > 3:
        return
    gd2 = gd.coarsen()
    g2ref = gref.coarsen()
    r_want = L.Transformer(gref, g2ref, nn, dtype).apply(a, phases=ph)
    c = rng.standard_normal((2,) + tuple(gd2.n_c))
    if dtype == complex:
        c = c + 1j * rng.standard_normal(c.shape)
    i_want = L.Transformer(g2ref, gref, nn, dtype).apply(c, phases=ph)
    rst = Transformer(gd, gd2, nn, dtype)
    itp = Transformer(gd2, gd, nn, dtype)
    for depth in (1, 2, 3, 4, 9, 0):
        rst.set_chunk(depth)
        itp.set_chunk(depth)
        assert np.array_equal(to_np(rst.apply(x, phases=ph)), r_want), depth
        assert np.array_equal(to_np(itp.apply(to_dev(c), phases=ph)),
                              i_want), depth


@pytest.mark.gpu
def test_tuner_picks_a_candidate(cuda):
    import torch
    from gpaw_b200 import GridDescriptor, Laplace, Transformer
    autotune.clear()
    gd = GridDescriptor((48, 40, 64), (6.0, 5.0, 8.0), 1)
    op = Laplace(gd, -0.5, 3, complex)
    x = torch.randn((4,) + tuple(gd.n_c), dtype=torch.complex128,
                    device='cuda')
    y = torch.empty_like(x)
    ph = gd.phase_factor_cd((0.25, 0.0, 0.1))
    best, times = autotune.tune_operator(op, x, y, ph, reps=2)
    assert best in autotune.candidates(48) and set(times) == \
        set(autotune.candidates(48))
    # second call: from the cache, no timing
    best2, times2 = autotune.tune_operator(op, x, y, ph)
    assert best2 == best and times2 is None
    gd2 = gd.coarsen()
    rst = Transformer(gd, gd2, 3, complex)
    c = torch.empty((4,) + tuple(gd2.n_c), dtype=torch.complex128,
                    device='cuda')
    b, t = autotune.tune_transformer(rst, x, c, ph, reps=2)
    assert b in autotune.candidates(24)
    autotune.clear()
