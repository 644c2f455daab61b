"""StepPipeline: a host-resident batch streamed through the GPU in chunks
gives the same results as the operators on the whole batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('chunk', [3, 8, 64])
def test_pipeline_equals_whole_batch(chunk, cuda):
    import torch
    from gpaw_b200 import GridDescriptor, Laplace, Transformer
    from gpaw_b200.pipeline import StepPipeline
    gd = GridDescriptor((24, 20, 28), (5.0, 4.0, 6.0), 1)
    gd2 = gd.coarsen()
    ph = gd.phase_factor_cd((0.25, 0.0, 0.1))
    kin = Laplace(gd, -0.5, 3, complex)
    rst = Transformer(gd, gd2, 3, complex)
    itp = Transformer(gd2, gd, 3, complex)
    nb = 11
    rng = np.random.default_rng(3)
    a = rng.standard_normal((nb,) + tuple(gd.n_c)) + \
        1j * rng.standard_normal((nb,) + tuple(gd.n_c))
    hin = torch.from_numpy(a).pin_memory()
    hy = torch.empty_like(hin).pin_memory()
    hz = torch.empty_like(hin).pin_memory()
    hc = torch.empty((nb,) + tuple(gd2.n_c), dtype=hin.dtype).pin_memory()
    StepPipeline(kin, rst, itp, chunk=chunk).run(hin, hy, hc, hz, ph)
    x = hin.cuda()
    y = torch.empty_like(x)
    kin.apply(x, y, ph)
    c = rst.apply(x, phases=ph)
    z = itp.apply(c, phases=ph)
    assert np.array_equal(hy.numpy(), y.cpu().numpy())
    assert np.array_equal(hc.numpy(), c.cpu().numpy())
    assert np.array_equal(hz.numpy(), z.cpu().numpy())
