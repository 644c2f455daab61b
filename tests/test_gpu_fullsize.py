"""The benchmark configurations at their full sizes, checked against the
reference on samples: the C2 batch (256 complex128 wave functions on a 96^3
Bloch-periodic grid) through the apply, restrict and interpolate kernels
with a few bands compared bit for bit to the reference's C core, and the C3
grid (192^3) solved by the mixed-precision solver against the reference's
FP64 multigrid."""
import numpy as np
import pytest

from oracle import gpaw_layer as L
from tests.helpers import to_np

pytestmark = pytest.mark.gpu


def test_c2_full_batch_sampled_bands(cuda):
    import torch
    from gpaw_b200 import GridDescriptor, Laplace, Transformer
    N, cell, kpt = (96, 96, 96), (96 * 0.18 / 0.52917721,) * 3, \
        (0.25, 0.0, 0.1)
    gd, go = GridDescriptor(N, cell, 1), L.GridDescriptor(N, cell, 1)
    gd2, go2 = gd.coarsen(), go.coarsen()
    ph = go.phase_factor_cd(kpt)
    g = torch.Generator(device='cuda')
    g.manual_seed(11)
    x = torch.randn((256,) + N, dtype=torch.complex128, device='cuda',
                    generator=g)
    y = torch.empty_like(x)
    Laplace(gd, -0.5, 3, complex).apply(x, y, ph)
    c = Transformer(gd, gd2, 3, complex).apply(x, phases=ph)
    z = Transformer(gd2, gd, 3, complex).apply(c, phases=ph)
    kin = L.Laplace(go, -0.5, 3, complex)
    rst = L.Transformer(go, go2, 3, complex)
    itp = L.Transformer(go2, go, 3, complex)
    for band in (0, 137, 255):
        a = to_np(x[band:band + 1])
        want = np.zeros_like(a)
        kin.apply(a, want, ph)
        assert np.array_equal(to_np(y[band:band + 1]), want), band
        wc = rst.apply(a, phases=ph)
        assert np.array_equal(to_np(c[band:band + 1]), wc), band
        assert np.array_equal(to_np(z[band:band + 1]),
                              itp.apply(wc, phases=ph)), band


def test_c3_full_grid_mixed_against_reference(cuda):
    import torch
    from gpaw_b200 import GridDescriptor, MixedPoissonSolver
    from gpaw_b200.workloads import BOHR, c3_density, neutralize
    h = 0.18 / BOHR
    N = (192, 192, 192)
    gd, go = GridDescriptor(N, (192 * h,) * 3, 0), \
        L.GridDescriptor(N, (192 * h,) * 3, 0)
    rho = neutralize(c3_density(go, 64), go)
    ps = MixedPoissonSolver(tol=1e-11)
    ps.set_grid_descriptor(gd)
    phi = gd.zeros()
    ps.solve_neutral(phi, torch.from_numpy(rho).cuda())
    eps = (1e-12 * float(np.sqrt((rho * rho).sum())))**2 * go.dv
    po = L.FDPoissonSolver(nn=3, eps=eps, maxiter=200)
    po.set_grid_descriptor(go)
    want = go.zeros()
    po.solve_neutral(want, rho)
    err = np.abs(to_np(phi) - want).max() / np.abs(want).max()
    assert err < 1e-9, err
