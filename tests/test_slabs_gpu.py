"""Slab geometry on the GPU without a process group."""
import numpy as np
import pytest


@pytest.mark.gpu
def test_slab_transfers_on_gpu(cuda):
    """Each of three emulated ranks restricts or interpolates its own output
    planes from a replicated input (so the gather is local) with the
    library's transformer kernels on the slab geometry (no axis-0 padding,
    slabs that start on odd points, an extra plane dropped): the planes
    equal the whole-grid transformer's bit for bit."""
    from gpaw_b200 import GridDescriptor
    from gpaw_b200.domains import (DistributedTransformer, SlabDomain,
                                   gpu_local_transformer)
    from gpaw_b200.transformers import Transformer
    from tests.helpers import to_dev, to_np
    bad = []
    for pbc0 in (1, 0):
        gd = GridDescriptor((26, 12, 10), (5.2, 2.4, 2.0), (pbc0, 1, 0))
        gd2 = gd.coarsen()
        ph = gd.phase_factor_cd((0.3, -0.2, 0.0))
        for dtype in (float, complex):
            phases = ph if dtype == complex else None
            for nn in (1, 3):
                for interp in (False, True):
                    gi, go = (gd2, gd) if interp else (gd, gd2)
                    rng = np.random.default_rng(nn + 2 * pbc0)
                    a = rng.standard_normal((2,) + tuple(gi.n_c))
                    if dtype == complex:
                        a = a + 1j * rng.standard_normal(a.shape)
                    x = to_dev(a)
                    ref = go.zeros((2,), dtype)
                    Transformer(gi, go, nn, dtype).apply(x, ref, phases)
                    ref = to_np(ref)
                    for r in range(3):
                        di = SlabDomain(gi.n_c, pbc0, r, 3, True)
                        do = SlabDomain(go.n_c, pbc0, r, 3)
                        t = DistributedTransformer(gi, go, nn, dtype, di, do,
                                                   gpu_local_transformer())
                        out = x.new_zeros((2,) + do.local_shape())
                        t.apply(x, out, phases)
                        if not np.array_equal(to_np(out),
                                              ref[:, do.beg:do.end]):
                            bad.append((pbc0, dtype.__name__, nn, interp, r))
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize('pbc0', [1, 0])
def test_single_slab_vcycles_on_gpu(cuda, pbc0):
    """One rank: three V-cycles of the slab solver with the library's
    kernels leave phi equal to the native executor's V-cycles."""
    from gpaw_b200 import FDPoissonSolver, GridDescriptor
    from gpaw_b200.domains import (DistributedFDPoissonSolver,
                                   gpu_local_operator, gpu_local_transformer)
    from tests.helpers import to_dev, to_np
    gd = GridDescriptor((24, 16, 16), (6.0, 4.0, 4.4), (pbc0, 1, 0))
    rng = np.random.default_rng(17)
    rho = to_dev(rng.standard_normal(tuple(gd.n_c)))
    phi0 = rng.standard_normal(tuple(gd.n_c)) * 0.1
    ps = FDPoissonSolver(nn=3, relax='J')
    ps.set_grid_descriptor(gd)
    ps._init()
    ref = to_dev(phi0)
    ref_err = [ps.iterate2(ps.step, phi=ref, rho=rho) for _ in range(3)]
    dps = DistributedFDPoissonSolver(ps, 0, 1,
                                     gpu_local_operator(float, ref.device),
                                     gpu_local_transformer())
    phi = to_dev(phi0)
    err = [dps.iterate(phi, rho) for _ in range(3)]
    assert np.array_equal(to_np(phi), to_np(ref))
    for e, r in zip(err, ref_err):
        assert abs(e - r) <= 1e-12 * abs(r)
