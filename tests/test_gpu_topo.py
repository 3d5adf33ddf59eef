"""GPU parity: media from topography (SurfGrid::build_media_matrix_with_topo,
src/surf_grid.cpp:80-190; gaussian_smooth_geo_2 / gradient_2_geo,
include/utils.h:505-649), the kernel-depth correction (:307-354) and the
batched forward/adjoint over those general (anisotropic-metric) media.

Bars (written here): gridded topography bit-identical (interp2d, plain
arithmetic); media and dip angle within 1e-12 relative / 1e-9 degrees (the
Gaussian weights use CUDA's sin/atan/exp, ulp-level apart from the C
library's, over windows of up to ~10^4 points); depth correction within
1e-13 of max|kernel| (cos of the dip angle, ulp-level); forward + adjoint on
the topography media with the oracle's iteration counts, synthetic times
within 1e-12 relative and adj_s within the propagated bound of the batch
tests (FP64 path), and within 1e-4 s (FP32 path)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c4():
    from surfattpp_b200 import workloads as W
    return W.config4(level=61, nsta=41, nper=4, src_range=(3, 5), lam=8.0)


def test_grid_topography(c4, gpu, orc):
    from surfattpp_b200 import surfgrid
    lon, lat, z = c4.meta["topo_raw"]
    got = surfgrid.grid_topography(lon, lat, z, c4.xx_deg, c4.yy_deg).cpu().numpy()
    X, Y = np.meshgrid(c4.xx_deg, c4.yy_deg)
    ref = orc.interp2d(lon, lat, z, X.ravel(), Y.ravel()).reshape(got.shape)
    assert np.array_equal(got, ref)


def test_topo_media(c4, gpu, orc):
    import torch
    from surfattpp_b200 import surfgrid
    lon, lat, z = c4.meta["topo_raw"]
    zg = surfgrid.grid_topography(lon, lat, z, c4.xx_deg, c4.yy_deg)
    sig = np.array([0.02, 0.05, 0.11, 0.3])
    m11, m12, m22, ang = surfgrid.build_media_with_topo(c4.xx_deg, c4.yy_deg, zg, sig)
    torch.cuda.synchronize()
    r11, r12, r22, rang = orc.topo_media(c4.xx_deg, c4.yy_deg, zg.cpu().numpy(), sig)
    for g, r in ((m11, r11), (m22, r22)):
        assert np.abs(g.cpu().numpy() - r).max() <= 1e-12
    assert np.abs(m12.cpu().numpy() - r12).max() <= 1e-12 * np.abs(r12).max()
    assert np.abs(ang.cpu().numpy() - rang).max() <= 1e-9
    assert np.all(ang.cpu().numpy() >= 0.0)


def test_sigma_from_wavelength(gpu):
    from surfattpp_b200 import surfgrid
    s = surfgrid.sigma_deg([3.0, 4.0], [10.0, 40.0], 2.5)
    assert np.allclose(s, [3.0 * 10 * 2.5 / (2 * np.pi) / (6371.0 * np.pi / 180),
                           4.0 * 40 * 2.5 / (2 * np.pi) / (6371.0 * np.pi / 180)], rtol=1e-15)


def test_correct_depth_with_topo(gpu, orc):
    import torch
    from surfattpp_b200 import surfgrid
    rng = np.random.default_rng(8)
    nx, ny, nz, nper = 13, 11, 30, 4
    zg = 2.0 * np.arange(nz)
    ang = rng.uniform(0.0, 40.0, (nper, ny, nx))
    ang[0, 0, 0] = 90.0       # vertical dip: cos guarded to 1e-6
    kers = [rng.normal(size=(nx, ny, nz, nper)) for _ in range(3)]
    t = [torch.as_tensor(k, device="cuda:0") for k in kers]
    surfgrid.correct_depth_with_topo(zg, torch.as_tensor(ang, device="cuda:0"), *t)
    torch.cuda.synchronize()
    for g, k in zip(t, kers):
        ref = orc.correct_depth_with_topo(zg, ang, k)
        assert np.abs(g.cpu().numpy() - ref).max() <= 1e-13 * np.abs(k).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_on_topography_media(c4, gpu, orc, precision):
    from surfattpp_b200 import preproc
    from test_gpu_batch import adj_bound, assert_within
    lon, lat, z = c4.meta["topo_raw"]
    X, Y = np.meshgrid(c4.xx_deg, c4.yy_deg)
    zg = orc.interp2d(lon, lat, z, X.ravel(), Y.ravel()).reshape(X.shape)
    sig = np.full(c4.nper, 0.05)
    m11, m12, m22, _ = orc.topo_media(c4.xx_deg, c4.yy_deg, zg, sig)
    c4.m11, c4.m12, c4.m22 = m11, m12, m22
    svel, st = orc.fwdsurf(c4.zgrid, c4.vs3d, c4.periods, nthreads=8)
    assert st.sum() == 0
    ev = c4.events()
    ref = orc.forward_for_events(c4.xx_deg, c4.yy_deg, svel, m11, m12, m22, ev, calc_adj=True,
                                 nthreads=8)
    out = preproc.forward_for_event(c4.xx_deg, c4.yy_deg, svel, ev, calc_adj=True, m11=m11,
                                    m12=m12, m22=m22, precision=precision)
    if precision == "fp64":
        assert np.array_equal(out["fwd_iters"], ref["fwd_iters"])
        assert np.max(np.abs(out["syn"] - ref["syn"]) / np.abs(ref["syn"])) <= 1e-12
        bound = adj_bound(orc, c4, svel, ev, ref, out["syn"])
        assert_within(out["adj_s"], ref["adj_s"], 2.0 * bound + 1e-300)
    else:
        assert np.max(np.abs(out["syn"] - ref["syn"])) <= 1e-4
        l2 = np.linalg.norm(out["adj_s"] - ref["adj_s"]) / np.linalg.norm(ref["adj_s"])
        assert l2 <= 1e-4
