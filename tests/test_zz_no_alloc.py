"""sa_eik_fwd_field_noalloc: the allocation-free forward solve, for callers
that cannot allocate device memory when they call in.  It keeps every
intermediate in a fixed device array, so here it is checked against the
ordinary entry point (sa_eik_fwd_field) on two calls in a row, which also
shows that the second call is not disturbed by the first call's leftovers.
Collected last on purpose (file name) so that a stop at the first failure
has already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(nx, ny, x0, y0, seed):
    xx = np.linspace(-12.0, 9.0, nx)
    yy = np.linspace(-7.0, 8.0, ny)
    lon, lat = np.meshgrid(np.radians(xx), np.radians(yy))
    rng = np.random.default_rng(seed)
    spha = 1.0 + 0.08 * np.sin(2.0 * lon) * np.cos(lat) + 0.01 * rng.random(lon.shape)
    sphb = 1.0 + 0.06 * np.cos(1.5 * lon) * np.sin(lat)
    sphc = 0.02 * np.sin(lon + lat)
    fun = 1.0 / (3.3 + 0.25 * np.cos(3.0 * lat) * np.sin(2.0 * lon))
    return xx, yy, spha, sphb, sphc, fun, x0, y0


def test_noalloc_matches_allocating_entry_point(gpu):
    import torch
    from surfattpp_b200 import _capi, eikonal
    lib = _capi.lib()
    dev = torch.device("cuda:0")
    for xx, yy, spha, sphb, sphc, fun, x0, y0 in (_case(71, 53, 0.7, -1.3, 1),
                                                 _case(64, 80, -3.2, 2.9, 2)):
        ny, nx = fun.shape
        want, it_want = eikonal.FSM_UW_PS_lonlat_2d(xx, yy, spha, sphb, sphc, fun, x0, y0,
                                                   precision="fp64", return_iters=True)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        dxx, dyy, da, db, dc, df = (t(a) for a in (xx, yy, spha, sphb, sphc, fun))
        out = torch.full((ny, nx), float("nan"), dtype=torch.float64, device=dev)
        niter = torch.zeros(1, dtype=torch.int32, device=dev)
        status = torch.full((1,), -1, dtype=torch.int32, device=dev)
        rc = lib.sa_eik_fwd_field_noalloc(nx, ny, dxx.data_ptr(), dyy.data_ptr(), da.data_ptr(),
                                          db.data_ptr(), dc.data_ptr(), df.data_ptr(), x0, y0,
                                          out.data_ptr(), niter.data_ptr(), status.data_ptr(),
                                          None)
        assert rc == _capi.SA_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert int(status.item()) == 0
        assert int(niter.item()) == it_want
        m = want > 0
        assert np.max(np.abs(got[m] - want[m]) / want[m]) <= 1e-12
        assert np.all(got[~m] == want[~m])


def test_noalloc_rejects_oversized_grid(gpu):
    import torch
    from surfattpp_b200 import _capi
    lib = _capi.lib()
    nx = ny = 800          # 640,000 cells: more than the fixed array holds
    p = torch.zeros(1, dtype=torch.float64, device="cuda:0").data_ptr()
    rc = lib.sa_eik_fwd_field_noalloc(nx, ny, p, p, p, p, p, p, 0.0, 0.0, p, None, None, None)
    assert rc == _capi.SA_ERR_ARG
