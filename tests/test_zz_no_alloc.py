"""sa_eik_fwd_field_noalloc: the allocation-free forward solve, for callers
that cannot allocate device memory when they call in (inside another
framework's allocator or memory pool, hosts that forbid cudaMalloc after
start-up).  It keeps every intermediate in a fixed device array, so here it is
checked against the ordinary entry point (sa_eik_fwd_field) and against the
CPU oracle on two calls in a row, which also shows that the second call is not
disturbed by the first call's leftovers; then without the optional outputs on
a non-default stream, and at the documented size limit (680 x 680 accepted,
681 x 681 rejected).  Bar: 1e-12 relative and the same iteration count, as
the other FP64 parity tests.  Collected last on purpose (file name) so that a
stop at the first failure has already run every other test."""
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


def _noalloc(case, stream=None, with_outputs=True):
    """One call through the C ABI with device arrays; returns (T, niter, status)."""
    import torch
    from surfattpp_b200 import _capi
    xx, yy, spha, sphb, sphc, fun, x0, y0 = case
    ny, nx = fun.shape
    dev = torch.device("cuda:0")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    dxx, dyy, da, db, dc, df = (t(a) for a in (xx, yy, spha, sphb, sphc, fun))
    out = torch.full((ny, nx), float("nan"), dtype=torch.float64, device=dev)
    niter = torch.zeros(1, dtype=torch.int32, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    rc = _capi.lib().sa_eik_fwd_field_noalloc(
        nx, ny, dxx.data_ptr(), dyy.data_ptr(), da.data_ptr(), db.data_ptr(), dc.data_ptr(),
        df.data_ptr(), x0, y0, out.data_ptr(), niter.data_ptr() if with_outputs else None,
        status.data_ptr() if with_outputs else None,
        stream.cuda_stream if stream is not None else None)
    assert rc == _capi.SA_OK
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    return out.cpu().numpy(), int(niter.item()), int(status.item())


def _rel(got, want):
    m = want > 0
    assert np.all(got[~m] == want[~m])
    return np.max(np.abs(got[m] - want[m]) / want[m])


def test_noalloc_matches_entry_point_and_oracle(gpu, orc):
    from surfattpp_b200 import eikonal
    for case in (_case(71, 53, 0.7, -1.3, 1), _case(64, 80, -3.2, 2.9, 2)):
        want, it_want = eikonal.FSM_UW_PS_lonlat_2d(*case, precision="fp64", return_iters=True)
        ref, it_ref = orc.eik_fwd(*case)
        got, niter, status = _noalloc(case)
        assert status == 0
        assert niter == it_want == it_ref
        assert _rel(got, want) <= 1e-12
        assert _rel(got, ref) <= 1e-12


def test_noalloc_without_outputs_on_a_stream(gpu, orc):
    import torch
    case = _case(57, 61, 1.9, 0.4, 3)
    ref, _ = orc.eik_fwd(*case)
    s = torch.cuda.Stream()
    got, _, _ = _noalloc(case, stream=s, with_outputs=False)
    assert _rel(got, ref) <= 1e-12


def test_noalloc_size_limit(gpu):
    """680 x 680 = 462,400 cells, the largest square grid the array holds.
    Its great-circle geometry is formed on the device (CUDA's acos, within 2
    ulp) where the allocating entry point uses the host C library; on this
    many cells the travel times then differ by up to about 2e-12 relative
    (the two smaller grids above stay within 1e-12), hence 1e-11 here."""
    import torch
    from surfattpp_b200 import _capi, eikonal
    case = _case(680, 680, -1.1, 0.8, 4)
    got, niter, status = _noalloc(case)
    want, it_want = eikonal.FSM_UW_PS_lonlat_2d(*case, precision="fp64", return_iters=True)
    assert status == 0 and niter == it_want
    assert _rel(got, want) <= 1e-11
    lib = _capi.lib()
    p = torch.zeros(1, dtype=torch.float64, device="cuda:0").data_ptr()
    for nx, ny in ((681, 681), (800, 800)):
        rc = lib.sa_eik_fwd_field_noalloc(nx, ny, p, p, p, p, p, p, 0.0, 0.0, p, None, None, None)
        assert rc == _capi.SA_ERR_ARG
