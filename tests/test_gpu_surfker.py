"""GPU parity: surfdisp96 / sregn96_hti / sregnpu columns and the kernel
combination against the CPU oracle.

The device routines use correctly rounded exp / log / sin / cos
(crmath.cuh).  Two oracle builds check them:
  * math="cr": the restatement with the same correctly rounded functions.
    Phase velocities, depth kernels and group kernels must be bit-identical:
    this checks the transliteration operation for operation.
  * the default build with the C library's functions (what the reference
    calls).  Phase velocities must still be bit-identical (the C library
    misrounds about 0.1 % of arguments, which moves no REAL*4-rounded root on
    C1 or the C3 rows tested).  The depth kernels then differ by the
    propagation of those misroundings through the eigenfunction recursions:
    the oracle itself, evaluated with correctly rounded functions, differs
    from its C-library build by up to 9.3e-12 (depth kernels) and 8.5e-11
    (group kernels) of the column's largest kernel on C1, which sets the
    bars 2e-11 and 2e-10.
Kernel combination: bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(orc):
    from surfattpp_b200 import workloads as W
    return W.config1()


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda:0")


def test_fwdsurf_matches_oracle(orc, gpu, c1):
    from surfattpp_b200 import surfker
    w = c1
    ref, st = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    ref_cr, _ = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8, math="cr")
    svel, status = surfker.fwdsurf(w.zgrid, _dev(w.vs3d), w.periods)
    got = svel.cpu().numpy()
    assert int(status.max()) == 0 and st.sum() == 0
    assert np.array_equal(got, ref_cr)
    assert np.array_equal(got, ref)


def test_fwdsurf_c3_rows_match_oracle(orc, gpu):
    """20 rows of the 301 x 301 x 40 random-field model (6020 columns x 20
    periods): every phase velocity bit-identical to the C-library oracle."""
    from surfattpp_b200 import surfker
    from surfattpp_b200 import workloads as W
    w = W.config3()
    vs = np.ascontiguousarray(w.vs3d[100:120])
    ref, st = orc.fwdsurf(w.zgrid, vs, w.periods, nthreads=8)
    got, status = surfker.fwdsurf(w.zgrid, _dev(vs), w.periods)
    assert st.sum() == 0 and int(status.max()) == 0
    assert np.array_equal(got.cpu().numpy(), ref)


def test_fwdsurf_multi_wave_grid_matches_oracle(orc, gpu):
    """A grid of more columns than one wave of the 10-block launch holds
    (24 copies of 20 C3 rows: 144,480 columns), which takes the 16-block
    form of the dispersion kernel: every copy bit-identical to the oracle's
    phase velocities of the 20 rows."""
    from surfattpp_b200 import surfker
    from surfattpp_b200 import workloads as W
    w = W.config3()
    vs = np.ascontiguousarray(w.vs3d[100:120])
    ref, st = orc.fwdsurf(w.zgrid, vs, w.periods, nthreads=8)
    big = np.ascontiguousarray(np.tile(vs, (24, 1, 1)))
    got, status = surfker.fwdsurf(w.zgrid, _dev(big), w.periods)
    assert st.sum() == 0 and int(status.max()) == 0
    got = got.cpu().numpy()
    for t in range(24):
        assert np.array_equal(got[:, :, 20 * t:20 * (t + 1)], ref)


@pytest.mark.parametrize("igr,iwave", [(1, 2), (0, 1), (1, 1)])
def test_fwdsurf_group_and_love(orc, gpu, c1, igr, iwave):
    from surfattpp_b200 import surfker
    w = c1
    vs = w.vs3d[::4, ::4].copy()
    ref, _ = orc.fwdsurf(w.zgrid, vs, w.periods, iwave=iwave, igr=igr, nthreads=8)
    ref_cr, _ = orc.fwdsurf(w.zgrid, vs, w.periods, iwave=iwave, igr=igr, nthreads=8, math="cr")
    got, _ = surfker.fwdsurf(w.zgrid, _dev(vs), w.periods, iwave=iwave, igr=igr)
    got = got.cpu().numpy()
    assert np.array_equal(got, ref_cr)
    assert np.array_equal(got, ref)


def _column_err(g, r):
    scale = np.abs(r).max(axis=2, keepdims=True)   # per column and period
    return np.abs(g - r) / np.where(scale > 0, scale, 1.0)


def test_depthkernel_matches_oracle(orc, gpu, c1):
    from surfattpp_b200 import surfker
    w = c1
    vs = w.vs3d[::3, ::3].copy()
    ref = orc.depthkernel_hti(w.zgrid, vs, w.periods, nthreads=8)
    ref_cr = orc.depthkernel_hti(w.zgrid, vs, w.periods, nthreads=8, math="cr")
    cp, _ = surfker.fwdsurf(w.zgrid, _dev(vs), w.periods)
    got = surfker.depthkernel_hti(w.zgrid, _dev(vs), w.periods, cp)
    for g, r, rc in zip(got, ref[:3], ref_cr[:3]):
        g = g.cpu().numpy()
        assert np.array_equal(g, rc)
        assert np.max(_column_err(g, r)) <= 2e-11


def test_combine_kernels_matches_oracle(orc, gpu, c1):
    from surfattpp_b200 import surfker
    rng = np.random.default_rng(5)
    nx, ny, nz, nper = 9, 7, 12, 5
    adj = rng.standard_normal((nper, ny, nx))
    vs = 3.0 + rng.random((nx, ny, nz))
    vp = np.vectorize(orc.vs2vp)(vs)
    sv, sp, sr = (rng.standard_normal((nx, ny, nz, nper)) for _ in range(3))
    ref = orc.combine_kernels_vs(adj, vs, vp, sv, sp, sr)
    got = surfker.combine_kernels_vs(_dev(adj), _dev(vs), _dev(vp), _dev(sv), _dev(sp), _dev(sr))
    assert np.array_equal(got.cpu().numpy(), ref)


def test_group_depthkernel_matches_oracle(orc, gpu, c1):
    """Rayleigh group-velocity kernels (depthkernel_rayleigh_group / sregnpu):
    phase kernels at t(1 +- 0.005) differenced in period."""
    from surfattpp_b200 import surfker
    w = c1
    vs = w.vs3d[::4, ::4].copy()
    ref = orc.depthkernel_group(w.zgrid, vs, w.periods, nthreads=8)
    ref_cr = orc.depthkernel_group(w.zgrid, vs, w.periods, nthreads=8, math="cr")
    assert ref[3].sum() == 0
    got = surfker.depthkernel_group(w.zgrid, _dev(vs), w.periods)
    for g, r, rc in zip(got, ref[:3], ref_cr[:3]):
        g = g.cpu().numpy()
        assert np.array_equal(g, rc)
        assert np.max(_column_err(g, r)) <= 2e-10


@pytest.mark.parametrize("igr", [0, 1])
def test_love_depthkernel_matches_oracle(orc, gpu, c1, igr):
    """Love-wave kernels (depthkernel_love_phase / _group through slegn96 /
    slegnpu): bit-identical to the correctly-rounded-math oracle, within
    1e-12 of each column's largest kernel of the C-library oracle (whose
    own floor here is 2e-13)."""
    from surfattpp_b200 import surfker
    w = c1
    vs = w.vs3d[::4, ::4].copy()
    ref = orc.depthkernel_love(w.zgrid, vs, w.periods, igr=igr, nthreads=8)
    ref_cr = orc.depthkernel_love(w.zgrid, vs, w.periods, igr=igr, nthreads=8, math="cr")
    assert ref[2].sum() == 0
    got = surfker.depthkernel_love(w.zgrid, _dev(vs), w.periods, igr=igr)
    for g, r, rc in zip(got, ref[:2], ref_cr[:2]):
        g = g.cpu().numpy()
        assert np.array_equal(g, rc)
        assert np.max(_column_err(g, r)) <= 1e-12
