"""GPU parity: surfdisp96 / sregn96_hti columns and the kernel combination
against the CPU oracle.

Bars: phase velocities are REAL*4-rounded roots (cg = sngl(c)); the device's
transcendentals differ from the C library by an ulp, which moves the FP64
root by ~1e-15 and so flips the final float rounding only where the root sits
on a rounding boundary: >= 99.9 % of values bit-identical, all within one
float ulp (2^-23 relative).  Depth kernels at identical phase velocities:
<= 1e-11 relative to the column's largest kernel (typically 1e-15; the
propagator products amplify the ulp-level differences of the device's
exp/sin/cos/log).  Kernel combination: bit-identical."""
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
    svel, status = surfker.fwdsurf(w.zgrid, _dev(w.vs3d), w.periods)
    got = svel.cpu().numpy()
    assert int(status.max()) == 0 and st.sum() == 0
    same = got == ref
    assert same.mean() >= 0.999
    assert np.max(np.abs(got - ref) / ref) <= 2.0 ** -23


@pytest.mark.parametrize("igr,iwave", [(1, 2), (0, 1)])
def test_fwdsurf_group_and_love(orc, gpu, c1, igr, iwave):
    from surfattpp_b200 import surfker
    w = c1
    vs = w.vs3d[::4, ::4].copy()
    ref, _ = orc.fwdsurf(w.zgrid, vs, w.periods, iwave=iwave, igr=igr, nthreads=8)
    got, _ = surfker.fwdsurf(w.zgrid, _dev(vs), w.periods, iwave=iwave, igr=igr)
    got = got.cpu().numpy()
    assert (got == ref).mean() >= 0.99
    assert np.max(np.abs(got - ref) / ref) <= 4 * 2.0 ** -23


def test_depthkernel_matches_oracle(orc, gpu, c1):
    from surfattpp_b200 import surfker
    w = c1
    vs = w.vs3d[::3, ::3].copy()
    rv, rp, rr, st = orc.depthkernel_hti(w.zgrid, vs, w.periods, nthreads=8)
    cp, _ = surfker.fwdsurf(w.zgrid, _dev(vs), w.periods)
    gv, gp, gr = surfker.depthkernel_hti(w.zgrid, _dev(vs), w.periods, cp)
    ref_cp, _ = orc.fwdsurf(w.zgrid, vs, w.periods, nthreads=8)
    same_cp = (cp.cpu().numpy() == ref_cp)           # (nper, ny, nx)
    for g, r in ((gv, rv), (gp, rp), (gr, rr)):
        g = g.cpu().numpy()
        scale = np.abs(r).max(axis=2, keepdims=True)  # per column and period
        err = np.abs(g - r) / scale
        mask = np.transpose(same_cp, (2, 1, 0))[:, :, None, :]
        assert np.max(np.where(mask, err, 0.0)) <= 1e-11
        assert np.max(err) <= 1e-5


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
    """Rayleigh group-velocity kernels (depthkernel_rayleigh_group / sregnpu).
    The kernels difference phase kernels at t(1 +- 0.005), which amplifies a
    one-ulp flip of a phase velocity 200-fold: columns whose three phase
    velocities are bit-identical to the oracle's within 1e-10 of the column's
    largest kernel, all columns within 1e-3."""
    from surfattpp_b200 import surfker
    w = c1
    vs = w.vs3d[::4, ::4].copy()
    rv, rp, rr, st = orc.depthkernel_group(w.zgrid, vs, w.periods, nthreads=8)
    assert st.sum() == 0
    gv, gp, gr = surfker.depthkernel_group(w.zgrid, _dev(vs), w.periods)
    same = np.ones(vs.shape[:2][::-1] + (w.nper,), bool)   # (ny, nx, nper)
    for f in (1.0, 1.005, 0.995):
        per = w.periods * f if f == 1.0 else np.array([p * (1.0 + 0.5 * 0.01 * (1 if f > 1 else -1))
                                                        for p in w.periods])
        d, _ = surfker.fwdsurf(w.zgrid, _dev(vs), per)
        r, _ = orc.fwdsurf(w.zgrid, vs, per, nthreads=8)
        same &= np.transpose(d.cpu().numpy() == r, (1, 2, 0))
    mask = np.transpose(same, (1, 0, 2))[:, :, None, :]      # (nx, ny, 1, nper)
    assert mask.mean() > 0.5
    for g, r in ((gv, rv), (gp, rp), (gr, rr)):
        g = g.cpu().numpy()
        scale = np.abs(r).max(axis=2, keepdims=True)
        err = np.abs(g - r) / scale
        assert np.max(np.where(mask, err, 0.0)) <= 2e-9
        assert np.max(err) <= 1e-3
