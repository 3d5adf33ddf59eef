"""GPU parity: PostProc::pde_smooth (src/postproc.cpp:388-463) against the
oracle's restatement.

Bars (written here): bit-identical fields on grids the oracle finishes in
seconds (the device evaluates every product and sum in the reference's order
with FMA contraction off, and the row/depth factors come from the host C
library); at a C5-sized grid (601x601x50) the size-independent properties:
a constant field is unchanged exactly, the step count equals the reference
formula's, and the smoothed field's extrema lie within the input's (the
explicit scheme is a convex combination at these stable coefficients)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grid(nx, ny, nz, lat0=24.0, d=0.05, dz=2.0):
    y = lat0 + d * np.arange(ny)
    z = dz * np.arange(nz)
    return y, z


@pytest.mark.parametrize("shape,d,sig", [((3, 3, 3), 0.1, (0.15, 3.0)),
                                          ((21, 23, 12), 0.05, (0.1, 4.0)),
                                          ((41, 37, 30), 0.05, (0.2, 6.0)),
                                          ((17, 64, 9), 0.01, (0.03, 10.0))])
def test_pde_smooth_bit_exact(gpu, orc, shape, d, sig):
    import torch
    from surfattpp_b200 import postproc
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape)
    y, z = _grid(*shape, d=d)
    ref, ns_ref = orc.pde_smooth(f, d, d, 2.0, y, z, sig[0], sig[1])
    t = torch.as_tensor(f, device="cuda:0").contiguous()
    out, ns = postproc.pde_smooth(t, y, z, d, d, 2.0, sig[0], sig[1])
    torch.cuda.synchronize()
    assert ns == ns_ref
    got = out.cpu().numpy()
    assert np.array_equal(got, ref), np.abs(got - ref).max()


def test_pde_smooth_kernel_list(gpu, orc):
    import torch
    from surfattpp_b200 import postproc
    rng = np.random.default_rng(5)
    shape = (21, 23, 12)
    y, z = _grid(*shape)
    ks = [torch.as_tensor(rng.standard_normal(shape), device="cuda:0"), None,
          torch.as_tensor(rng.standard_normal(shape), device="cuda:0")]
    sm = postproc.kernel_smooth(ks, y, z, 0.05, 0.05, 2.0, 0.1, 4.0)
    torch.cuda.synchronize()
    assert sm[1] is None
    for k, s in zip((ks[0], ks[2]), (sm[0], sm[2])):
        ref, _ = orc.pde_smooth(k.cpu().numpy(), 0.05, 0.05, 2.0, y, z, 0.1, 4.0)
        assert np.array_equal(s.cpu().numpy(), ref)


def test_pde_smooth_c5_properties(gpu, orc):
    import torch
    from surfattpp_b200 import postproc
    nx, ny, nz = 601, 601, 50
    y, z = _grid(nx, ny, nz, d=0.005)
    sig = (0.02, 6.0)
    ns_ref, _, _ = orc.pde_smooth_nstep(ny, 0.005, 0.005, 2.0, y[0], y[-1], *sig)
    c = torch.full((nx, ny, nz), 3.25, dtype=torch.float64, device="cuda:0")
    work = torch.empty_like(c)
    out, ns = postproc.pde_smooth(c, y, z, 0.005, 0.005, 2.0, *sig, work=work)
    torch.cuda.synchronize()
    assert ns == ns_ref
    assert bool((out == 3.25).all())
    g = torch.Generator(device="cuda:0").manual_seed(3)
    f = torch.rand((nx, ny, nz), dtype=torch.float64, device="cuda:0", generator=g)
    lo, hi = float(f.min()), float(f.max())
    out, _ = postproc.pde_smooth(f, y, z, 0.005, 0.005, 2.0, *sig, work=work)
    torch.cuda.synchronize()
    assert lo <= float(out.min()) and float(out.max()) <= hi
    assert float(out.std()) < 0.5 * 0.2887


def test_pde_smooth_rejects_bad_sigma(gpu):
    import torch
    from surfattpp_b200 import _capi, postproc
    y, z = _grid(5, 5, 5)
    t = torch.zeros((5, 5, 5), dtype=torch.float64, device="cuda:0")
    with pytest.raises(_capi.SAError):
        postproc.pde_smooth(t, y, z, 0.05, 0.05, 2.0, 0.0, 4.0)


@pytest.mark.parametrize("n_inv,nset", [((5, 5, 4), 3), ((7, 4, 3), 2), ((12, 9, 8), 1)])
def test_multigrid_smoothing_matches_oracle(gpu, orc, n_inv, nset):
    """smooth_method 1 (PostProc::InvGrid::fwd2inv / inv2fwd,
    src/postproc.cpp:160-386): bit-identical to the oracle on the
    checkerboard grid (41 x 41 x 30) for three coarse-grid shapes."""
    import torch
    from surfattpp_b200 import postproc
    from surfattpp_b200 import workloads as W
    w = W.config1()
    rng = np.random.default_rng(31)
    field = rng.standard_normal(w.vs3d.shape)
    ref = orc.multigrid_smooth(field, w.xx_deg, w.yy_deg, w.zgrid, n_inv, nset)
    sm = postproc.MultigridSmoother(w.xx_deg, w.yy_deg, w.zgrid, n_inv, nset)
    got = sm.smooth(torch.as_tensor(field, device="cuda:0"))
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), ref)
    sm.close()
