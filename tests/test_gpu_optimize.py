"""GPU parity: the optimizer (src/optimize.cpp, src/inversion.cpp:302-490) for
the vs-only parametrisation against the oracle restatement.

Bars (written here): model update bit-identical; inner products, max-abs
normalisation and the descent angle within 1e-13 relative (fixed-order tree
sums vs sequential sums); the L-BFGS direction within 1e-11 relative (the log
of the model differs from the C library's by at most an ulp); a 3-iteration
L-BFGS inversion of the checkerboard case (41x41x30, FP64 sweeps, PDE
smoothing) follows the oracle-driven inversion: same accepted step lengths and
line-search sub-iterations, misfits within 1e-6 relative, final model within
1e-6 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda:0")


def test_model_update_bit_exact(gpu, orc):
    from surfattpp_b200 import optimize
    rng = np.random.default_rng(1)
    vs = rng.uniform(2.5, 4.8, 200_001)
    d = rng.normal(size=vs.size)
    a, b, c = optimize.model_update_vs(_t(vs), _t(d), 0.02)
    ra, rb, rc = orc.model_update_vs(vs, d, 0.02)
    for x, y in ((a, ra), (b, rb), (c, rc)):
        assert np.array_equal(x.cpu().numpy(), y)


def test_reductions(gpu, orc):
    from surfattpp_b200 import optimize
    rng = np.random.default_rng(2)
    x = rng.normal(size=1_000_003)
    y = rng.normal(size=x.size)
    got = optimize.dot(_t(x), _t(y))
    assert abs(got - float(np.dot(x, y))) <= 1e-13 * np.abs(x * y).sum()
    g = _t(x)
    m = optimize.grad_normalization(g)
    rg, rm = orc.grad_normalization(x)
    assert m == rm and np.array_equal(g.cpu().numpy(), rg)
    ang = optimize.calc_descent_angle(_t(y), _t(x))
    assert abs(ang - orc.descent_angle(y, x)) <= 1e-10
    z = _t(np.zeros(10))
    assert optimize.grad_normalization(z) == 0.0
    assert optimize.calc_descent_angle(z, _t(np.ones(10))) == 90.0


@pytest.mark.parametrize("nhist", [0, 1, 3, 5, 7])
def test_lbfgs_direction(gpu, orc, nhist):
    from surfattpp_b200 import optimize
    rng = np.random.default_rng(10 + nhist)
    n = 150_001
    models = [np.exp(rng.normal(1.2, 0.05, n))]
    grads = [rng.normal(size=n)]
    for _ in range(nhist):
        models.append(models[-1] * (1 - 0.02 * rng.normal(size=n) * 0.3))
        grads.append(grads[-1] * 0.8 + 0.1 * rng.normal(size=n))
    lb = optimize.LBFGS(n)
    for k, (m, g) in enumerate(zip(models, grads)):
        lb.store(k, _t(m), _t(g))
    d = lb.direction(nhist).cpu().numpy()
    keep = min(nhist, optimize.MAX_LBFGS_STORE)
    ref = orc.lbfgs_direction(models[nhist - keep:], grads[nhist - keep:])
    assert np.abs(d - ref).max() <= 1e-11 * np.abs(ref).max()


def _oracle_inversion(orc, w, ev, vs0, smooth, niter, step=0.02, max_sub=10):
    """Inversion::run_inversion with L-BFGS (src/inversion.cpp:106-160,
    :396-463) driven by the oracle chain."""
    m11, m12, m22 = w.media()

    def fa(vs):
        sv, st = orc.fwdsurf(w.zgrid, vs, w.periods, nthreads=8)
        assert st.sum() == 0
        o = orc.forward_for_events(w.xx_deg, w.yy_deg, sv, m11, m12, m22, ev, calc_adj=True,
                                   nthreads=8)
        sv_, sp_, sr_, st = orc.depthkernel_hti(w.zgrid, vs, w.periods, nthreads=8)
        vp = np.vectorize(orc.vs2vp)(vs)
        ker = orc.combine_kernels_vs(o["adj_s"], vs, vp, sv_, sp_, sr_)
        sm, _ = orc.pde_smooth(ker, smooth["dx"], smooth["dy"], smooth["dz"], smooth["ygrid"],
                               smooth["zgrid"], smooth["sigma_h"], smooth["sigma_v"])
        return o["chi"], ker, sm / o["chi"]

    vs = vs0.copy()
    models, grads, misfit, alphas, subs = [], [], [], [], []
    iter_start = 0
    for it in range(niter):
        model = vs.copy()
        f0, ker, grad = fa(vs)
        misfit.append(f0)
        models.append(model.ravel())
        grads.append(grad.ravel())
        while True:
            if it == iter_start:
                d = grad.ravel().copy()
            else:
                keep = min(it, 5)
                d = orc.lbfgs_direction(models[it - keep:], grads[it - keep:])
            d, _ = orc.grad_normalization(d)
            if it > iter_start and orc.descent_angle(d, grad.ravel()) > 92.0:
                iter_start = it
                continue
            gd = float(np.dot(ker.ravel(), d))
            alpha, aL, aR = step, 0.0, 0.0
            restart = False
            for sub in range(max_sub):
                trial = orc.model_update_vs(model, d, alpha)[0].reshape(model.shape)
                f1, ker, grad = fa(trial)
                kd = float(np.dot(ker.ravel(), d))
                st, nxt, aL, aR = orc.wolfe_condition(gd, kd, alpha, aL, aR, f0, f1, sub, 0.1,
                                                      0.9, max_sub, step)
                if st == 0:
                    break
                if st == 1:
                    alpha = nxt
                    continue
                restart = True
                break
            if restart:
                iter_start = it
                continue
            vs = trial
            alphas.append(alpha)
            subs.append(sub + 1)
            break
    return vs, misfit, alphas, subs


@pytest.mark.slow
@pytest.mark.parametrize("autograd", [False, True, "fused"])
def test_lbfgs_inversion_follows_oracle(gpu, orc, autograd):
    import torch
    from surfattpp_b200 import inversion, preproc
    from surfattpp_b200 import workloads as W
    w = W.config1()
    ev = w.events()
    m11, m12, m22 = w.media()
    sv_true, _ = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    ev["tt_obs"] = orc.forward_for_events(w.xx_deg, w.yy_deg, sv_true, m11, m12, m22, ev,
                                          calc_adj=False, nthreads=8)["syn"].copy()
    vs0 = w.meta["vs_start"]
    smooth = dict(ygrid=w.yy_deg, zgrid=w.zgrid, dx=0.05, dy=0.05, dz=2.0, sigma_h=0.1,
                  sigma_v=2.0)
    niter = 3
    rvs, rmis, ral, rsub = _oracle_inversion(orc, w, ev, vs0, smooth, niter)
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp64")
    g = inversion.MisfitGradient(plan, w.zgrid, w.periods)
    # autograd True: the kernel as the backward of chi built in torch on
    # TravelTimes; "fused": the backward of TravelTimeMisfit (same evaluation)
    inv = inversion.Inversion(g, _t(ev["tt_obs"]), _t(ev["weight"]), smooth=smooth, niter=niter,
                              autograd=autograd)
    vs = inv.run(_t(vs0))
    torch.cuda.synchronize()
    assert inv.alphas == ral and inv.sub_iters == rsub
    assert np.allclose(inv.misfit, rmis, rtol=1e-6, atol=0)
    assert rmis[-1] < rmis[0]
    got = vs.cpu().numpy()
    assert np.abs(got - rvs).max() <= 1e-6 * np.abs(rvs).max()
