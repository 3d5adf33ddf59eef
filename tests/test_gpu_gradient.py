"""GPU parity: one misfit-gradient evaluation (Inversion::run_forward_adjoint,
src/inversion.cpp:245-276: fwdsurf -> dispersion kernels -> forward_for_event
-> combine_kernels) against the oracle's chain on the checkerboard case
(41x41x30, 10 periods, 250 events; observed times from the checkerboard
model, evaluated at the 1-D starting model).

Bars (written here):
  * FP64 plan: misfit <= 1e-12 relative, ker_vs <= 1e-12 of max|ker_vs|.
    The phase velocities are bit-identical to the oracle's, so the travel
    times and misfit are too; adj_s is summed with FP64 atomics in completion
    order, and the depth kernels differ from the C-library oracle's by the
    propagation of the C library's own misroundings (about 1e-11 of a
    column's largest kernel, 2e-16 of max|ker_vs| after the combination).
  * FP32 plan: misfit <= 1e-4 relative, ker_vs <= 1e-3 of max|ker_vs|.
  * The chain equals its parts run one by one (sa_surfdisp_columns,
    sa_plan_forward_adjoint, sa_depthkernel_columns, sa_combine_kernels_vs)
    bit for bit, except adj_s (FP64 atomics in completion order: 1e-12).
  * The reference's ker_vs is not a derivative with respect to the vs nodes:
    central differences of chi (+-1e-3 km/s) agree with it in sign at every
    node where |ker_vs| > 5 % of its maximum and correlate with it (Pearson
    r >= 0.95), while their ratio varies by node (about 4.5 to 9.5 on this
    case, for the oracle as for the device).  The factor is the cell area
    (the adjoint source is divided by it, src/eikonal_solver.cpp:366-367:
    about 28 km^2 here) times the depth-kernel conventions (sregn96 returns
    b dc/db, a dc/da and a density kernel whose elastic terms carry the
    velocities once more, and combine_kernels chains them as plain
    derivatives: 0.18-0.37 here).  The "derivative" convention of
    test_gpu_autograd.py applies those Jacobians.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2(orc):
    from surfattpp_b200 import workloads as W
    w = W.config1()
    m11, m12, m22 = w.media()
    ev = w.events()
    sv_true, st = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    assert st.sum() == 0
    ev["tt_obs"] = orc.forward_for_events(w.xx_deg, w.yy_deg, sv_true, m11, m12, m22, ev,
                                          calc_adj=False, nthreads=8)["syn"].copy()
    vs0 = w.meta["vs_start"]
    sv0, st = orc.fwdsurf(w.zgrid, vs0, w.periods, nthreads=8)
    assert st.sum() == 0
    ref = orc.forward_for_events(w.xx_deg, w.yy_deg, sv0, m11, m12, m22, ev, calc_adj=True,
                                 nthreads=8)
    sen_vs, sen_vp, sen_rho, st = orc.depthkernel_hti(w.zgrid, vs0, w.periods, nthreads=8)
    assert st.sum() == 0
    vp0 = np.vectorize(orc.vs2vp)(vs0)
    ker = orc.combine_kernels_vs(ref["adj_s"], vs0, vp0, sen_vs, sen_vp, sen_rho)
    return w, ev, vs0, dict(chi=ref["chi"], ker=ker, svel=sv0, adj_s=ref["adj_s"])


def _grad(w, ev, precision):
    import torch
    from surfattpp_b200 import inversion, preproc
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision=precision)
    g = inversion.MisfitGradient(plan, w.zgrid, w.periods)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    return plan, g, t(ev["tt_obs"]), t(ev["weight"]), t


@pytest.mark.parametrize("precision,chi_tol,ker_tol", [("fp64", 1e-12, 1e-12),
                                                        ("fp32", 1e-4, 1e-3)])
def test_gradient_matches_oracle_chain(c2, gpu, precision, chi_tol, ker_tol):
    import torch
    w, ev, vs0, ref = c2
    plan, g, tt, wt, t = _grad(w, ev, precision)
    out = g.run(t(vs0), tt, wt)
    torch.cuda.synchronize()
    assert int(out["status"][0]) == 0
    chi = float(out["chi"][0])
    assert abs(chi - ref["chi"]) <= chi_tol * abs(ref["chi"]), (chi, ref["chi"])
    ker = out["ker_vs"].cpu().numpy()
    scale = np.abs(ref["ker"]).max()
    err = np.abs(ker - ref["ker"]).max() / scale
    assert err <= ker_tol, err


def test_gradient_chain_equals_parts(c2, gpu, orc):
    import torch
    from surfattpp_b200 import surfker
    w, ev, vs0, ref = c2
    plan, g, tt, wt, t = _grad(w, ev, "fp64")
    vs = t(vs0)
    out = g.run(vs, tt, wt)
    torch.cuda.synchronize()
    sen = g.sen()
    sv, st = surfker.fwdsurf(w.zgrid, vs, w.periods)
    assert torch.equal(sv, out["svel"])
    parts = plan.run(sv, tt, wt)
    kv, kp, kr = surfker.depthkernel_hti(w.zgrid, vs, w.periods, sv)
    torch.cuda.synchronize()
    for a, b in zip((kv, kp, kr), sen):
        assert torch.equal(a, b)
    # adj_s is accumulated with FP64 atomics in completion order: equal to
    # rounding, not bit for bit, between two runs
    scale = float(parts["adj_s"].abs().max())
    assert float((parts["adj_s"] - out["adj_s"]).abs().max()) <= 1e-12 * scale
    assert torch.equal(parts["chi"], out["chi"])
    K = surfker.combine_kernels_vs(out["adj_s"], vs, None, kv, kp, kr)
    torch.cuda.synchronize()
    assert torch.equal(K, out["ker_vs"])
    # an explicit vp3d equal to vs2vp(vs3d) gives the same kernel
    vp = torch.as_tensor(np.vectorize(orc.vs2vp)(vs0), device=vs.device)
    K2 = surfker.combine_kernels_vs(out["adj_s"], vs, vp, kv, kp, kr)
    torch.cuda.synchronize()
    assert torch.equal(K2, out["ker_vs"])
    # sa_grad_combine: the last run's depth kernels with a given adj_s (the
    # multi-rank path passes the rank sum); linear in adj_s
    K3 = g.combine(vs, out["adj_s"])
    K4 = g.combine(vs, 2.0 * out["adj_s"], vp)
    torch.cuda.synchronize()
    assert torch.equal(K3, out["ker_vs"])
    assert torch.equal(K4, 2.0 * out["ker_vs"])


def test_gradient_repeat_and_autograd(c2, gpu):
    import torch
    from surfattpp_b200 import inversion
    w, ev, vs0, ref = c2
    plan, g, tt, wt, t = _grad(w, ev, "fp32")
    vs = t(vs0).requires_grad_(True)
    chi = inversion.TravelTimeMisfit.apply(g, vs, tt, wt)
    chi.backward()
    out = g.run(t(vs0), tt, wt)
    torch.cuda.synchronize()
    assert float(chi.detach()) == float(out["chi"][0])
    # a second run re-accumulates adj_s with atomics: equal to rounding
    scale = float(out["ker_vs"].abs().max())
    assert float((vs.grad - out["ker_vs"]).abs().max()) <= 1e-10 * scale


def test_gradient_finite_differences(c2, gpu):
    import torch
    w, ev, vs0, ref = c2
    plan, g, tt, wt, t = _grad(w, ev, "fp64")
    out = g.run(t(vs0), tt, wt)
    torch.cuda.synchronize()
    ker = out["ker_vs"].cpu().numpy().copy()
    big = np.argwhere(np.abs(ker) > 0.05 * np.abs(ker).max())
    rng = np.random.default_rng(2002)
    nodes = big[rng.choice(len(big), size=min(20, len(big)), replace=False)]
    h = 1e-3
    fd, kk = [], []
    for i, j, k in nodes:
        chis = []
        for s in (1.0, -1.0):
            v = vs0.copy()
            v[i, j, k] += s * h
            o = g.run(t(v), tt, wt, out=out)
            torch.cuda.synchronize()
            chis.append(float(o["chi"][0]))
        fd.append((chis[0] - chis[1]) / (2 * h))
        kk.append(ker[i, j, k])
    fd, kk = np.array(fd), np.array(kk)
    assert np.all(np.sign(fd) == np.sign(kk)), np.c_[fd, kk]
    r = np.corrcoef(fd, kk)[0, 1]
    assert r >= 0.95, r


def test_joint_phase_and_group_gradient(c2, gpu, orc):
    """Rayleigh phase and group data together (src/inversion.cpp:250-296):
    misfit_total = sum w_t chi_t, ker_curr = sum w_t K_t, gradient = sum
    w_t K_t / chi_t over the two types.  Group data: group velocities from
    fwdsurf (igr = 1) and the sregnpu kernels.  FP64 against the oracle's
    chain: misfits 1e-12; kernels 1e-12 of max against the oracle evaluated
    with the device's correctly rounded exp/log/sin/cos, 1e-9 against the
    C-library oracle (group kernels carry the C library's misroundings at
    1e-10 of a column's largest value)."""
    import torch
    from surfattpp_b200 import inversion
    w, ev, vs0, ref = c2
    m11, m12, m22 = w.media()
    u_true, _ = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, igr=1, nthreads=8)
    ev_gr = dict(ev)
    ev_gr["tt_obs"] = orc.forward_for_events(w.xx_deg, w.yy_deg, u_true, m11, m12, m22, ev,
                                             calc_adj=False, nthreads=8)["syn"].copy()
    u0, _ = orc.fwdsurf(w.zgrid, vs0, w.periods, igr=1, nthreads=8)
    ref_gr = orc.forward_for_events(w.xx_deg, w.yy_deg, u0, m11, m12, m22, ev_gr, calc_adj=True,
                                    nthreads=8)
    vp0 = np.vectorize(orc.vs2vp)(vs0)
    wph, wgr = 0.7, 0.3
    kers = []
    for math in ("cr", "libc"):
        sp = orc.depthkernel_hti(w.zgrid, vs0, w.periods, nthreads=8, math=math)
        sg = orc.depthkernel_group(w.zgrid, vs0, w.periods, nthreads=8, math=math)
        kph = orc.combine_kernels_vs(ref["adj_s"], vs0, vp0, *sp[:3])
        kgr = orc.combine_kernels_vs(ref_gr["adj_s"], vs0, vp0, *sg[:3])
        kers.append((kph, kgr))
    plan, g_ph, tt, wt, t = _grad(w, ev, "fp64")
    g_gr = inversion.MisfitGradient(plan, w.zgrid, w.periods, data_type="gr")
    inv = inversion.Inversion(g_ph, tt, wt, smooth=None, data_weight=wph,
                              more_data=[(g_gr, t(ev_gr["tt_obs"]), wt, wgr)])
    total, ker_curr, grad = inv.run_forward_adjoint(t(vs0))
    torch.cuda.synchronize()
    want = wph * ref["chi"] + wgr * ref_gr["chi"]
    assert abs(total - want) <= 1e-12 * abs(want)
    kc, gr = ker_curr.cpu().numpy(), grad.cpu().numpy()
    for (kph, kgr), tol in zip(kers, (1e-12, 1e-9)):
        kref = wph * kph + wgr * kgr
        gref = wph * kph / ref["chi"] + wgr * kgr / ref_gr["chi"]
        assert np.abs(kc - kref).max() <= tol * np.abs(kref).max()
        assert np.abs(gr - gref).max() <= tol * np.abs(gref).max()


def test_kernel_density_preconditioning(c2, gpu, orc):
    """is_kden (src/preproc.cpp:128-137, :294-300; src/postproc.cpp:487-517):
    the kernel-density adjoint (source -w, accumulated unmasked), its
    combination into ker_den and the preconditioning, FP64, against the
    oracle: kden_s and ker_den 1e-11 of their maxima (FP64 atomics in
    completion order), the preconditioning of identical inputs bit for bit,
    and the preconditioned gradient of one inversion step 1e-9 of its
    maximum."""
    import torch
    from surfattpp_b200 import inversion, postproc
    w, ev, vs0, ref = c2
    m11, m12, m22 = w.media()
    sv0 = ref["svel"]
    rk = orc.forward_for_events(w.xx_deg, w.yy_deg, sv0, m11, m12, m22, ev, calc_adj=True,
                                nthreads=8, kden=True)
    assert np.array_equal(rk["adj_s"], ref["adj_s"])   # the kden pass leaves adj_s alone
    sen = orc.depthkernel_hti(w.zgrid, vs0, w.periods, nthreads=8)
    vp0 = np.vectorize(orc.vs2vp)(vs0)
    kden_ref = orc.combine_kernels_vs(rk["kden_s"], vs0, vp0, *sen[:3])
    plan, g, tt, wt, t = _grad(w, ev, "fp64")
    g.set_kden(True)
    out = g.run(t(vs0), tt, wt)
    torch.cuda.synchronize()
    kd = out["ker_den"].cpu().numpy()
    assert np.abs(kd - kden_ref).max() <= 1e-11 * np.abs(kden_ref).max()
    # the preconditioning itself, on identical inputs (with tiny and negative
    # densities): bit for bit
    rng = np.random.default_rng(8)
    dens = rng.standard_normal(5000) * np.where(rng.random(5000) < 0.1, 1e-14, 1.0)
    ker = rng.standard_normal(5000)
    got = postproc.kernel_precondition(t(dens), t(ker).clone())
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), orc.kernel_precondition(dens, ker))
    # one inversion step with is_kden (no smoothing)
    inv = inversion.Inversion(g, tt, wt, smooth=None, kden=True)
    total, ker_curr, grad = inv.run_forward_adjoint(t(vs0))
    torch.cuda.synchronize()
    gref = orc.kernel_precondition(kden_ref, ref["ker"]) / ref["chi"]
    assert np.abs(grad.cpu().numpy() - gref).max() <= 1e-9 * np.abs(gref).max()
    assert np.abs(ker_curr.cpu().numpy() - ref["ker"]).max() <= 1e-12 * np.abs(ref["ker"]).max()


def test_love_group_gradient(c2, gpu, orc):
    """Love group-velocity data (the reference's only Love path in an
    inversion: depthkernel1d for group data, src/surf_grid.cpp:282-286):
    group velocities from fwdsurf (iwave 1, igr 1), the slegnpu kernels, no
    vp kernel.  FP64 against the oracle's chain: misfit 1e-12, ker_vs 1e-12
    of max.  Love phase data are rejected, as the reference's
    depthkernelHTI1d does."""
    import torch
    from surfattpp_b200 import _capi, inversion
    w, ev, vs0, ref = c2
    m11, m12, m22 = w.media()
    u_true, _ = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, iwave=1, igr=1, nthreads=8)
    ev_l = dict(ev)
    ev_l["tt_obs"] = orc.forward_for_events(w.xx_deg, w.yy_deg, u_true, m11, m12, m22, ev,
                                            calc_adj=False, nthreads=8)["syn"].copy()
    u0, _ = orc.fwdsurf(w.zgrid, vs0, w.periods, iwave=1, igr=1, nthreads=8)
    rl = orc.forward_for_events(w.xx_deg, w.yy_deg, u0, m11, m12, m22, ev_l, calc_adj=True,
                                nthreads=8)
    sv, sr, st = orc.depthkernel_love(w.zgrid, vs0, w.periods, igr=1, nthreads=8)
    assert st.sum() == 0
    vp0 = np.vectorize(orc.vs2vp)(vs0)
    kref = orc.combine_kernels_vs(rl["adj_s"], vs0, vp0, sv, np.zeros_like(sv), sr)
    plan, g, tt, wt, t = _grad(w, ev_l, "fp64")
    g_love = inversion.MisfitGradient(plan, w.zgrid, w.periods, data_type="gr", wave="love")
    out = g_love.run(t(vs0), tt, wt)
    torch.cuda.synchronize()
    assert int(out["status"][0]) == 0
    assert abs(float(out["chi"][0]) - rl["chi"]) <= 1e-12 * abs(rl["chi"])
    ker = out["ker_vs"].cpu().numpy()
    assert np.abs(ker - kref).max() <= 1e-12 * np.abs(kref).max()
    g_ph = inversion.MisfitGradient(plan, w.zgrid, w.periods, data_type="ph", wave="love")
    with pytest.raises(_capi.SAError):
        g_ph.run(t(vs0), tt, wt)
