"""The exact gradient of the discrete forward model on the device (FP64 plan
with the adjoint set to "exact"), on the checkerboard case (41x41x30, 10
periods, 250 events, observed times from the checkerboard model):

* receiver times after forward solves to a fixed point equal the oracle's
  (1e-12 relative; the FP64 sweeps round as the oracle's);
* dchi/dsvel of the discrete adjoint equals the oracle's (1e-9 of its
  maximum: the device sweeps lambda Gauss-Seidel, the oracle by Jacobi
  iteration, so the sums round differently);
* dc/dvs from the phase-velocity roots equals the oracle's (1e-6 relative
  to each column's largest value: both difference the layer matrices);
* the autograd gradient of chi built in torch on TravelTimes with
  convention "exact" matches central differences of chi (+-1e-2 km/s,
  oracle forward solves to a fixed point) within 1e-3 on 12 nodes where it
  exceeds 5 % of its maximum, and sa_grad_run on the same plan returns the
  same gradient (1e-12 of its maximum).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2(orc):
    from surfattpp_b200 import workloads as W
    w = W.config1()
    ev = w.events()
    m11, m12, m22 = w.media()
    sv_true, st = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    assert st.sum() == 0
    ev["tt_obs"] = orc.discrete_for_events(w.xx_deg, w.yy_deg, sv_true, m11, m12, m22, ev,
                                           tol=0.0, grad=False, nthreads=8)["syn"].copy()
    return w, ev, w.meta["vs_start"]


def _plan(w, ev):
    from surfattpp_b200 import inversion, preproc
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp64")
    plan.set_adjoint("exact")
    return plan, inversion.MisfitGradient(plan, w.zgrid, w.periods)


def _t(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda:0")


def test_discrete_adjoint_matches_oracle(c2, gpu, orc):
    import torch
    w, ev, vs0 = c2
    plan, g = _plan(w, ev)
    sv0, _ = orc.fwdsurf(w.zgrid, vs0, w.periods, nthreads=8)
    m11, m12, m22 = w.media()
    ref = orc.discrete_for_events(w.xx_deg, w.yy_deg, sv0, m11, m12, m22, ev, tol=0.0,
                                  nthreads=8)
    out = plan.run(_t(sv0), _t(ev["tt_obs"]), _t(ev["weight"]))
    torch.cuda.synchronize()
    assert int(out["status"][0]) == 0
    syn = out["syn"].cpu().numpy()[: ref["syn"].size]
    assert np.max(np.abs(syn - ref["syn"]) / ref["syn"]) <= 1e-12
    assert abs(float(out["chi"][0]) - ref["chi"]) <= 1e-12 * ref["chi"]
    got = out["adj_s"].cpu().numpy()
    scale = np.abs(ref["grad_svel"]).max()
    assert np.max(np.abs(got - ref["grad_svel"])) <= 1e-9 * scale


def test_root_derivatives_match_oracle(c2, gpu, orc):
    import torch
    from exact_chain import dcdvs_nodes
    w, ev, vs0 = c2
    vs = vs0[::4, ::4].copy()
    sv, _ = orc.fwdsurf(w.zgrid, vs, w.periods, nthreads=8)
    ref = dcdvs_nodes(orc, w.zgrid, vs, w.periods, sv)
    # a one-event plan on the coarse grid owns the handle
    from surfattpp_b200 import preproc, inversion
    xx, yy = w.xx_deg[::4], w.yy_deg[::4]
    p2 = preproc.ForwardAdjointPlan(xx, yy, w.nper, np.array([xx[2]]), np.array([yy[2]]),
                                    np.array([0]), np.array([0, 1]), np.array([0]),
                                    np.array([xx[5]]), np.array([yy[6]]), precision="fp64")
    g2 = inversion.MisfitGradient(p2, w.zgrid, w.periods)
    got = g2.dcdvs(_t(vs))
    torch.cuda.synchronize()
    got = got.cpu().numpy()
    colmax = np.abs(ref).max(axis=2, keepdims=True)
    assert np.max(np.abs(got - ref) / np.maximum(colmax, 1e-30)) <= 1e-6


def test_exact_gradient_matches_differences(c2, gpu, orc):
    import torch
    from surfattpp_b200 import inversion
    w, ev, vs0 = c2
    plan, g = _plan(w, ev)
    tt, wt = _t(ev["tt_obs"]), _t(ev["weight"])
    vs = _t(vs0).requires_grad_(True)
    chi = inversion.misfit(g, vs, tt, wt, convention="exact")
    chi.backward()
    torch.cuda.synchronize()
    ker = vs.grad.cpu().numpy()
    assert int(g.last_status[0]) == 0
    # the fused evaluation on the same plan gives the same gradient
    out = g.run(_t(vs0), tt, wt)
    torch.cuda.synchronize()
    assert np.max(np.abs(out["ker_vs"].cpu().numpy() - ker)) <= 1e-12 * np.abs(ker).max()
    m11, m12, m22 = w.media()

    def chi_of(v):
        sv, _ = orc.fwdsurf(w.zgrid, v, w.periods, nthreads=8)
        return orc.discrete_for_events(w.xx_deg, w.yy_deg, sv, m11, m12, m22, ev, tol=0.0,
                                       grad=False, nthreads=8)["chi"]

    big = np.argwhere(np.abs(ker[:, :, :-1]) > 0.05 * np.abs(ker).max())
    nodes = big[np.random.default_rng(2002).choice(len(big), size=12, replace=False)]
    h = 1e-2
    ratios = []
    for i, j, k in nodes:
        vp, vm = vs0.copy(), vs0.copy()
        vp[i, j, k] += h
        vm[i, j, k] -= h
        ratios.append((chi_of(vp) - chi_of(vm)) / (2 * h) / ker[i, j, k])
    ratios = np.array(ratios)
    assert np.all(np.abs(ratios - 1.0) <= 1e-3), ratios


def test_discrete_adjoint_on_topography_and_deterministic(gpu, orc):
    """General (anisotropic) metric from fractal topography: the winner's
    metric comes from the per-period media planes.  With event-order
    accumulation the result is reproducible bit for bit and agrees with the
    atomic one."""
    import torch
    from surfattpp_b200 import preproc
    from surfattpp_b200 import workloads as W
    c4 = W.config4(level=61, nsta=41, nper=4, src_range=(3, 5), lam=8.0)
    lon, lat, z = c4.meta["topo_raw"]
    X, Y = np.meshgrid(c4.xx_deg, c4.yy_deg)
    zg = orc.interp2d(lon, lat, z, X.ravel(), Y.ravel()).reshape(X.shape)
    m11, m12, m22, _ = orc.topo_media(c4.xx_deg, c4.yy_deg, zg, np.full(c4.nper, 0.05))
    svel, st = orc.fwdsurf(c4.zgrid, c4.vs3d, c4.periods, nthreads=8)
    assert st.sum() == 0
    ev = c4.events()
    ev["tt_obs"] = np.asarray(ev["tt_obs"]) * 1.01
    ref = orc.discrete_for_events(c4.xx_deg, c4.yy_deg, svel, m11, m12, m22, ev, tol=0.0,
                                  nthreads=8)
    plan = preproc.ForwardAdjointPlan(c4.xx_deg, c4.yy_deg, c4.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp64")
    plan.set_adjoint("exact")
    args = dict(m11=_t(m11), m12=_t(m12), m22=_t(m22))
    tt, wt = _t(ev["tt_obs"]), _t(ev["weight"])
    out = plan.run(_t(svel), tt, wt, **args)
    torch.cuda.synchronize()
    assert int(out["status"].max()) == 0
    syn = out["syn"].cpu().numpy()[: ref["syn"].size]
    assert np.max(np.abs(syn - ref["syn"]) / ref["syn"]) <= 1e-12
    got = out["adj_s"].cpu().numpy()
    scale = np.abs(ref["grad_svel"]).max()
    assert scale > 0
    assert np.max(np.abs(got - ref["grad_svel"])) <= 1e-9 * scale
    plan.set_deterministic(True)
    a = plan.run(_t(svel), tt, wt, **args)["adj_s"].clone()
    b = plan.run(_t(svel), tt, wt, **args)["adj_s"].clone()
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert np.max(np.abs(a.cpu().numpy() - got)) <= 1e-12 * scale


def test_exact_adjoint_edge_cases(c2, gpu, orc):
    """An event without receivers, receivers outside the grid (NaN times, as
    interp2d; they add nothing to the adjoint source) and a receiver on the
    grid's edge, against the oracle; an FP32 plan refuses the exact adjoint."""
    import torch
    from surfattpp_b200 import _capi, preproc
    w, ev, vs0 = c2
    xx, yy = w.xx_deg, w.yy_deg
    stlo = np.array([xx[5], xx[30], xx[0], xx[-1] + 1.0, xx[12]])
    stla = np.array([yy[7], yy[33], yy[20], yy[10], yy[-1]])
    evlo = np.array([xx[20], xx[10], xx[25]])
    evla = np.array([yy[21], yy[30], yy[8]])
    iper = np.array([0, 3, 7], np.int32)
    rec_ptr = np.array([0, 4, 4, 8], np.int32)          # event 1 has no receivers
    rec_idx = np.array([0, 1, 2, 3, 1, 2, 3, 4], np.int32)
    e = dict(evlo=evlo, evla=evla, iper=iper, rec_ptr=rec_ptr, rec_idx=rec_idx, stlo=stlo,
             stla=stla, weight=np.ones(8), tt_obs=np.full(8, 30.0))
    sv0, _ = orc.fwdsurf(w.zgrid, vs0, w.periods, nthreads=8)
    m11, m12, m22 = w.media()
    ref = orc.discrete_for_events(xx, yy, sv0, m11, m12, m22, e, tol=0.0, nthreads=1)
    plan = preproc.ForwardAdjointPlan(xx, yy, w.nper, evlo, evla, iper, rec_ptr, rec_idx, stlo,
                                      stla, precision="fp64")
    plan.set_adjoint("exact")
    out = plan.run(_t(sv0), _t(e["tt_obs"]), _t(e["weight"]))
    torch.cuda.synchronize()
    syn = out["syn"].cpu().numpy()[:8]
    assert np.array_equal(np.isnan(syn), np.isnan(ref["syn"]))
    assert np.isnan(syn[3]) and np.isnan(syn[6])
    ok = ~np.isnan(ref["syn"])
    assert np.max(np.abs(syn[ok] - ref["syn"][ok]) / ref["syn"][ok]) <= 1e-12
    got = out["adj_s"].cpu().numpy()
    assert np.all(np.isfinite(got))
    scale = np.abs(ref["grad_svel"]).max()
    assert scale > 0
    assert np.max(np.abs(got - ref["grad_svel"])) <= 1e-9 * scale
    assert not np.any(got[3]) and not np.any(ref["grad_svel"][3])   # event 1's period
    p32 = preproc.ForwardAdjointPlan(xx, yy, w.nper, evlo, evla, iper, rec_ptr, rec_idx, stlo,
                                     stla, precision="fp32")
    with pytest.raises(_capi.SAError):
        p32.set_adjoint("exact")
