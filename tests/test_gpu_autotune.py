"""The batch-kernel launch autotuner (sa_plan_autotune / sa_plan_set_tune).

Bars (written here):
  * FP64 plans (one kernel, all or part of the slots): synthetic times and
    iteration counts bit for bit, misfit to 1e-12 relative, adj_s to 1e-12 of
    its maximum (FP64 atomics accumulate in completion order).
  * FP32 variants (forward step rolled or unrolled, adjoint lead 2 or 3,
    tail teams on or off) run the same explicit operations -- every product,
    sum and fused multiply-add of the sweeps is spelled out -- so synthetic
    times and iteration counts are bit for bit the same, the misfit to 1e-12
    relative and adj_s to 1e-12 of its maximum (FP64 atomics).
The autotuner times every candidate on the plan's own workload, keeps the
fastest and hands it to later plans of the same grid size.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(precision, nsta=25, n=None):
    import torch
    from surfattpp_b200 import preproc
    from surfattpp_b200 import workloads as W
    w = W.config1() if n is None else W.config3(nsta=nsta, nper=4, n=n)
    ev = w.events()
    X, Y = np.meshgrid(w.xx_deg, w.yy_deg)
    svel = np.stack([3.0 + 0.2 * k + 0.1 * np.sin(9 * X + k) * np.cos(7 * Y)
                     for k in range(w.nper)])
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    mk = lambda: preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                           ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                           ev["stla"], precision=precision)
    return mk, t(svel), t(ev["tt_obs"]), t(ev["weight"])


def _run(plan, sv, tt, wt):
    import torch
    out = plan.run(sv, tt, wt)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy().copy() for k, v in out.items()}


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_every_configuration_gives_the_same_results(gpu, precision):
    mk, sv, tt, wt = _setup(precision)
    plan = mk()
    ref = _run(plan, sv, tt, wt)
    nslots = plan.tune()["nslots"]
    nvar = 8 if precision == "fp32" else 1
    for v in range(nvar):
        for active in (0, max(1, nslots // 3)):
            plan.set_tune(v, active)
            got = _run(plan, sv, tt, wt)
            assert plan.tune()["variant"] == v
            assert np.array_equal(got["syn"], ref["syn"]), (v, active)
            assert np.array_equal(got["fwd_iters"], ref["fwd_iters"]), (v, active)
            assert np.array_equal(got["adj_iters"], ref["adj_iters"]), (v, active)
            assert abs(got["chi"][0] - ref["chi"][0]) <= 1e-12 * abs(ref["chi"][0])
            scale = np.abs(ref["adj_s"]).max()
            assert np.abs(got["adj_s"] - ref["adj_s"]).max() <= 1e-12 * scale
    with pytest.raises(RuntimeError):
        plan.set_tune(nvar, 0)


def test_autotune_picks_and_hands_on(gpu):
    import torch
    mk, sv, tt, wt = _setup("fp32", n=101, nsta=40)
    plan = mk()
    ref = _run(plan, sv, tt, wt)
    adj = torch.empty_like(torch.as_tensor(ref["adj_s"], device=sv.device))
    res = plan.autotune(sv, tt, wt, adj_s=adj)
    # 8 variants x (all, 3/4 of the slots) + the 4 team variants x 1/4
    assert len(res["ms"]) == 20 and all(m > 0 for m in res["ms"])
    assert res["choice"] == int(np.argmin(res["ms"]))
    got = _run(plan, sv, tt, wt)
    assert np.array_equal(got["syn"], ref["syn"])
    # a later plan of the same grid size starts from the tuned configuration
    plan2 = mk()
    assert plan2.tune()["variant"] == res["variant"]
    assert plan2.tune()["active_slots"] == res["active_slots"]
