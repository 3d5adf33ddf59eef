"""GPU parity: preproc::forward_for_event batches against the CPU oracle.

Bars (written here): FP64 path <= 1e-12 relative on synthetic times, misfit
and adj_s with the oracle's per-event iteration counts; FP32 path
<= 1e-4 s max travel-time error and <= 1e-4 relative L2 on adj_s."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def assert_within(got, want, bound):
    bad = np.abs(got - want) > bound
    if bad.any():
        i = np.unravel_index(np.argmax(np.abs(got - want) - bound), got.shape)
        raise AssertionError(f"{bad.sum()} cells outside bound; worst at {i}: got {got[i]!r} "
                             f"want {want[i]!r} bound {bound[i]!r}")


def adj_bound(orc, w, svel, ev, ref, syn_gpu):
    """Elementwise error bound for adj_s = sum_e Ta_e * svel^-3.

    The adjoint is linear in the receiver residuals r and its Green's
    functions are non-negative, so running the oracle with residuals
    q = 1e-12*|r| + |syn_gpu - syn_ref| gives sum_i q_i G_i: FP64 rounding of
    every accumulated term (1e-12 relative, accumulation order differs:
    device atomics vs event order) plus the exact propagation of the
    synthetic-time differences into the residuals (r is a difference of
    nearly equal times, so its relative error exceeds that of T)."""
    ev2 = dict(ev)
    r = ref["syn"] - ev["tt_obs"]
    q = 1e-12 * np.abs(r) + np.abs(syn_gpu - ref["syn"])
    ev2["tt_obs"] = ref["syn"] - q
    m11, m12, m22 = w.media()
    return orc.forward_for_events(w.xx_deg, w.yy_deg, svel, m11, m12, m22, ev2,
                                  calc_adj=True, nthreads=8)["adj_s"]


@pytest.fixture(scope="module")
def c1(orc):
    from surfattpp_b200 import workloads as W
    w = W.config1()
    svel, st = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    assert st.sum() == 0
    m11, m12, m22 = w.media()
    ev = w.events()
    obs = orc.forward_for_events(w.xx_deg, w.yy_deg, svel, m11, m12, m22, ev, calc_adj=False,
                                 nthreads=8)
    ev["tt_obs"] = obs["syn"].copy()
    svel0, _ = orc.fwdsurf(w.zgrid, w.meta["vs_start"], w.periods, nthreads=8)
    ref = orc.forward_for_events(w.xx_deg, w.yy_deg, svel0, m11, m12, m22, ev, calc_adj=True,
                                 nthreads=8)
    return w, svel0, ev, ref


def test_c1_fp64_parity(c1, gpu, orc):
    from surfattpp_b200 import preproc
    w, svel0, ev, ref = c1
    out = preproc.forward_for_event(w.xx_deg, w.yy_deg, svel0, ev, calc_adj=True,
                                    precision="fp64")
    assert np.array_equal(out["fwd_iters"], ref["fwd_iters"])
    assert np.array_equal(out["adj_iters"], ref["adj_iters"])
    assert np.max(np.abs(out["syn"] - ref["syn"]) / np.abs(ref["syn"])) <= 1e-12
    assert abs(out["chi"] - ref["chi"]) <= 1e-12 * abs(ref["chi"])
    bound = adj_bound(orc, w, svel0, ev, ref, out["syn"])
    assert_within(out["adj_s"], ref["adj_s"], 2.0 * bound + 1e-300)


def test_c1_fp32_tolerance(c1, gpu):
    from surfattpp_b200 import preproc
    w, svel0, ev, ref = c1
    out = preproc.forward_for_event(w.xx_deg, w.yy_deg, svel0, ev, calc_adj=True,
                                    precision="fp32")
    assert np.max(np.abs(out["syn"] - ref["syn"])) <= 1e-4
    l2 = np.linalg.norm(out["adj_s"] - ref["adj_s"]) / np.linalg.norm(ref["adj_s"])
    assert l2 <= 1e-4
    assert abs(out["chi"] - ref["chi"]) <= 1e-3 * abs(ref["chi"])


def test_c3_subset_parity(orc, gpu):
    """8 events at the 301x301 batched-workload resolution."""
    from surfattpp_b200 import preproc
    from surfattpp_b200 import workloads as W
    w = W.config3(nsta=4, nper=2)
    svel, st = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    m11, m12, m22 = w.media()
    ev = w.events()
    ref = orc.forward_for_events(w.xx_deg, w.yy_deg, svel, m11, m12, m22, ev, calc_adj=True,
                                 nthreads=8)
    o64 = preproc.forward_for_event(w.xx_deg, w.yy_deg, svel, ev, precision="fp64")
    assert np.array_equal(o64["fwd_iters"], ref["fwd_iters"])
    assert np.array_equal(o64["adj_iters"], ref["adj_iters"])
    assert np.max(np.abs(o64["syn"] - ref["syn"]) / np.abs(ref["syn"])) <= 1e-12
    bound = adj_bound(orc, w, svel, ev, ref, o64["syn"])
    assert_within(o64["adj_s"], ref["adj_s"], 2.0 * bound + 1e-300)
    o32 = preproc.forward_for_event(w.xx_deg, w.yy_deg, svel, ev, precision="fp32")
    assert np.max(np.abs(o32["syn"] - ref["syn"])) <= 1e-4
    l2 = np.linalg.norm(o32["adj_s"] - ref["adj_s"]) / np.linalg.norm(ref["adj_s"])
    assert l2 <= 1e-4


def test_ragged_and_empty_receivers(orc, gpu):
    """Events with 0, 1 and many receivers in one batch; one receiver outside
    the grid gives NaN (include/utils.h:378-381) in both implementations."""
    from surfattpp_b200 import preproc
    from surfattpp_b200 import workloads as W
    w = W.config1()
    svel, _ = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    stlo = np.r_[w.stlo[:6], 150.0]
    stla = np.r_[w.stla[:6], 24.5]
    ev = dict(evlo=np.array([w.stlo[0], w.stlo[1], w.stlo[2]]),
              evla=np.array([w.stla[0], w.stla[1], w.stla[2]]),
              iper=np.array([0, 3, 9], np.int32),
              rec_ptr=np.array([0, 0, 1, 6], np.int32),
              rec_idx=np.array([3, 1, 3, 4, 5, 6], np.int32),
              stlo=stlo, stla=stla, tt_obs=np.zeros(6), weight=np.ones(6))
    m11, m12, m22 = w.media()
    ref = orc.forward_for_events(w.xx_deg, w.yy_deg, svel, m11, m12, m22, ev, calc_adj=False)
    out = preproc.forward_for_event(w.xx_deg, w.yy_deg, svel, ev, calc_adj=False)
    assert np.isnan(ref["syn"][-1]) and np.isnan(out["syn"][-1])
    ok = ~np.isnan(ref["syn"])
    assert np.max(np.abs(out["syn"][ok] - ref["syn"][ok]) / ref["syn"][ok]) <= 1e-12


def test_plan_graph_replay_is_stable(orc, gpu):
    """One plan, several evaluations: CUDA-graph replay and direct launches
    agree; misfit is bitwise reproducible (fixed-order event sum)."""
    import torch
    from surfattpp_b200 import preproc
    from surfattpp_b200 import workloads as W
    w = W.config1()
    svel, _ = orc.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=8)
    ev = w.events()
    ev["tt_obs"] = np.full(ev["rec_idx"].size, 10.0)
    dev = torch.device("cuda:0")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp64", graph=True)
    sv, tt, wt = t(svel), t(ev["tt_obs"]), t(ev["weight"])
    outs = []
    o = None
    for _ in range(3):       # first call captures the graph, the others replay it
        o = plan.run(sv, tt, wt, out=o)
        torch.cuda.synchronize()
        outs.append({k: v.clone() for k, v in o.items()})
    plan2 = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                       ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                       ev["stla"], precision="fp64", graph=False)
    o2 = plan2.run(sv, tt, wt)
    torch.cuda.synchronize()
    for o in outs[1:] + [o2]:
        assert torch.equal(o["syn"], outs[0]["syn"])
        assert torch.equal(o["chi"], outs[0]["chi"])
        tol = 1e-12 * float(outs[0]["adj_s"].abs().max())
        assert float((o["adj_s"] - outs[0]["adj_s"]).abs().max()) <= tol
    assert int(outs[0]["status"].max()) == 0
