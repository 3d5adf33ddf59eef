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


def test_c3_full_size_properties(gpu):
    """The full C3 batch (301x301, 400 stations, 20 periods, 8000 FP32
    forward + adjoint solves) checked through size-independent properties
    (the oracle would take minutes here; subsets are compared with it above):
      * every solve converges, every output is finite;
      * straight-path bounds for pairs at least 10 km apart: d / vmax <= T <=
        d / vmin to 1e-3 (the eikonal time is the fastest path; no path is
        faster than the fastest medium, the straight one is no slower than the
        slowest).  Closer pairs lie within a few cells of the source, where the
        discretisation error is a large fraction of T (the FP64 oracle reaches
        d / vmin * 1.016 below 5 km);
      * source-receiver reciprocity T(a -> b) = T(b -> a) for the same pairs:
        max 3e-3, median 1e-4 relative (discretisation around either source:
        the FP64 oracle shows 1.7e-4 / 1.1e-5 over 190 pairs, this run
        1.3e-3 at worst over 1.5 M);
      * adj_s is zero outside the grid interior and the misfit equals the sum
        of 0.5 w r^2 over all observations."""
    import torch
    import bench
    from surfattpp_b200 import preproc
    from surfattpp_b200.workloads import _gc_km

    class A:
        n, nsta, nper, precision = 301, 400, 20, "fp32"

    w, svel = bench.make_inputs(A, 0)
    ev = w.events()
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp32")
    out = plan.run(t(svel), t(ev["tt_obs"]), t(ev["weight"]))
    torch.cuda.synchronize()
    assert int(out["status"].max()) == 0
    syn = out["syn"].cpu().numpy()[: ev["rec_idx"].size]
    adj = out["adj_s"].cpu().numpy()
    assert np.all(np.isfinite(syn)) and np.all(np.isfinite(adj))
    nsta, nper = A.nsta, A.nper
    cnt = np.diff(ev["rec_ptr"])
    src = np.repeat(np.repeat(np.arange(nsta), nper), cnt)
    per = np.repeat(ev["iper"], cnt)
    rec = ev["rec_idx"]
    d = _gc_km(ev["stlo"][src], ev["stla"][src], ev["stlo"][rec], ev["stla"][rec])
    flat = svel.reshape(nper, -1)
    far = d >= 10.0
    assert far.sum() > 0.9 * far.size
    assert (syn * flat.max(1)[per] / d)[far].min() >= 1.0 - 1e-3
    assert (syn * flat.min(1)[per] / d)[far].max() <= 1.0 + 1e-3
    T = np.zeros((nper, nsta, nsta))
    T[per, src, rec] = syn
    D = np.zeros((nsta, nsta))
    D[src, rec] = d
    a, b = np.triu_indices(nsta, 1)
    sel = D[a, b] >= 10.0
    a, b = a[sel], b[sel]
    rel = np.abs(T[:, a, b] - T[:, b, a]) / T[:, a, b]
    assert rel.max() <= 3e-3 and np.median(rel) <= 1e-4, (rel.max(), np.median(rel))
    assert np.all(adj[:, 0, :] == 0) and np.all(adj[:, -1, :] == 0)
    assert np.all(adj[:, :, 0] == 0) and np.all(adj[:, :, -1] == 0)
    r = syn - ev["tt_obs"]
    chi = 0.5 * np.sum(ev["weight"] * r * r)
    assert abs(float(out["chi"][0]) - chi) <= 1e-9 * chi


def test_c3_full_size_fp32_against_fp64(gpu):
    """FP32 accuracy on the whole C3 batch (8000 solves at 301x301): the FP64
    plan is the reference's arithmetic (<= 1e-12 of the oracle in the parity
    tests above), so it serves as the reference at full size.  Bars: max
    travel-time error 1e-4 s, adj_s 1e-4 relative L2, misfit 1e-4 relative."""
    import torch
    import bench
    from surfattpp_b200 import preproc

    class A:
        n, nsta, nper, precision = 301, 400, 20, "fp32"

    w, svel = bench.make_inputs(A, 0)
    ev = w.events()
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    res = {}
    for prec in ("fp64", "fp32"):
        plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                          ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                          ev["stla"], precision=prec)
        out = plan.run(t(svel), t(ev["tt_obs"]), t(ev["weight"]))
        torch.cuda.synchronize()
        assert int(out["status"].max()) == 0
        res[prec] = {k: v.cpu().numpy().copy() for k, v in out.items()}
        plan.close()
    n = ev["rec_idx"].size
    err = np.abs(res["fp32"]["syn"][:n] - res["fp64"]["syn"][:n]).max()
    assert err <= 1e-4, err
    a32, a64 = res["fp32"]["adj_s"], res["fp64"]["adj_s"]
    l2 = np.linalg.norm(a32 - a64) / np.linalg.norm(a64)
    assert l2 <= 1e-4, l2
    c32, c64 = res["fp32"]["chi"][0], res["fp64"]["chi"][0]
    assert abs(c32 - c64) <= 1e-4 * abs(c64)


@pytest.mark.parametrize("chunk_events", [0, 37])
def test_deterministic_adj_s_is_the_reference_sum(c1, gpu, orc, chunk_events):
    """sa_plan_set_deterministic: adj_s and chi summed in event order.  FP64:
    bit-identical to the oracle's single-thread event loop (the reference on
    one MPI rank) evaluated with the device's correctly rounded svel^-3 (the
    C library's pow(svel, -3) misrounds about 0.08 % of its arguments, where
    the C-library oracle's terms differ by one ulp: 1e-12 there); a second
    evaluation, and a run in chunks of 37 events, give the same bits."""
    import torch
    from surfattpp_b200 import preproc
    w, svel0, ev, ref = c1
    m11, m12, m22 = w.media()
    ref1 = orc.forward_for_events(w.xx_deg, w.yy_deg, svel0, m11, m12, m22, ev, calc_adj=True,
                                  nthreads=1, math="cr")
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp64")
    n = w.nx * w.ny
    plan.set_deterministic(True, max_bytes=chunk_events * n * 8)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    sv, tt, wt = t(svel0), t(ev["tt_obs"]), t(ev["weight"])
    outs = []
    for _ in range(2):
        o = plan.run(sv, tt, wt)
        torch.cuda.synchronize()
        outs.append((o["adj_s"].cpu().numpy().copy(), float(o["chi"][0])))
    for adj, chi in outs:
        assert np.array_equal(adj, ref1["adj_s"])
        assert chi == ref1["chi"]
    scale = np.abs(ref["adj_s"]).max()
    assert np.abs(outs[0][0] - ref["adj_s"]).max() <= 1e-12 * scale
    # FP32 plan: reproducible run to run
    p32 = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                     ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                     ev["stla"], precision="fp32")
    p32.set_deterministic(True, max_bytes=chunk_events * n * 8)
    a = p32.run(sv, tt, wt)["adj_s"].clone()
    b = p32.run(sv, tt, wt)["adj_s"].clone()
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    plan.close()
    p32.close()
