"""One persistent launch over plans of different grid size (sa_multi): two
levels of the topography workload (41^2 and 61^2 over the same span, general
metric from the fractal topography, a handful of sources per period) solved
in one launch must give each plan's own results -- FP64: synthetic times
and misfit bit for bit, adj_s to 1e-12 of its maximum (FP64 atomics in
completion order); FP32: within the FP32 path's bars (1e-4 s, 1e-4 relative
L2) -- on the first evaluation and on the second, whose queue is
ordered by the first one's work across the levels."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _level(level):
    import torch
    from surfattpp_b200 import surfgrid
    from surfattpp_b200 import workloads as W
    w = W.config4(level=level, nsta=25, nper=4, lam=5.0, src_range=(3, 6))
    lon, lat, z = w.meta["topo_raw"]
    avg = surfgrid.average_phase_velocity(w.zgrid, w.meta["vs1d"], w.periods)
    sig = surfgrid.sigma_deg(avg, w.periods, w.meta["wavelen_factor"])
    zg = surfgrid.grid_topography(lon, lat, z, w.xx_deg, w.yy_deg)
    m11, m12, m22, _ = surfgrid.build_media_with_topo(w.xx_deg, w.yy_deg, zg, sig)
    X, Y = np.meshgrid(w.xx_deg, w.yy_deg)
    svel = np.stack([avg[k] * (1.0 + 0.03 * np.sin(9 * X + k) * np.cos(7 * Y))
                     for k in range(w.nper)])
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    ev = w.events()
    return w, ev, t(svel), t(ev["tt_obs"]), t(ev["weight"]), (m11, m12, m22)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_multi_grid_launch_equals_plans(gpu, precision):
    import torch
    from surfattpp_b200 import preproc
    levels = [_level(41), _level(61)]
    plans = [preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                        ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                        ev["stla"], precision=precision)
             for w, ev, *_ in levels]
    want = []
    for p, (w, ev, sv, tt, wt, m) in zip(plans, levels):
        o = p.run(sv, tt, wt, m11=m[0], m12=m[1], m22=m[2])
        torch.cuda.synchronize()
        want.append({k: v.clone() for k, v in o.items()})
    multi = preproc.MultiPlan(plans)
    args = [list(x) for x in zip(*[(sv, tt, wt) for _, _, sv, tt, wt, _ in levels])]
    media = [list(x) for x in zip(*[m for *_, m in levels])]
    for _ in range(2):
        outs = multi.run(*args, m11=media[0], m12=media[1], m22=media[2])
        torch.cuda.synchronize()
        assert multi.worst_status() == 0
        for o, ref, (w, ev, *_) in zip(outs, want, levels):
            npair = ev["rec_idx"].size
            syn, syn_ref = o["syn"][:npair], ref["syn"][:npair]
            adj, adj_ref = o["adj_s"].cpu().numpy(), ref["adj_s"].cpu().numpy()
            if precision == "fp64":
                assert torch.equal(syn, syn_ref)
                assert torch.equal(o["chi"], ref["chi"])
                assert np.abs(adj - adj_ref).max() <= 1e-12 * np.abs(adj_ref).max()
            else:
                assert float((syn - syn_ref).abs().max()) <= 1e-4
                assert np.linalg.norm(adj - adj_ref) <= 1e-4 * np.linalg.norm(adj_ref)
                chi, chi_ref = float(o["chi"][0]), float(ref["chi"][0])
                assert abs(chi - chi_ref) <= 1e-4 * chi_ref
    assert multi.kernel_ms() > 0.0
    multi.close()
    for p in plans:
        p.close()
