"""Tail teams of the FP32 batch kernel (launch variants with bit 2 set): warps
without an event join the solves still running in their block and march
their strips pipelined behind each other.

Bar (written here): a team updates every cell exactly as the warp alone, with
the same explicit FP32 operations, and adds the L1 sums per strip in strip
order, so every team configuration gives the receiver times, iteration
counts, misfit and -- summed in event order (deterministic mode) -- adj_s of
variant 0 bit for bit.  Configurations: one slot per block (every solve
marched by a team of four warps from its first iteration), three slots per
block (teams of two), and all slots with more events than slots (teams form
in the queue's tail and grow from one iteration to the next).  No event may
report a team wait that gave up (status 7).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(n, nsta, nper, seed):
    import torch
    from surfattpp_b200 import preproc, surfker
    from surfattpp_b200 import workloads as W
    w = W.config3(seed=seed, nsta=nsta, nper=nper, n=n)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    sv, st = surfker.fwdsurf(w.zgrid, t(w.vs3d), w.periods)
    torch.cuda.synchronize()
    ev = w.events()
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp32")
    plan.set_deterministic(True)
    return plan, sv, t(ev["tt_obs"]), t(ev["weight"]), len(ev["evlo"])


def _outputs(plan, sv, tt, wt, variant, active, ne):
    import torch
    plan.set_tune(variant, active)
    out = plan.run(sv, tt, wt)
    plan.run(sv, tt, wt, out=out)    # second launch: queue in cost order
    torch.cuda.synchronize()
    return {k: out[k].cpu().numpy()[:ne] if k in ("fwd_iters", "adj_iters", "status")
            else out[k].cpu().numpy() for k in ("syn", "adj_s", "chi", "fwd_iters", "adj_iters",
                                                 "status")}


@pytest.mark.parametrize("n, nsta, nper, seed, share",
                         [(101, 40, 3, 5, 4), (101, 40, 3, 5, 4 / 3), (61, 200, 15, 6, 1)],
                         ids=["block-per-solve", "teams-of-two", "queue-tail"])
def test_teams_match_the_warp_alone(gpu, n, nsta, nper, seed, share):
    plan, sv, tt, wt, ne = _case(n, nsta, nper, seed)
    nslots = plan.tune()["nslots"]
    active = 0 if share == 1 else max(1, int(nslots / share))
    if share == 1:
        assert ne > nslots   # the queue outlasts the first pull
    a = _outputs(plan, sv, tt, wt, 0, 0, ne)
    b = _outputs(plan, sv, tt, wt, 4, active, ne)
    assert a["status"].max() == 0 and b["status"].max() == 0
    for k in ("syn", "fwd_iters", "adj_iters", "chi", "adj_s"):
        assert np.array_equal(a[k], b[k]), k
    plan.close()
