"""GPU: an observation table read by SrcRec drives the batched forward /
adjoint (preproc::forward_for_event over SrcRec::events_local) with FP64
parity against the oracle on the same events, and the forward times are
written back as the reference's forward CSV."""
import csv

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_table_to_batch(tmp_path, gpu, orc):
    from surfattpp_b200 import preproc
    from surfattpp_b200 import workloads as W
    from surfattpp_b200.srcrec import SrcRec
    w = W.config1()
    names = [f"ST{k:02d}" for k in range(w.stlo.size)]
    p = tmp_path / "src_rec_file_ph.csv"
    with open(p, "w", newline="") as f:
        wr = csv.writer(f)
        wr.writerow(["tt", "staname", "stla", "stlo", "evtname", "evla", "evlo", "period"])
        src = np.repeat(np.arange(w.stlo.size), w.nper)
        for e in range(0, w.n_events, 7):
            s = src[e]
            for r in w.rec_idx[w.rec_ptr[e]:w.rec_ptr[e + 1]]:
                wr.writerow([f"{20.0 + 0.1 * r:.6f}", names[r], f"{w.stla[r]:.6f}",
                             f"{w.stlo[r]:.6f}", names[s], f"{w.stla[s]:.6f}", f"{w.stlo[s]:.6f}",
                             f"{w.periods[w.iper[e]]:.6f}"])
    sr = SrcRec(p)
    assert sr.nperiod <= w.nper
    svel, st = orc.fwdsurf(w.zgrid, w.vs3d, sr.periods, nthreads=8)
    ev = sr.events()
    m11 = np.ones_like(svel)
    ref = orc.forward_for_events(w.xx_deg, w.yy_deg, svel, m11, np.full_like(svel, -0.0), m11, ev,
                                 calc_adj=True, nthreads=8)
    out = preproc.forward_for_event(w.xx_deg, w.yy_deg, svel, ev, calc_adj=True,
                                    precision="fp64")
    assert np.array_equal(out["fwd_iters"], ref["fwd_iters"])
    assert np.max(np.abs(out["syn"] - ref["syn"]) / np.abs(ref["syn"])) <= 1e-12
    q = tmp_path / "forward_PH.csv"
    sr.write(q, sr.tt_fwd(out["syn"]))
    back = SrcRec(q)
    assert np.allclose(back.obs["tt"][sr.rec_idx], out["syn"], atol=5e-7, rtol=0)
