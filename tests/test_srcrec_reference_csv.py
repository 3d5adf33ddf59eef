"""SrcRec::load / get_periods / get_events (reference src/src_rec.cpp:20-264)
on the reference's own example tables (examples/00_checkerboard_iso,
copied to tests/golden/ by make_fixtures.py): 4800 observations, 16
periods, 24 sources (each station pair once, so the last station is never a
source), one event per (source, period) -- 384 events with ragged receiver
lists of 1 to 24 -- in the std::map order of the "{evtname}_{iper}" keys
(lexicographic: MX00_0, MX00_1, MX00_10, ...), each event's receivers the
matching rows in file order (:147-168).  Checked against the plain-Python
restatement of tests/test_srcrec.py; mean velocities to 1e-12 relative."""
import csv
import os

import numpy as np
import pytest

from test_srcrec import _restated

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["src_rec_file_ph.csv", "src_rec_file_gr.csv"])
def test_reference_example_table(name):
    from surfattpp_b200.srcrec import SrcRec
    path = os.path.join(GOLDEN, name)
    with open(path, newline="") as f:
        rows = list(csv.DictReader(f))
    sr = SrcRec(path)
    per, meanvel, dist, keys, evs = _restated(rows)
    assert sr.n_obs == len(rows) == 4800
    assert list(sr.periods) == per and len(per) == 16
    assert np.allclose(sr.meanvel, meanvel, rtol=1e-12, atol=0)
    assert np.allclose(sr.obs["dist"], dist, rtol=1e-12, atol=0)
    assert len(keys) == 384 and keys[:3] == ["MX00_0", "MX00_1", "MX00_10"]
    assert sr.event_names == keys
    for e, k in enumerate(keys):
        ip, idx, lo, la = evs[k]
        assert sr.iper[e] == ip and sr.evlo[e] == lo and sr.evla[e] == la
        assert list(sr.rec_idx[sr.rec_ptr[e]:sr.rec_ptr[e + 1]]) == idx
    sizes = np.diff(sr.rec_ptr)
    assert sizes.min() == 1 and sizes.max() == 24 and sizes.sum() == 4800
    ev = sr.events()
    assert np.array_equal(ev["tt_obs"], sr.obs["tt"][sr.rec_idx])
