"""Observation table and event builder (SrcRec::load / get_periods /
get_events / write, reference src/src_rec.cpp:20-264, :407-457): host code
of the library checked against a plain-Python restatement on seeded
synthetic tables (no GPU).  Bars: periods, counts, event order and receiver
rows identical; mean velocities and default distances to 1e-12 relative;
writing then reading reproduces the table to the written precision."""
import csv
import math
import os

import numpy as np
import pytest

pytestmark = []


def _table(path, rng, with_optional):
    names = [f"ST{k:02d}" for k in range(12)]
    lat = 24.0 + rng.uniform(0, 1, 12)
    lon = 102.0 + rng.uniform(0, 1, 12)
    periods = [4.0, 8.0, 12.5, 20.0, 40.0]
    rows = []
    for s in range(12):
        for p in periods:
            for r in range(12):
                if r == s or rng.random() < 0.3:
                    continue
                tt = 10 + 30 * rng.random()
                row = dict(tt=f"{tt:.6f}", staname=names[r], stla=f"{lat[r]:.4f}",
                           stlo=f"{lon[r]:.4f}", evtname=names[s], evla=f"{lat[s]:.4f}",
                           evlo=f"{lon[s]:.4f}", period=f"{p:.2f}")
                if with_optional:
                    row.update(weight=f"{0.5 + rng.random():.4f}", dist="%.3f" % (50 + r),
                               vel=f"{3 + rng.random():.6f}")
                rows.append(row)
    order = rng.permutation(len(rows))
    rows = [rows[i] for i in order]
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=list(rows[0].keys()))
        w.writeheader()
        w.writerows(rows)
    return rows


def _restated(rows):
    """src/src_rec.cpp:20-228 in plain Python."""
    f = lambda r, k: float(r[k])
    n = len(rows)

    def gps2dist(la0, lo0, la1, lo1):
        d2r = math.pi / 180.0
        dlat, dlon = (la0 - la1) * d2r, (lo1 - lo0) * d2r
        a = math.sin(dlat * 0.5) ** 2 + math.sin(dlon * 0.5) ** 2 * math.cos(la0 * d2r) * math.cos(la1 * d2r)
        return 6371.0 * 2.0 * math.atan2(math.sqrt(a), math.sqrt(1.0 - a))

    dist = [f(r, "dist") if "dist" in r else gps2dist(f(r, "stla"), f(r, "stlo"), f(r, "evla"),
                                                      f(r, "evlo")) for r in rows]
    vel = [f(r, "vel") if "vel" in r else (dist[i] / f(r, "tt") if f(r, "tt") > 0 else 0.0)
           for i, r in enumerate(rows)]
    per = sorted(set(f(r, "period") for r in rows))
    meanvel = [np.mean([vel[j] for j in range(n) if abs(f(rows[j], "period") - p) < 1e-6])
               for p in per]
    evs = {}
    for src in sorted(set(r["evtname"] for r in rows)):
        for ip, p in enumerate(per):
            idx = [i for i in range(n) if rows[i]["evtname"] == src
                   and abs(p - f(rows[i], "period")) < 1e-6]
            if idx:
                evs[f"{src}_{ip}"] = (ip, idx, f(rows[idx[-1]], "evlo"), f(rows[idx[-1]], "evla"))
    keys = sorted(evs)          # std::map order
    return per, meanvel, dist, keys, evs


@pytest.mark.parametrize("with_optional", [False, True])
def test_event_builder(tmp_path, with_optional):
    from surfattpp_b200.srcrec import SrcRec
    rng = np.random.default_rng(3 + with_optional)
    p = tmp_path / "src_rec.csv"
    rows = _table(p, rng, with_optional)
    sr = SrcRec(p)
    per, meanvel, dist, keys, evs = _restated(rows)
    assert sr.n_obs == len(rows)
    assert list(sr.periods) == per
    assert np.allclose(sr.meanvel, meanvel, rtol=1e-12, atol=0)
    assert np.allclose(sr.obs["dist"], dist, rtol=1e-12, atol=0)
    assert sr.event_names == keys
    for e, k in enumerate(keys):
        ip, idx, lo, la = evs[k]
        assert sr.iper[e] == ip and sr.evlo[e] == lo and sr.evla[e] == la
        assert list(sr.rec_idx[sr.rec_ptr[e]:sr.rec_ptr[e + 1]]) == idx
    ev = sr.events()
    assert np.array_equal(ev["tt_obs"], sr.obs["tt"][sr.rec_idx])
    if not with_optional:
        assert np.all(sr.obs["weight"] == 1.0)


def test_write_roundtrip(tmp_path):
    from surfattpp_b200.srcrec import SrcRec
    rng = np.random.default_rng(9)
    p = tmp_path / "in.csv"
    _table(p, rng, True)
    sr = SrcRec(p)
    q = tmp_path / "out.csv"
    syn = sr.obs["tt"][sr.rec_idx] * 1.01
    sr.write(q, sr.tt_fwd(syn))
    back = SrcRec(q)
    assert back.n_obs == sr.n_obs and back.event_names == sr.event_names
    assert np.allclose(back.obs["tt"], sr.obs["tt"] * 1.01, atol=5e-7, rtol=0)
    assert np.allclose(back.obs["vel"], sr.obs["dist"] / (sr.obs["tt"] * 1.01), atol=5e-6)
    with open(q) as f:
        assert f.readline().strip() == "tt,staname,stla,stlo,evtname,evla,evlo,period,weight,dist,vel"


def test_missing_column_raises(tmp_path):
    from surfattpp_b200.srcrec import SrcRec
    p = tmp_path / "bad.csv"
    p.write_text("tt,staname,stla\n1,A,2\n")
    with pytest.raises(ValueError):
        SrcRec(p)
    with pytest.raises(ValueError):
        SrcRec(tmp_path / "nope.csv")
