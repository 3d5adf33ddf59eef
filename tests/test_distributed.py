"""Multi-rank host logic on CPU (gloo): the event decomposition of
Parallel::select_rank_for_src (include/parallel.h:39-41) as SrcRec::get_events
applies it (src/src_rec.cpp:136-228), the FP64 rank sums of adj_s and the
misfit (src/preproc.cpp:146, :238) and SrcRec::gather_syn_tt
(src/src_rec.cpp:326-371).

Two gloo ranks each run their shard of the checkerboard event set (41x41,
10 periods, 250 events) through the oracle, reduce, and must reproduce the
single-rank run: synthetic times bit for bit (every event is solved the same
way wherever it runs), adj_s and chi to 1e-13 relative (the same FP64 terms
summed in another order).
"""
import os
import socket

import numpy as np
import pytest


def _case(orc):
    from surfattpp_b200 import workloads as W
    w = W.config1()
    rng = np.random.default_rng(77)
    ev = w.events()
    X, Y = np.meshgrid(w.xx_deg, w.yy_deg)
    svel = np.stack([3.0 + 0.1 * k + 0.08 * np.sin(5 * X + k) * np.cos(7 * Y)
                     for k in range(w.nper)])
    ones = np.ones_like(svel)
    ev["tt_obs"] = rng.uniform(5.0, 60.0, ev["rec_idx"].size)
    ev["weight"] = rng.uniform(0.5, 1.5, ev["rec_idx"].size)
    return w, ev, svel, ones


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, size, port, outdir):
    import datetime
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from surfattpp_b200 import distributed as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w, ev, svel, ones = _case(O)
        loc = D.shard_events(ev, rank, size)
        r = O.forward_for_events(w.xx_deg, w.yy_deg, svel, ones, 0 * ones, ones, loc,
                                 calc_adj=True, nthreads=2)
        adj_s = torch.as_tensor(r["adj_s"].copy())
        chi = torch.tensor([r["chi"]], dtype=torch.float64)
        status = torch.tensor([rank], dtype=torch.int32)
        D.reduce_gradient(adj_s, chi, status)
        syn = D.gather_syn(torch.as_tensor(r["syn"]), loc["obs_ids"], ev["rec_idx"].size)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), adj_s=adj_s.numpy(), chi=chi.numpy(),
                 syn=syn.numpy(), status=status.numpy(), events=loc["event_ids"])
    finally:
        dist.destroy_process_group()


def test_shard_events_partition():
    from surfattpp_b200 import distributed as D
    from surfattpp_b200 import workloads as W
    ev = W.config1().events()
    ne, nobs = len(ev["evlo"]), ev["rec_idx"].size
    for size in (1, 2, 3, 7, 300):
        seen_ev, seen_obs = [], []
        for rank in range(size):
            loc = D.shard_events(ev, rank, size)
            ids = loc["event_ids"]
            assert np.all(ids % size == rank)
            assert loc["rec_ptr"].size == ids.size + 1 and loc["rec_ptr"][0] == 0
            for j, e in enumerate(ids):
                a, b = ev["rec_ptr"][e], ev["rec_ptr"][e + 1]
                la, lb = loc["rec_ptr"][j], loc["rec_ptr"][j + 1]
                assert np.array_equal(loc["rec_idx"][la:lb], ev["rec_idx"][a:b])
                assert np.array_equal(loc["tt_obs"][la:lb], ev["tt_obs"][a:b])
                assert np.array_equal(loc["obs_ids"][la:lb], np.arange(a, b))
            assert np.array_equal(loc["iper"], ev["iper"][ids])
            assert np.array_equal(loc["evlo"], ev["evlo"][ids])
            seen_ev.append(ids)
            seen_obs.append(loc["obs_ids"])
        assert np.array_equal(np.sort(np.concatenate(seen_ev)), np.arange(ne))
        assert np.array_equal(np.sort(np.concatenate(seen_obs)), np.arange(nobs))
    # more ranks than events: the extra ranks hold an empty, well-formed shard
    loc = D.shard_events(ev, ne + 3, ne + 5)
    assert loc["event_ids"].size == 0 and list(loc["rec_ptr"]) == [0]
    with pytest.raises(ValueError):
        D.shard_events(ev, 2, 2)


def test_single_rank_reduce_is_identity():
    import torch
    from surfattpp_b200 import distributed as D
    a = torch.arange(6, dtype=torch.float64).reshape(1, 2, 3)
    c = torch.tensor([2.5], dtype=torch.float64)
    D.reduce_gradient(a, c)
    assert a.sum().item() == 15.0 and c.item() == 2.5
    syn = D.gather_syn(torch.tensor([1.0, 2.0]), [3, 0], 4)
    assert syn.tolist() == [2.0, 0.0, 0.0, 1.0]


def test_two_rank_gloo_matches_single_rank(orc, tmp_path):
    import torch.multiprocessing as mp
    w, ev, svel, ones = _case(orc)
    ref = orc.forward_for_events(w.xx_deg, w.yy_deg, svel, ones, 0 * ones, ones, ev,
                                 calc_adj=True, nthreads=4)
    size, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(size, port, str(tmp_path)), nprocs=size, join=True,
                       start_method="spawn")
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(size)]
    ids = np.sort(np.concatenate([r["events"] for r in res]))
    assert np.array_equal(ids, np.arange(len(ev["evlo"])))
    scale = np.abs(ref["adj_s"]).max()
    for r in res:
        assert np.array_equal(r["syn"], ref["syn"])
        assert np.abs(r["adj_s"] - ref["adj_s"]).max() <= 1e-13 * scale
        assert abs(r["chi"][0] - ref["chi"]) <= 1e-13 * abs(ref["chi"])
        assert r["status"][0] == size - 1
    # both ranks hold the same sums
    assert np.array_equal(res[0]["adj_s"], res[1]["adj_s"])
