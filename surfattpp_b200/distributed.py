"""Multi-rank decomposition of the (source, period) event set.

The reference distributes events over MPI ranks and sums the kernels once
per misfit evaluation; the same layout is kept here, one process per GPU:

* event ``i_src`` -- its position in the sorted (event name, period) list that
  ``SrcRec::get_events`` builds (src/src_rec.cpp:136-228) -- runs on rank
  ``select_rank_for_src(i_src) = i_src % size`` (include/parallel.h:39-41);
* each rank runs its own events as one batch with no exchange inside it;
* afterwards adj_s and the misfit are summed over ranks
  (``mpi.sum_all_all``, src/preproc.cpp:146 and :238), then combined with the
  depth kernels (``preproc::combine_kernels``, src/preproc.cpp:225-304);
* synthetic times go back to their global observation slots
  (``SrcRec::gather_syn_tt``, src/src_rec.cpp:326-371).

The phase velocities (``SurfGrid::fwdsurf``) and the depth kernels are computed
whole on every rank rather than split by column and all-gathered
(src/surf_grid.cpp:194-245): on one GPU they take a few hundred ms for the
largest grid, less than the all-gather of the depth kernels would move.

The reductions go through ``torch.distributed`` (NCCL for device tensors,
gloo for host tensors) and are FP64 sums, like the reference's MPI_SUM.
"""
from __future__ import annotations

import numpy as np


def select_rank_for_src(id_src, size):
    """Parallel::select_rank_for_src (include/parallel.h:39-41)."""
    if size < 1:
        raise ValueError("size must be >= 1")
    return id_src % size


def local_event_ids(n_events, rank, size):
    """Global ids of the events rank ``rank`` of ``size`` runs, in order."""
    if not 0 <= rank < size:
        raise ValueError("rank must be in [0, size)")
    ids = np.arange(n_events, dtype=np.int64)
    return ids[select_rank_for_src(ids, size) == rank]


def shard_events(ev, rank, size):
    """This rank's share of an event set.

    ``ev`` holds evlo, evla, iper (per event), rec_ptr (CSR offsets), rec_idx,
    tt_obs, weight (per observation) and stlo, stla (the receiver table).
    Returns a dict of the same keys for the local events -- receiver lists
    re-based, the receiver table unchanged -- plus ``event_ids`` (global event
    ids) and ``obs_ids`` (global observation index of each local observation,
    for ``gather_syn``)."""
    ptr = np.asarray(ev["rec_ptr"], dtype=np.int64)
    n_events = ptr.size - 1
    if len(ev["evlo"]) != n_events:
        raise ValueError("rec_ptr must have one entry more than evlo")
    sel = local_event_ids(n_events, rank, size)
    counts = ptr[sel + 1] - ptr[sel]
    new_ptr = np.zeros(sel.size + 1, dtype=np.int32)
    np.cumsum(counts, out=new_ptr[1:])
    # global observation index of every local observation, event by event
    starts = np.repeat(ptr[sel] - new_ptr[:-1], counts)
    obs = starts + np.arange(int(new_ptr[-1]), dtype=np.int64)
    out = dict(evlo=np.asarray(ev["evlo"])[sel], evla=np.asarray(ev["evla"])[sel],
               iper=np.asarray(ev["iper"], dtype=np.int32)[sel], rec_ptr=new_ptr,
               rec_idx=np.asarray(ev["rec_idx"], dtype=np.int32)[obs],
               stlo=ev["stlo"], stla=ev["stla"], event_ids=sel, obs_ids=obs)
    for key in ("tt_obs", "weight"):
        if key in ev:
            out[key] = np.asarray(ev[key])[obs]
    return out


def _world(group):
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return None, 1
    return dist, dist.get_world_size(group)


def reduce_gradient(adj_s, chi, status=None, group=None):
    """Sum adj_s (nper, ny, nx) and chi (1,) over ranks in place
    (mpi.sum_all_all, src/preproc.cpp:146, :238); ``status`` (int32, may be
    None) takes the worst (largest) code of any rank.  No-op on one rank."""
    import torch
    dist, size = _world(group)
    if size == 1:
        return adj_s, chi
    if adj_s.dtype != torch.float64 or chi.dtype != torch.float64:
        raise TypeError("adj_s and chi are summed in float64")
    dist.all_reduce(adj_s, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(chi, op=dist.ReduceOp.SUM, group=group)
    if status is not None:
        dist.all_reduce(status, op=dist.ReduceOp.MAX, group=group)
    return adj_s, chi


def gather_syn(syn_local, obs_ids, n_obs, group=None):
    """SrcRec::gather_syn_tt (src/src_rec.cpp:326-371): every rank returns
    the (n_obs,) synthetic times of all observations; each observation
    belongs to exactly one rank, so the gather is a sum of zero-filled
    arrays."""
    import torch
    full = torch.zeros(n_obs, dtype=torch.float64, device=syn_local.device)
    idx = torch.as_tensor(np.asarray(obs_ids, dtype=np.int64), device=syn_local.device)
    full.index_copy_(0, idx, syn_local.to(torch.float64)[: idx.numel()])
    dist, size = _world(group)
    if size > 1:
        dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full
