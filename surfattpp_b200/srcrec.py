"""SrcRec (reference include/src_rec.h, src/src_rec.cpp): the observation
table read from CSV, its periods and its events, and the table written back
with observed or forward times.  Parsing and event building run in
libsurfatt_gpu.so (host code); ``events()`` returns the arrays that
``preproc.ForwardAdjointPlan`` takes, with each observation row as a
receiver.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi


class SrcRec:
    def __init__(self, csv_path: str):
        h = C.c_void_p()
        rc = _capi.lib().sa_srcrec_load(str(csv_path).encode(), C.byref(h))
        if rc != _capi.SA_OK:
            raise ValueError(f"SrcRec: cannot read observation table {csv_path}")
        self.h = h
        n, npr, ne = C.c_int(), C.c_int(), C.c_int()
        _capi.lib().sa_srcrec_sizes(h, C.byref(n), C.byref(npr), C.byref(ne))
        self.n_obs, self.nperiod, self.n_events = n.value, npr.value, ne.value
        L = _capi.lib()
        p = lambda a: a.ctypes.data
        self.periods, self.meanvel = np.zeros(self.nperiod), np.zeros(self.nperiod)
        self.n_obs_per_period = np.zeros(self.nperiod, np.int32)
        L.sa_srcrec_periods(h, p(self.periods), p(self.meanvel), p(self.n_obs_per_period))
        o = {k: np.zeros(self.n_obs) for k in ("stlo", "stla", "tt", "weight", "dist", "vel",
                                                "period")}
        L.sa_srcrec_observations(h, *(p(o[k]) for k in ("stlo", "stla", "tt", "weight", "dist",
                                                        "vel", "period")))
        self.obs = o
        self.evlo, self.evla = np.zeros(self.n_events), np.zeros(self.n_events)
        self.iper = np.zeros(self.n_events, np.int32)
        self.rec_ptr = np.zeros(self.n_events + 1, np.int32)
        L.sa_srcrec_events(h, p(self.evlo), p(self.evla), p(self.iper), p(self.rec_ptr), None)
        self.rec_idx = np.zeros(max(int(self.rec_ptr[-1]), 1), np.int32)
        L.sa_srcrec_events(h, None, None, None, None, p(self.rec_idx))
        self.rec_idx = self.rec_idx[:int(self.rec_ptr[-1])]
        self.event_names = [L.sa_srcrec_event_name(h, e).decode() for e in range(self.n_events)]

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().sa_srcrec_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def events(self):
        """Event arrays for ForwardAdjointPlan / forward_for_event."""
        return dict(evlo=self.evlo, evla=self.evla, iper=self.iper, rec_ptr=self.rec_ptr,
                    rec_idx=self.rec_idx, stlo=self.obs["stlo"], stla=self.obs["stla"],
                    tt_obs=self.obs["tt"][self.rec_idx], weight=self.obs["weight"][self.rec_idx])

    def tt_fwd(self, syn):
        """SrcRec::gather_syn_tt: per-pair synthetic times -> per-row table."""
        t = np.zeros(self.n_obs)
        t[self.rec_idx] = np.asarray(syn)[:self.rec_idx.size]
        return t

    def write(self, csv_path: str, tt_fwd=None):
        t = None if tt_fwd is None else np.ascontiguousarray(tt_fwd, dtype=np.float64)
        rc = _capi.lib().sa_srcrec_write(self.h, str(csv_path).encode(),
                                         None if t is None else t.ctypes.data)
        if rc != _capi.SA_OK:
            raise ValueError(f"SrcRec: cannot write {csv_path}")
