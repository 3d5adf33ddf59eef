"""preproc:: call surface (reference include/preproc.h) on the GPU.

``forward_for_event`` is the drop-in for preproc::forward_for_event
(src/preproc.cpp:71-148): every (source, period) event runs forward, receiver
interpolation, residuals, adjoint, source mask and accumulation into adj_s.
``ForwardAdjointPlan`` keeps the event set, per-source geometry and scratch
resident on the device across misfit evaluations (one plan per inversion).
Device memory is held in torch tensors (allocation only; all arithmetic runs
in libsurfatt_gpu.so).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import SA_FP32, SA_FP64, default_context, ptr


def _prec(p):
    return {"fp64": SA_FP64, "fp32": SA_FP32, SA_FP64: SA_FP64, SA_FP32: SA_FP32}[p]


def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dtype=dt)


class ForwardAdjointPlan:
    """sa_plan: grid + event set fixed; call ``run`` once per misfit evaluation."""

    def __init__(self, xx_deg, yy_deg, nper, evlo, evla, iper, rec_ptr, rec_idx, stlo, stla,
                 precision="fp64", ctx=None, graph=True):
        self.ctx = ctx or default_context()
        self.precision = _prec(precision)
        self._keep = [_c(xx_deg), _c(yy_deg), _c(evlo), _c(evla), _c(iper, np.int32),
                      _c(rec_ptr, np.int32), _c(rec_idx, np.int32), _c(stlo), _c(stla)]
        xx, yy, elo, ela, ip, rp, ri, slo, sla = self._keep
        self.nx, self.ny, self.nper = xx.size, yy.size, int(nper)
        self.ne, self.nsta = elo.size, slo.size
        self.npair = int(rp[-1]) if rp.size else 0
        h = C.c_void_p()
        addr = (lambda a: a.ctypes.data if a.size else None)
        rc = _capi.lib().sa_plan_create(self.ctx.h, self.precision, self.nx, self.ny, self.nper,
                                        xx, yy, self.ne, addr(elo), addr(ela), addr(ip), addr(rp),
                                        addr(ri), self.nsta, addr(slo), addr(sla), C.byref(h))
        _capi.check(self.ctx.h, rc)
        self.h = h
        _capi.lib().sa_plan_set_graph(self.h, int(bool(graph)))

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().sa_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_adjoint(self, kind="reference"):
        """"reference": the reference's adjoint and forward stopping rule;
        "exact" (FP64 plans): forward solves to a fixed point and the exact
        discrete adjoint, adj_s = dchi/dsvel (sa_plan_set_adjoint)."""
        k = {"reference": 0, "exact": 1}[kind]
        _capi.check(self.ctx.h, _capi.lib().sa_plan_set_adjoint(self.h, k))
        self.adjoint = kind

    def set_deterministic(self, enable=True, max_bytes=0):
        """Sum adj_s and chi in event order (reproducible bit for bit; FP64:
        the reference's single-rank sums) instead of with atomics
        (sa_plan_set_deterministic)."""
        rc = _capi.lib().sa_plan_set_deterministic(self.h, int(bool(enable)), int(max_bytes))
        _capi.check(self.ctx.h, rc)

    def kernel_timing(self, enable=True):
        """Record CUDA events around the batch kernel (runs without the graph)."""
        _capi.check(self.ctx.h, _capi.lib().sa_plan_kernel_timing(self.h, int(bool(enable))))

    def kernel_ms(self):
        """Duration of the last batch kernel launch (waits for it)."""
        ms = C.c_float(0.0)
        _capi.check(self.ctx.h, _capi.lib().sa_plan_kernel_ms(self.h, C.byref(ms)))
        return ms.value

    def autotune(self, svel, tt_obs, weight, calc_adj=True, m11=None, m12=None, m22=None,
                 adj_s=None, stream=None):
        """Pick the fastest batch-kernel launch configuration on this plan's own
        workload (sa_plan_autotune); kept for this plan and later plans of the
        same grid size on its context.  Returns dict(ms=[per candidate],
        choice=index, variant, active_slots, nslots)."""
        ms = (C.c_float * 32)()
        n, ch = C.c_int(0), C.c_int(0)
        rc = _capi.lib().sa_plan_autotune(self.h, ptr(svel), ptr(m11), ptr(m12), ptr(m22),
                                          ptr(tt_obs), ptr(weight), int(bool(calc_adj)),
                                          ptr(adj_s), ms, C.byref(n), C.byref(ch), stream)
        _capi.check(self.ctx.h, rc)
        return dict(ms=list(ms)[:n.value], choice=ch.value, **self.tune())

    def set_tune(self, variant, active_slots=0):
        """Use a known launch configuration (sa_plan_set_tune)."""
        _capi.check(self.ctx.h, _capi.lib().sa_plan_set_tune(self.h, int(variant),
                                                             int(active_slots)))

    def tune(self):
        """Current launch configuration: variant, active_slots, nslots."""
        v, a, n = C.c_int(0), C.c_int(0), C.c_int(0)
        _capi.check(self.ctx.h, _capi.lib().sa_plan_get_tune(self.h, C.byref(v), C.byref(a),
                                                             C.byref(n)))
        return dict(variant=v.value, active_slots=a.value, nslots=n.value)

    def debug_fields(self, T_out=None, Ta_out=None):
        _capi.lib().sa_plan_debug_fields(self.h, ptr(T_out), ptr(Ta_out))

    def run(self, svel, tt_obs, weight, calc_adj=True, m11=None, m12=None, m22=None, out=None,
            stream=None):
        """Enqueue one evaluation on device tensors (float64, contiguous).

        svel: (nper, ny, nx); tt_obs/weight: (npair,).  ``out`` is a dict of
        preallocated device tensors (syn, adj_s, chi, fwd_iters, adj_iters,
        status); missing ones are allocated.  Returns ``out``; synchronise the
        stream before reading."""
        import torch
        dev = svel.device
        out = {} if out is None else out
        f64 = dict(dtype=torch.float64, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        out.setdefault("syn", torch.empty(max(self.npair, 1), **f64))
        out.setdefault("adj_s", torch.empty((self.nper, self.ny, self.nx), **f64))
        out.setdefault("chi", torch.zeros(1, **f64))
        out.setdefault("fwd_iters", torch.zeros(max(self.ne, 1), **i32))
        out.setdefault("adj_iters", torch.zeros(max(self.ne, 1), **i32))
        out.setdefault("status", torch.zeros(max(self.ne, 1), **i32))
        rc = _capi.lib().sa_plan_forward_adjoint(
            self.h, ptr(svel), ptr(m11), ptr(m12), ptr(m22), ptr(tt_obs), ptr(weight),
            int(bool(calc_adj)), ptr(out["syn"]), ptr(out["adj_s"]), ptr(out["chi"]),
            ptr(out["fwd_iters"]), ptr(out["adj_iters"]), ptr(out["status"]),
            stream if stream is not None else None)
        _capi.check(self.ctx.h, rc)
        return out


def forward_for_event(xx_deg, yy_deg, svel, events, calc_adj=True, m11=None, m12=None, m22=None,
                      precision="fp64", ctx=None):
    """Host-array drop-in for preproc::forward_for_event.

    svel (nper, ny, nx); ``events`` holds evlo, evla, iper, rec_ptr, rec_idx,
    stlo, stla, tt_obs, weight.  Returns dict(syn, adj_s, chi, fwd_iters,
    adj_iters).  Raises NoConvergence if an event hit the iteration cap."""
    ctx = ctx or default_context()
    svel = _c(svel)
    nper, ny, nx = svel.shape
    ev = events
    ne = len(ev["evlo"])
    npair = int(ev["rec_ptr"][-1])
    syn = np.zeros(max(npair, 1))
    adj_s = np.zeros((nper, ny, nx))
    chi = C.c_double(0.0)
    fi = np.zeros(max(ne, 1), np.int32)
    ai = np.zeros(max(ne, 1), np.int32)
    addr = (lambda a: None if a is None else _c(a).ctypes.data)
    keep = [_c(m) for m in (m11, m12, m22) if m is not None]
    mp = [k.ctypes.data for k in keep] if keep else [None, None, None]
    rc = _capi.lib().sa_forward_for_events(
        ctx.h, _prec(precision), nx, ny, nper, _c(xx_deg), _c(yy_deg), svel, mp[0], mp[1], mp[2],
        ne, _c(ev["evlo"]), _c(ev["evla"]), _c(ev["iper"], np.int32), _c(ev["rec_ptr"], np.int32),
        _c(ev["rec_idx"], np.int32), len(ev["stlo"]), _c(ev["stlo"]), _c(ev["stla"]),
        _c(ev["tt_obs"]), _c(ev["weight"]), int(bool(calc_adj)), syn, adj_s, C.byref(chi), fi, ai)
    _capi.check(ctx.h, rc)
    return dict(syn=syn[:npair], adj_s=adj_s, chi=chi.value, fwd_iters=fi[:ne],
                adj_iters=ai[:ne])


class MultiPlan:
    """One persistent launch over the events of several plans -- grid levels
    of different size (sa_multi): each queue entry names its plan, scratch
    slots hold the largest grid, and the queue is ordered by work across the
    plans.  ``run`` takes per-plan lists and returns per-plan output dicts
    (syn, adj_s, chi, status) equal to each plan's own ``run``."""

    def __init__(self, plans):
        self.plans = list(plans)
        self.ctx = self.plans[0].ctx
        n = len(self.plans)
        arr = (C.c_void_p * n)(*[p.h for p in self.plans])
        h = C.c_void_p()
        rc = _capi.lib().sa_multi_create(arr, n, C.byref(h))
        _capi.check(self.ctx.h, rc)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().sa_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, svel, tt_obs, weight, calc_adj=True, m11=None, m12=None, m22=None, outs=None,
            stream=None):
        import torch
        n = len(self.plans)
        outs = [{} for _ in range(n)] if outs is None else outs
        for p, o, sv in zip(self.plans, outs, svel):
            f64 = dict(dtype=torch.float64, device=sv.device)
            o.setdefault("syn", torch.empty(max(p.npair, 1), **f64))
            o.setdefault("adj_s", torch.empty((p.nper, p.ny, p.nx), **f64))
            o.setdefault("chi", torch.zeros(1, **f64))
            o.setdefault("status", torch.zeros(max(p.ne, 1), dtype=torch.int32, device=sv.device))
        arr = lambda xs: (C.c_void_p * n)(*[ptr(x) for x in xs])
        none = [None] * n
        rc = _capi.lib().sa_multi_forward_adjoint(
            self.h, arr(svel), arr(m11 or none), arr(m12 or none), arr(m22 or none), arr(tt_obs),
            arr(weight), int(bool(calc_adj)), arr([o["syn"] for o in outs]),
            arr([o["adj_s"] for o in outs]), arr([o["chi"] for o in outs]),
            arr([o["status"] for o in outs]), stream)
        _capi.check(self.ctx.h, rc)
        return outs

    def kernel_ms(self):
        """Device time of the last evaluation's batch launch."""
        ms = C.c_float(0.0)
        _capi.check(self.ctx.h, _capi.lib().sa_multi_kernel_ms(self.h, C.byref(ms)))
        return ms.value

    def worst_status(self):
        w = C.c_int(0)
        _capi.check(self.ctx.h, _capi.lib().sa_multi_status(self.h, C.byref(w)))
        return w.value
