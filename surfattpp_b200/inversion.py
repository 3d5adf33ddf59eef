"""Inversion::run_forward_adjoint (reference src/inversion.cpp:245-296) on the GPU.

``MisfitGradient`` binds a ``ForwardAdjointPlan`` (grid, events, precision)
to a depth grid and the periods, and evaluates one misfit and its vs gradient
per call for Rayleigh phase-velocity data with the vs-only parametrisation:

    fwdsurf -> forward_for_event (all events, adjoint on) -> combine_kernels
               `-> compute_dispersion_kernel (second stream, overlapped)

Kernel preconditioning and smoothing (src/postproc.cpp) are not applied; the
result is ``sg.ker_loc[0]`` right after ``preproc::combine_kernels``.

``TravelTimeMisfit`` exposes the same evaluation as a torch.autograd.Function
of vs3d: forward returns chi, backward returns ``grad_out * ker_vs`` -- the
reference's adjoint gradient, which is the continuous adjoint of the eikonal
(not the exact derivative of the discretised chi).  Device memory is held in
torch tensors; all arithmetic runs in libsurfatt_gpu.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import ptr
from .preproc import ForwardAdjointPlan, _c


class MisfitGradient:
    """One misfit-gradient evaluation per ``run`` (sa_grad)."""

    def __init__(self, plan: ForwardAdjointPlan, zgrid, periods):
        self.plan = plan
        self.zgrid = _c(zgrid)
        self.periods = _c(periods)
        if self.periods.size != plan.nper:
            raise ValueError("periods must have the plan's nper entries")
        self.nz = self.zgrid.size
        h = C.c_void_p()
        rc = _capi.lib().sa_grad_create(plan.h, self.nz, self.zgrid, self.periods, C.byref(h))
        _capi.check(plan.ctx.h, rc)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().sa_grad_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, vs3d, tt_obs, weight, vp3d=None, out=None, stream=None):
        """Enqueue one evaluation on device tensors (float64, contiguous).

        vs3d (nx, ny, nz); vp3d (nx, ny, nz) or None for vs2vp(vs3d).
        Returns dict(ker_vs (nx, ny, nz), chi (1,), svel, adj_s
        (nper, ny, nx), status (1,)); synchronise before reading."""
        import torch
        dev = vs3d.device
        p = self.plan
        out = {} if out is None else out
        f64 = dict(dtype=torch.float64, device=dev)
        out.setdefault("ker_vs", torch.empty((p.nx, p.ny, self.nz), **f64))
        out.setdefault("chi", torch.zeros(1, **f64))
        out.setdefault("svel", torch.empty((p.nper, p.ny, p.nx), **f64))
        out.setdefault("adj_s", torch.empty((p.nper, p.ny, p.nx), **f64))
        out.setdefault("status", torch.zeros(1, dtype=torch.int32, device=dev))
        rc = _capi.lib().sa_grad_run(self.h, ptr(vs3d), ptr(vp3d), ptr(tt_obs), ptr(weight),
                                     ptr(out["ker_vs"]), ptr(out["chi"]), ptr(out["svel"]),
                                     ptr(out["adj_s"]), ptr(out["status"]), stream)
        _capi.check(p.ctx.h, rc)
        return out

    def sen(self, stream=None):
        """(sen_vs, sen_vp, sen_rho) of the last run as device tensors
        (nx, ny, nz, nper)."""
        import torch
        p = self.plan
        dev = torch.device("cuda", torch.cuda.current_device())
        res = [torch.empty((p.nx, p.ny, self.nz, p.nper), dtype=torch.float64, device=dev)
               for _ in range(3)]
        rc = _capi.lib().sa_grad_sen(self.h, *[ptr(t) for t in res], stream)
        _capi.check(p.ctx.h, rc)
        return tuple(res)


class TravelTimeMisfit:
    """chi(vs3d) with the reference's adjoint gradient as a torch.autograd.Function."""

    @staticmethod
    def apply(grad: MisfitGradient, vs3d, tt_obs, weight):
        return _fn().apply(vs3d, grad, tt_obs, weight)


_FN = None


def _fn():
    global _FN
    if _FN is not None:
        return _FN
    import torch

    class _Misfit(torch.autograd.Function):
        @staticmethod
        def forward(ctx, vs3d, grad, tt_obs, weight):
            vs = vs3d.detach().contiguous()
            out = grad.run(vs, tt_obs, weight)
            ctx.save_for_backward(out["ker_vs"])
            return out["chi"][0].clone()

        @staticmethod
        def backward(ctx, g):
            (ker,) = ctx.saved_tensors
            return g * ker, None, None, None

    _FN = _Misfit
    return _FN
