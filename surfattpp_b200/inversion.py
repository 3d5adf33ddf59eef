"""Inversion::run_forward_adjoint (reference src/inversion.cpp:245-296) on the GPU.

``MisfitGradient`` binds a ``ForwardAdjointPlan`` (grid, events, precision)
to a depth grid and the periods, and evaluates one misfit and its vs gradient
per call for Rayleigh phase-velocity data with the vs-only parametrisation:

    fwdsurf -> forward_for_event (all events, adjoint on) -> combine_kernels
               `-> compute_dispersion_kernel (second stream, overlapped)

Kernel preconditioning and smoothing (src/postproc.cpp) are not applied; the
result is ``sg.ker_loc[0]`` right after ``preproc::combine_kernels``.

``TravelTimes`` is the torch.autograd.Function vs3d -> receiver travel times
T_rec: its forward runs fwdsurf and every event's forward solve and stores no
field; its backward, for an upstream gradient g on T_rec, recomputes the
phase velocities and every forward field, drives the adjoint with g in place
of the residuals w (Tsyn - Tobs) (the reference's adjoint applied to g), and
combines the depth kernels.  ``misfit`` builds chi = 0.5 sum w (T - Tobs)^2
in torch on top of it; with ``convention="reference"`` its gradient is the
reference's ker_vs.  ``TravelTimeMisfit`` is the fused form (one pass: forward,
residuals and adjoint per event) with the same gradient.

Conventions of the vs gradient:
  * "reference": preproc::combine_kernels -- a kernel per unit area built
    from sregn96's dimensionless depth kernels;
  * "derivative": the derivative with respect to the vs nodes (cell-area
    Jacobian, plain dc/dvs, corrected density kernel, half-space at the
    deepest node).  Its eikonal part is still the reference's continuous
    adjoint, which differs from the derivative of the discretised travel
    times by the discretisation error (about 10 % on the checkerboard case);
  * "exact" (the plan's adjoint set to "exact", FP64): the gradient of the
    discrete forward model itself -- forward solves to a fixed point, the
    exact discrete adjoint of the factored fast-sweeping solve, and dc/dvs by
    implicit differentiation of surfdisp96's secular function; it matches
    central differences of chi (2.4e-4 on the checkerboard case).
Device memory is held in torch tensors; all arithmetic runs in
libsurfatt_gpu.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import ptr
from .preproc import ForwardAdjointPlan, _c


class MisfitGradient:
    """One misfit-gradient evaluation per ``run`` (sa_grad)."""

    def __init__(self, plan: ForwardAdjointPlan, zgrid, periods, data_type="ph",
                 wave="rayleigh"):
        """data_type "ph" (phase velocities) or "gr" (group); wave "rayleigh"
        or "love" (Love kernels exist for group data only, as in the
        reference)."""
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
        self.data_type = data_type
        igr = {"ph": 0, "gr": 1}[data_type]
        if igr:
            _capi.check(plan.ctx.h, _capi.lib().sa_grad_set_data_type(self.h, igr))
        self.wave = wave
        iwave = {"rayleigh": 2, "love": 1}[wave]
        if iwave != 2:
            _capi.check(plan.ctx.h, _capi.lib().sa_grad_set_wave_type(self.h, iwave))

    def set_kden(self, enable=True):
        """is_kden: every run also returns ker_den, the kernel density
        (sa_grad_set_kden / sa_grad_ker_den)."""
        _capi.check(self.plan.ctx.h, _capi.lib().sa_grad_set_kden(self.h, int(bool(enable))))
        self.kden = bool(enable)

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().sa_grad_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, vs3d, tt_obs, weight, vp3d=None, out=None, stream=None, group=None):
        """Enqueue one evaluation on device tensors (float64, contiguous).

        vs3d (nx, ny, nz); vp3d (nx, ny, nz) or None for vs2vp(vs3d).
        Returns dict(ker_vs (nx, ny, nz), chi (1,), svel, adj_s
        (nper, ny, nx), status (1,)); synchronise before reading.

        Under torch.distributed with more than one rank, the plan holds this
        rank's events (``distributed.shard_events``): adj_s and chi are summed
        over ``group`` and ker_vs is combined from the sums, as
        src/preproc.cpp:146, :225-304 do after the local events.  The work
        then runs on torch's current stream (``stream`` must be None)."""
        from . import distributed
        multi = distributed._world(group)[1] > 1
        if multi and stream is not None:
            raise ValueError("a multi-rank run uses torch's current stream")
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
        if multi:
            stream = torch.cuda.current_stream(dev).cuda_stream
        rc = _capi.lib().sa_grad_run(self.h, ptr(vs3d), ptr(vp3d), ptr(tt_obs), ptr(weight),
                                     ptr(out["ker_vs"]), ptr(out["chi"]), ptr(out["svel"]),
                                     ptr(out["adj_s"]), ptr(out["status"]), stream)
        _capi.check(p.ctx.h, rc)
        if multi:
            distributed.reduce_gradient(out["adj_s"], out["chi"], out["status"], group)
            self.combine(vs3d, out["adj_s"], vp3d, out["ker_vs"], stream)
        if getattr(self, "kden", False):
            if multi:
                raise NotImplementedError("kernel density with more than one rank")
            out.setdefault("ker_den", torch.empty((p.nx, p.ny, self.nz), **f64))
            rc = _capi.lib().sa_grad_ker_den(self.h, ptr(vs3d), ptr(vp3d), ptr(out["ker_den"]),
                                             stream)
            _capi.check(p.ctx.h, rc)
        return out

    def combine(self, vs3d, adj_s, vp3d=None, ker_vs=None, stream=None):
        """combine_kernels of the last run's depth kernels with ``adj_s``
        (nper, ny, nx) -- e.g. the rank sum -- into ker_vs (nx, ny, nz)
        (sa_grad_combine)."""
        import torch
        p = self.plan
        if ker_vs is None:
            ker_vs = torch.empty((p.nx, p.ny, self.nz), dtype=torch.float64, device=vs3d.device)
        rc = _capi.lib().sa_grad_combine(self.h, ptr(vs3d), ptr(vp3d), ptr(adj_s), ptr(ker_vs),
                                         stream)
        _capi.check(p.ctx.h, rc)
        return ker_vs

    def forward_times(self, vs3d, syn=None, svel=None, stream=None):
        """Receiver travel times T_rec [npair] of vs3d (sa_grad_forward), on
        torch's current stream unless `stream` is given."""
        import torch
        p = self.plan
        dev = vs3d.device
        if stream is None:
            stream = torch.cuda.current_stream(dev).cuda_stream
        if syn is None:
            syn = torch.empty(max(p.npair, 1), dtype=torch.float64, device=dev)
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        rc = _capi.lib().sa_grad_forward(self.h, ptr(vs3d), ptr(syn), ptr(svel), ptr(st), stream)
        _capi.check(p.ctx.h, rc)
        self.last_status = st
        return syn[:p.npair]

    def vjp(self, vs3d, source_adj, convention="reference", vp3d=None, grad=None,
            adj_s=None, stream=None):
        """The vs gradient of sum(source_adj * T_rec) (sa_grad_vjp), on
        torch's current stream unless `stream` is given; see the module
        docstring for the conventions."""
        import torch
        p = self.plan
        if stream is None:
            stream = torch.cuda.current_stream(vs3d.device).cuda_stream
        conv = {"reference": 0, "derivative": 1, "exact": 2}[convention]
        if grad is None:
            grad = torch.empty((p.nx, p.ny, self.nz), dtype=torch.float64, device=vs3d.device)
        st = torch.zeros(1, dtype=torch.int32, device=vs3d.device)
        rc = _capi.lib().sa_grad_vjp(self.h, ptr(vs3d), ptr(vp3d), ptr(source_adj), conv,
                                     ptr(grad), None, ptr(adj_s), ptr(st), stream)
        _capi.check(p.ctx.h, rc)
        self.last_status = st
        return grad

    def dcdvs(self, vs3d, stream=None):
        """dc/dvs (nx, ny, nz, nper) of the Rayleigh phase velocities of vs3d
        from the derivatives of surfdisp96's roots (sa_grad_root_derivatives)."""
        import torch
        p = self.plan
        if stream is None:
            stream = torch.cuda.current_stream(vs3d.device).cuda_stream
        out = torch.empty((p.nx, p.ny, self.nz, p.nper), dtype=torch.float64, device=vs3d.device)
        rc = _capi.lib().sa_grad_root_derivatives(self.h, ptr(vs3d), ptr(out), stream)
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


class TravelTimes:
    """T_rec(vs3d) as a torch.autograd.Function (receiver times [npair])."""

    @staticmethod
    def apply(grad: MisfitGradient, vs3d, convention="reference"):
        return _tt_fn().apply(vs3d, grad, convention)


def misfit(grad: MisfitGradient, vs3d, tt_obs, weight, convention="reference"):
    """chi = 0.5 sum w (T_rec - Tobs)^2 (src/preproc.cpp:142) in torch on top
    of TravelTimes; its backward hands w (T - Tobs) to the adjoint, exactly
    the reference's adjoint source (src/preproc.cpp:111-115)."""
    T = TravelTimes.apply(grad, vs3d, convention)
    r = T - tt_obs
    return 0.5 * (weight * (r * r)).sum()


_TT_FN = None


def _tt_fn():
    global _TT_FN
    if _TT_FN is not None:
        return _TT_FN
    import torch

    class _TravelTimes(torch.autograd.Function):
        @staticmethod
        def forward(ctx, vs3d, grad, convention):
            vs = vs3d.detach().contiguous()
            T = grad.forward_times(vs).clone()
            ctx.grad = grad
            ctx.convention = convention
            ctx.save_for_backward(vs)     # the model only: no forward field is kept
            return T

        @staticmethod
        def backward(ctx, g):
            (vs,) = ctx.saved_tensors
            g = g.detach().to(torch.float64).contiguous()
            return ctx.grad.vjp(vs, g, ctx.convention), None, None

    _TT_FN = _TravelTimes
    return _TT_FN


class TravelTimeMisfit:
    """chi(vs3d) with the reference's adjoint gradient as a torch.autograd.Function
    (fused: one forward-residual-adjoint pass per event)."""

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
            grad.last = out      # status / svel / adj_s of this evaluation
            ctx.save_for_backward(out["ker_vs"])
            return out["chi"][0].clone()

        @staticmethod
        def backward(ctx, g):
            (ker,) = ctx.saved_tensors
            return g * ker, None, None, None

    _FN = _Misfit
    return _FN


class Inversion:
    """Inversion::run_inversion (reference src/inversion.cpp:106-160) for
    Rayleigh phase and/or group data, vs-only parametrisation, on the device.

    Per iteration: the forward/adjoint gradient (``MisfitGradient``), kernel
    smoothing (PostProc::pde_smooth, smooth_method 0) giving
    gradient = smooth(K) * w / chi, then either steepest descent
    (src/inversion.cpp:375-394) or L-BFGS with the strong-Wolfe line search
    and restarts (src/inversion.cpp:396-463, src/optimize.cpp), and the
    multiplicative model update vs *= (1 - alpha*dir) with Brocher vp, rho.
    The model and gradient history the reference writes to HDF5 stays on the
    device (optimize.LBFGS).  Kernel-density preconditioning (is_kden) is
    applied when asked for.
    """

    BREAK_ITER = 5          # include/config.h:94
    MAX_DESC_ANGLE = 92.0   # include/config.h:95

    def __init__(self, grad: MisfitGradient, tt_obs, weight, smooth=None, niter=10,
                 optim="lbfgs", step_length=0.02, max_sub_niter=10, c1=0.1, c2=0.9,
                 maxshrink=0.8, min_derr=0.0, data_weight=1.0, autograd=False,
                 more_data=None, kden=False):
        """smooth = dict(ygrid, zgrid, dx, dy, dz, sigma_h, sigma_v) or None.
        more_data: further data types as (MisfitGradient, tt_obs, weight,
        data_weight) tuples, e.g. group-velocity data next to phase data; the
        misfit, kernel and gradient are summed over the types as
        src/inversion.cpp:250-296 does.
        kden: kernel-density preconditioning of every type's kernel before
        the smoothing (postproc::kernel_precondition, src/postproc.cpp:
        487-517; the reference's is_kden).
        autograd: take the kernel as a torch.autograd gradient.  True: chi
        built in torch on TravelTimes (forward: receiver times, nothing
        stored; backward: every forward field recomputed, the adjoint driven
        by w (T - Tobs)) -- the reference's kernel, one extra forward pass.
        "fused": chi from TravelTimeMisfit, whose forward is the one fused
        forward-residual-adjoint pass of the reference and whose backward
        scales the stored kernel -- the same kernel at the cost of the
        plain evaluation."""
        self.g = grad
        self.tt, self.wt = tt_obs, weight
        self.smooth = smooth
        self.niter, self.optim = int(niter), optim
        self.step_length, self.max_sub_niter = step_length, int(max_sub_niter)
        self.c1, self.c2, self.maxshrink, self.min_derr = c1, c2, maxshrink, min_derr
        self.w = data_weight
        self.data = [(grad, tt_obs, weight, data_weight)] + list(more_data or [])
        self._outs = [None] * len(self.data)
        if autograd not in (False, True, "fused"):
            raise ValueError("autograd must be False, True or 'fused'")
        self.autograd = autograd
        self.kden = bool(kden)
        if self.kden:
            if self.autograd:
                raise ValueError("kden preconditioning runs on the fused evaluation")
            for g, *_ in self.data:
                g.set_kden(True)
        self.misfit, self.alphas, self.sub_iters, self.restarts = [], [], [], 0
        self._out = None

    def run_forward_adjoint(self, vs):
        """Inversion::run_forward_adjoint(true) (src/inversion.cpp:245-296):
        for every data type, misfit_total += chi w, ker_curr += K w and
        gradient += smooth(K) w / chi; returns (misfit_total, ker_curr,
        gradient)."""
        import torch
        from . import postproc
        total, ker_curr, grad = 0.0, None, None
        for i, (g, tt, wt, dw) in enumerate(self.data):
            if self.autograd == "fused":
                v = vs.detach().clone().requires_grad_(True)
                c = TravelTimeMisfit.apply(g, v, tt, wt)
                c.backward()
                out = g.last
                ker = v.grad
            elif self.autograd:
                v = vs.detach().clone().requires_grad_(True)
                c = misfit(g, v, tt, wt)
                c.backward()
                out = {"status": g.last_status, "chi": c.detach().reshape(1)}
                ker = v.grad
            else:
                out = g.run(vs, tt, wt, out=self._outs[i])
                self._outs[i] = out
                ker = out["ker_vs"]
            torch.cuda.synchronize()
            if int(out["status"][0]) != 0:
                raise _capi.SAError(int(out["status"][0]), "forward/adjoint evaluation failed")
            chi = float(out["chi"][0])
            sm = ker.clone()
            if self.kden:
                postproc.kernel_precondition(out["ker_den"], sm)
            if self.smooth is not None:
                s = self.smooth
                postproc.pde_smooth(sm, s["ygrid"], s["zgrid"], s["dx"], s["dy"], s["dz"],
                                    s["sigma_h"], s["sigma_v"])
            total += chi * dw
            ker_curr = ker * dw if ker_curr is None else ker_curr + ker * dw
            grad = sm * dw / chi if grad is None else grad + sm * dw / chi
        return total, ker_curr, grad

    def _check_convergence(self, it):
        """src/inversion.cpp:212-243."""
        B = self.BREAK_ITER
        if it <= B:
            return False
        prev = sum(self.misfit[it - 1 - i] for i in range(B + 1)) / B
        curr = sum(self.misfit[it - i] for i in range(B + 1)) / B
        red = 100 * (prev - curr) / prev
        return red < 0 or red < self.min_derr

    MAX_RESTARTS = 8   # a guard: the reference restarts without bound

    def run(self, vs0):
        """Returns the final model (same shape as vs0)."""
        from . import optimize as O
        vs = vs0.detach().clone().contiguous()
        n = vs.numel()
        lb = O.LBFGS(n) if self.optim == "lbfgs" else None
        iter_start = 0
        alpha = self.step_length
        for it in range(self.niter):
            model_it = vs.clone()
            f0, self._ker, self._grad = self.run_forward_adjoint(vs)
            self.misfit.append(f0)
            if lb is not None:
                lb.store(it, model_it.view(-1), self._grad.view(-1))
            if self.optim == "sd":
                d = self._grad.clone().view(-1)
                O.grad_normalization(d)
                if it > 0 and self.misfit[it] >= self.misfit[it - 1]:
                    alpha *= self.maxshrink
                vs, _, _ = O.model_update_vs(vs.view(-1), d, alpha)
                vs = vs.view_as(vs0)
                self.alphas.append(alpha)
            else:
                nrs = 0
                while True:
                    restart, vs_new, a, nsub = self._line_search(lb, it, iter_start, model_it, f0)
                    if not restart or nrs >= self.MAX_RESTARTS:
                        break
                    iter_start = it
                    nrs += 1
                    self.restarts += 1
                vs = vs_new
                self.alphas.append(a)
                self.sub_iters.append(nsub)
            if self._check_convergence(it):
                break
        return vs

    def _line_search(self, lb, it, iter_start, model, f0):
        """Inversion::line_search (src/inversion.cpp:396-463).  As in the
        reference, each trial replaces the current kernel and gradient
        (gradient_, ker_curr_), which a restart then starts from."""
        from . import optimize as O
        if it == iter_start:
            d = self._grad.clone().view(-1)
        else:
            d = lb.direction(it)
        O.grad_normalization(d)
        if it > iter_start:
            if O.calc_descent_angle(d, self._grad.view(-1)) > self.MAX_DESC_ANGLE:
                return True, model, 0.0, 0
        ker_prev = self._ker
        gd = O.dot(ker_prev.view(-1), d)
        alpha, aL, aR = self.step_length, 0.0, 0.0
        trial = model
        for sub in range(self.max_sub_niter):
            trial, _, _ = O.model_update_vs(model.view(-1), d, alpha)
            trial = trial.view_as(model)
            f1, self._ker, self._grad = self.run_forward_adjoint(trial)
            kd = O.dot(self._ker.view(-1), d)
            st, nxt, aL, aR = O.wolfe_condition(gd, kd, alpha, aL, aR, f0, f1, sub, self.c1,
                                                self.c2, self.max_sub_niter, self.step_length)
            if st == O.ACCEPT:
                return False, trial, alpha, sub + 1
            if st == O.TRY:
                alpha = nxt
                continue
            return True, trial, alpha, sub + 1
        return True, trial, alpha, self.max_sub_niter
