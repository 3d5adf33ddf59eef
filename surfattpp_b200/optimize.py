"""optimize:: and the model update (reference include/optimize.h,
src/optimize.cpp, src/inversion.cpp:302-323, :465-490) on the GPU, for the
vs-only parametrisation.  Fields are float64 CUDA tensors of n values; the
history of iterates that the reference keeps in HDF5 stays on the device.
"""
from __future__ import annotations

import ctypes as C

from . import _capi
from ._capi import default_context, ptr

ACCEPT, TRY, FAIL = 0, 1, 2
MAX_LBFGS_STORE = 5


class LBFGS:
    """Device history of (model vs, gradient) iterates (sa_lbfgs)."""

    def __init__(self, n: int, ctx=None):
        self.ctx = ctx or default_context()
        self.n = int(n)
        h = C.c_void_p()
        _capi.check(self.ctx.h, _capi.lib().sa_lbfgs_create(self.ctx.h, self.n, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().sa_lbfgs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def store(self, it: int, model, grad):
        """Inversion::store_model + store_gradient for iteration ``it``."""
        _capi.check(self.ctx.h, _capi.lib().sa_lbfgs_store(self.h, int(it), ptr(model), ptr(grad)))

    def direction(self, it: int, out=None):
        """optimize::lbfgs_direction(it): H_k g_k (the reference's search_dir)."""
        import torch
        if out is None:
            out = torch.empty(self.n, dtype=torch.float64, device="cuda")
        _capi.check(self.ctx.h, _capi.lib().sa_lbfgs_direction(self.h, int(it), ptr(out)))
        return out


def dot(a, b, ctx=None) -> float:
    ctx = ctx or default_context()
    r = C.c_double()
    _capi.check(ctx.h, _capi.lib().sa_dot(ctx.h, a.numel(), ptr(a), ptr(b), C.byref(r)))
    return r.value


def grad_normalization(g, ctx=None) -> float:
    """In place g /= max|g| (skipped below DBL_EPSILON); returns max|g|."""
    ctx = ctx or default_context()
    m = C.c_double()
    _capi.check(ctx.h, _capi.lib().sa_grad_normalization(ctx.h, g.numel(), ptr(g), C.byref(m)))
    return m.value


def calc_descent_angle(direction, gradient, ctx=None) -> float:
    ctx = ctx or default_context()
    r = C.c_double()
    _capi.check(ctx.h, _capi.lib().sa_descent_angle(ctx.h, direction.numel(), ptr(direction),
                                                    ptr(gradient), C.byref(r)))
    return r.value


def wolfe_condition(gd, kd, alpha, alpha_L, alpha_R, f0, f1, subiter, c1=0.1, c2=0.9,
                    max_sub_niter=10, alpha_init=0.02):
    """optimize::wolfe_condition from gd = grad.dir and kd = ker_next.dir.
    Returns (status, next_alpha, alpha_L, alpha_R)."""
    aL, aR, nxt = C.c_double(alpha_L), C.c_double(alpha_R), C.c_double()
    st = _capi.lib().sa_wolfe_condition(gd, kd, alpha, C.byref(aL), C.byref(aR), f0, f1,
                                        int(subiter), c1, c2, int(max_sub_niter), alpha_init,
                                        C.byref(nxt))
    return st, nxt.value, aL.value, aR.value


def model_update_vs(vs, direction, alpha, vs_out=None, vp_out=None, rho_out=None, ctx=None):
    """vs_out = vs*(1 - alpha*dir); vp = vs2vp(vs_out); rho = vp2rho(vp)."""
    import torch
    ctx = ctx or default_context()
    vs_out = torch.empty_like(vs) if vs_out is None else vs_out
    vp_out = torch.empty_like(vs) if vp_out is None else vp_out
    rho_out = torch.empty_like(vs) if rho_out is None else rho_out
    _capi.check(ctx.h, _capi.lib().sa_model_update_vs(ctx.h, vs.numel(), ptr(vs), ptr(direction),
                                                      alpha, ptr(vs_out), ptr(vp_out),
                                                      ptr(rho_out), None))
    return vs_out, vp_out, rho_out
