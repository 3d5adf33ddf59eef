"""eikonal:: call surface (reference include/eikonal_solver.h:32-89) on the GPU.

Same names, argument meaning and error behaviour as the reference:
fields are (nx x ny) column-major, i.e. numpy arrays shaped (ny, nx); a grid
smaller than 3x3 raises ValueError (std::invalid_argument in the reference);
non-convergence is reported as a warning on stderr, as the reference does.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import _capi
from ._capi import SA_FP32, SA_FP64, default_context


def _prec(precision):
    return {"fp64": SA_FP64, "fp32": SA_FP32, SA_FP64: SA_FP64, SA_FP32: SA_FP32}[precision]


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def FSM_UW_PS_lonlat_2d(xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg, y0_deg,
                        precision="fp64", return_iters=False, ctx=None):
    """Factored anisotropic eikonal travel-time field (src/eikonal_solver.cpp:22-318)."""
    ctx = ctx or default_context()
    xx, yy = _c(xx_deg), _c(yy_deg)
    nx, ny = xx.size, yy.size
    if nx < 3 or ny < 3:
        raise ValueError("Grid must be at least 3x3")
    T = np.zeros((ny, nx))
    it = C.c_int(0)
    rc = _capi.lib().sa_eik_fwd_field(ctx.h, _prec(precision), nx, ny, xx, yy, _c(spha),
                                      _c(sphb), _c(sphc), _c(fun), float(x0_deg), float(y0_deg),
                                      T, C.byref(it))
    if rc == _capi.SA_ERR_NOCONV:
        print(f"[eikonal] WARNING: FSM did not converge after 2000 iterations. "
              f"src=({x0_deg:.4f},{y0_deg:.4f})", file=sys.stderr)
    elif rc != _capi.SA_OK:
        _capi.check(ctx.h, rc)
    return (T, it.value) if return_iters else T


def FSM_O1_JSE_lonlat_2d(xx_deg, yy_deg, spha, sphb, sphc, T, xrec_deg, yrec_deg, sourceAdj,
                         precision="fp64", return_iters=False, ctx=None):
    """Adjoint field (src/eikonal_solver.cpp:323-511); zero on the boundary."""
    ctx = ctx or default_context()
    xx, yy = _c(xx_deg), _c(yy_deg)
    nx, ny = xx.size, yy.size
    if nx < 3 or ny < 3:
        raise ValueError("Grid must be at least 3x3")
    xr, yr, sa = _c(xrec_deg).ravel(), _c(yrec_deg).ravel(), _c(sourceAdj).ravel()
    Ta = np.zeros((ny, nx))
    it = C.c_int(0)
    p = (lambda a: a.ctypes.data if a.size else None)
    rc = _capi.lib().sa_eik_adj_field(ctx.h, _prec(precision), nx, ny, xx, yy, _c(spha),
                                      _c(sphb), _c(sphc), _c(T), xr.size, p(xr), p(yr), p(sa),
                                      Ta, C.byref(it))
    if rc not in (_capi.SA_OK, _capi.SA_ERR_NOCONV):
        _capi.check(ctx.h, rc)
    return (Ta, it.value) if return_iters else Ta


def mask_uniform_grid(xx, yy, tableAdj, x0, y0):
    """Zero the adjoint field within 1.5 cells of the source, in place
    (src/eikonal_solver.cpp:514-536)."""
    if tableAdj.dtype != np.float64 or not tableAdj.flags.c_contiguous:
        raise TypeError("tableAdj must be a C-contiguous float64 array")
    xx, yy = _c(xx), _c(yy)
    rc = _capi.lib().sa_mask_uniform_grid(xx.size, yy.size, xx, yy, tableAdj, float(x0), float(y0))
    _capi.check(None, rc)
    return tableAdj
