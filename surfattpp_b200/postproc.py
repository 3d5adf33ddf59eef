"""postproc:: call surface (reference include/postproc.h) on the GPU.

``pde_smooth`` is PostProc::pde_smooth (src/postproc.cpp:388-463) on one
rank: nstep explicit Euler steps of the spherical 7-point Laplacian with
Neumann boundary copies, over a (nx, ny, nz) row-major field (depth fastest,
as Tensor3r).  ``kernel_smooth`` applies it to each kernel of a list
(postproc::kernel_smooth, :519-534); ``kernel_precondition`` the kernel-density
preconditioning (:487-517).  Device memory is held in torch tensors;
the arithmetic runs in libsurfatt_gpu.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import default_context, ptr


def pde_smooth_nstep(ygrid, dx_deg, dy_deg, dz_km, sigma_h, sigma_v):
    """(nstep, ch, cv) of src/postproc.cpp:394-434; ValueError for invalid sigma."""
    y = np.ascontiguousarray(ygrid, dtype=np.float64)
    n, ch, cv = C.c_int(), C.c_double(), C.c_double()
    rc = _capi.lib().sa_pde_smooth_nstep(y.size, dx_deg, dy_deg, dz_km, y, sigma_h, sigma_v,
                                         C.byref(n), C.byref(ch), C.byref(cv))
    if rc != _capi.SA_OK:
        raise ValueError("Invalid sigma values or grid spacing for PDE-based smoothing")
    return n.value, ch.value, cv.value


def pde_smooth(field, ygrid, zgrid, dx_deg, dy_deg, dz_km, sigma_h, sigma_v, work=None,
               ctx=None, stream=None):
    """Smooth a float64 CUDA tensor (nx, ny, nz) in place; returns (field, nstep)."""
    ctx = ctx or default_context()
    nx, ny, nz = field.shape
    y = np.ascontiguousarray(ygrid, dtype=np.float64)
    z = np.ascontiguousarray(zgrid, dtype=np.float64)
    if y.size != ny or z.size != nz:
        raise ValueError("ygrid/zgrid must match the field's ny/nz")
    ns = C.c_int(0)
    rc = _capi.lib().sa_pde_smooth(ctx.h, nx, ny, nz, dx_deg, dy_deg, dz_km, y, z, sigma_h,
                                   sigma_v, ptr(field), ptr(work), C.byref(ns), stream)
    _capi.check(ctx.h, rc)
    return field, ns.value


def kernel_smooth(kernels, ygrid, zgrid, dx_deg, dy_deg, dz_km, sigma_h, sigma_v, ctx=None):
    """postproc::kernel_smooth: a smoothed copy of each kernel (None stays None)."""
    import torch
    out = []
    work = None
    for k in kernels:
        if k is None:
            out.append(None)
            continue
        if work is None or work.shape != k.shape:
            work = torch.empty_like(k)
        s = k.clone()
        pde_smooth(s, ygrid, zgrid, dx_deg, dy_deg, dz_km, sigma_h, sigma_v, work=work, ctx=ctx)
        out.append(s)
    return out


def kernel_precondition(ker_den, ker, ctx=None, stream=None):
    """postproc::kernel_precondition (src/postproc.cpp:487-517), in place on
    the device tensor ker: ker *= 1 / (ker_den / max|ker_den|) where that
    ratio exceeds 1e-12, unchanged elsewhere, nothing if max|ker_den| <
    1e-12 (sa_kernel_precondition)."""
    ctx = ctx or default_context()
    rc = _capi.lib().sa_kernel_precondition(ctx.h, ker.numel(), ptr(ker_den), ptr(ker), stream)
    _capi.check(ctx.h, rc)
    return ker


class MultigridSmoother:
    """The reference's multigrid smoothing (smooth_method 1,
    PostProc::InvGrid, src/postproc.cpp:160-386): nset staggered coarse grids
    of n_inv + 2 nodes per axis over the model grid; ``smooth`` projects a
    (nx, ny, nz) device field onto them and interpolates back
    (sa_multigrid_*)."""

    def __init__(self, xgrid, ygrid, zgrid, n_inv, nset, device=0):
        x = np.ascontiguousarray(xgrid, np.float64)
        y = np.ascontiguousarray(ygrid, np.float64)
        z = np.ascontiguousarray(zgrid, np.float64)
        ni = np.ascontiguousarray(n_inv, np.int32)
        h = C.c_void_p()
        rc = _capi.lib().sa_multigrid_create(int(device), x.size, y.size, z.size, x, y, z, ni,
                                             int(nset), C.byref(h))
        if rc != _capi.SA_OK:
            raise _capi.SAError(rc, "sa_multigrid_create")
        self.h = h
        self.shape = (x.size, y.size, z.size)

    def smooth(self, field, out=None, stream=None):
        import torch
        if out is None:
            out = torch.empty_like(field)
        rc = _capi.lib().sa_multigrid_smooth(self.h, ptr(field), ptr(out), stream)
        if rc != _capi.SA_OK:
            raise _capi.SAError(rc, "sa_multigrid_smooth")
        return out

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().sa_multigrid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
