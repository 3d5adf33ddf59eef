"""surfker:: call surface (reference include/surfdisp.h) over many columns on the GPU.

``fwdsurf`` replaces SurfGrid::fwdsurf (phase/group velocity per column and
period), ``depthkernel_hti`` replaces SurfGrid::compute_dispersion_kernel for
Rayleigh phase velocity (sen_vs, sen_vp, sen_rho), and ``combine_kernels_vs``
replaces preproc::combine_kernels (vs-only parametrisation).  Arrays are torch
CUDA tensors (float64, contiguous); all arithmetic runs in libsurfatt_gpu.so.
"""
from __future__ import annotations

import numpy as np

from . import _capi
from ._capi import default_context, ptr


class DispersionError(RuntimeError):
    """surfdisp96 found no root for some column (the reference stops with
    'Dispersion calculation failed')."""


def fwdsurf(zgrid, vs3d, periods, iwave=2, igr=0, ctx=None, stream=None, check=True):
    """vs3d (nx, ny, nz) on device -> svel (nper, ny, nx), status (ny, nx)."""
    import torch
    ctx = ctx or default_context()
    nx, ny, nz = vs3d.shape
    p = np.ascontiguousarray(periods, dtype=np.float64)
    z = np.ascontiguousarray(zgrid, dtype=np.float64)
    svel = torch.empty((p.size, ny, nx), dtype=torch.float64, device=vs3d.device)
    status = torch.zeros((ny, nx), dtype=torch.int32, device=vs3d.device)
    rc = _capi.lib().sa_surfdisp_columns(ctx.h, nx, ny, nz, z, ptr(vs3d), p.size, p, iwave, igr,
                                         ptr(svel), ptr(status), stream)
    _capi.check(ctx.h, rc)
    if check:
        torch.cuda.synchronize(vs3d.device)
        if int(status.max()) != 0:
            raise DispersionError(f"Dispersion calculation failed in {int(status.sum())} columns")
    return svel, status


def depthkernel_hti(zgrid, vs3d, periods, cp, ctx=None, stream=None, out=None):
    """Rayleigh phase-velocity depth kernels (nx, ny, nz, nper) x 3 at the
    phase velocities cp (nper, ny, nx) from fwdsurf(igr=0); `out` (three
    such float64 device tensors) is reused when given."""
    import torch
    ctx = ctx or default_context()
    nx, ny, nz = vs3d.shape
    p = np.ascontiguousarray(periods, dtype=np.float64)
    z = np.ascontiguousarray(zgrid, dtype=np.float64)
    shp = (nx, ny, nz, p.size)
    if out is None:
        out = [torch.empty(shp, dtype=torch.float64, device=vs3d.device) for _ in range(3)]
    elif any(tuple(o.shape) != shp or o.dtype != torch.float64 or not o.is_contiguous()
             for o in out):
        raise ValueError("out: three contiguous float64 tensors of shape (nx, ny, nz, nper)")
    rc = _capi.lib().sa_depthkernel_columns(ctx.h, nx, ny, nz, z, ptr(vs3d), p.size, p, ptr(cp),
                                            ptr(out[0]), ptr(out[1]), ptr(out[2]), stream)
    _capi.check(ctx.h, rc)
    return tuple(out)


def combine_kernels_vs(adj_s, vs3d, vp3d, sen_vs, sen_vp, sen_rho, ctx=None, stream=None):
    """K_vs (nx, ny, nz) from adj_s (nper, ny, nx) and the depth kernels."""
    import torch
    ctx = ctx or default_context()
    nper, ny, nx = adj_s.shape
    nz = vs3d.shape[2]
    ker = torch.empty((nx, ny, nz), dtype=torch.float64, device=adj_s.device)
    rc = _capi.lib().sa_combine_kernels_vs(ctx.h, nx, ny, nz, nper, ptr(adj_s), ptr(vs3d),
                                           ptr(vp3d), ptr(sen_vs), ptr(sen_vp), ptr(sen_rho),
                                           ptr(ker), stream)
    _capi.check(ctx.h, rc)
    return ker


def depthkernel_group(zgrid, vs3d, periods, ctx=None, stream=None):
    """Rayleigh group-velocity depth kernels (surfker::depthkernel_rayleigh_group):
    (sen_vs, sen_vp, sen_rho) each (nx, ny, nz, nper); raises DispersionError
    where a root search fails."""
    import torch
    ctx = ctx or default_context()
    nx, ny, nz = vs3d.shape
    p = np.ascontiguousarray(periods, dtype=np.float64)
    z = np.ascontiguousarray(zgrid, dtype=np.float64)
    out = [torch.empty((nx, ny, nz, p.size), dtype=torch.float64, device=vs3d.device)
           for _ in range(3)]
    status = np.zeros(nx * ny, np.int32)
    rc = _capi.lib().sa_depthkernel_columns_group(ctx.h, nx, ny, nz, z, ptr(vs3d), p.size, p,
                                                  ptr(out[0]), ptr(out[1]), ptr(out[2]),
                                                  status.ctypes.data, stream)
    if rc == _capi.SA_ERR_NOROOT:
        raise DispersionError(f"Dispersion calculation failed in {int((status != 0).sum())} columns")
    _capi.check(ctx.h, rc)
    return tuple(out)


def depthkernel_love(zgrid, vs3d, periods, igr=0, ctx=None, stream=None):
    """Love-wave depth kernels (surfker::depthkernel_love_phase for igr 0,
    depthkernel_love_group for igr 1): (sen_vs, sen_rho) each (nx, ny, nz,
    nper) -- dc/db, dc/drho (du/db, du/drho); raises DispersionError where a
    root search fails."""
    import torch
    ctx = ctx or default_context()
    nx, ny, nz = vs3d.shape
    p = np.ascontiguousarray(periods, dtype=np.float64)
    z = np.ascontiguousarray(zgrid, dtype=np.float64)
    out = [torch.empty((nx, ny, nz, p.size), dtype=torch.float64, device=vs3d.device)
           for _ in range(2)]
    status = np.zeros(nx * ny, np.int32)
    rc = _capi.lib().sa_depthkernel_columns_love(ctx.h, nx, ny, nz, z, ptr(vs3d), p.size, p,
                                                 int(igr), ptr(out[0]), ptr(out[1]),
                                                 status.ctypes.data, stream)
    if rc == _capi.SA_ERR_NOROOT:
        raise DispersionError(f"Dispersion calculation failed in {int((status != 0).sum())} columns")
    _capi.check(ctx.h, rc)
    return tuple(out)
