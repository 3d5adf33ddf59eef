"""SurfGrid:: topography parts (reference src/surf_grid.cpp:80-190, :307-354,
src/topo.cpp) on the GPU: gridding the topography, the per-period media
matrices m11/m12/m22 with the dip angle, and the kernel-depth correction.
2-D fields are (ny, nx) planes ([iy][ix], the reference's column-major
nx x ny); per-period fields are (nper, ny, nx).  Device memory is held in
torch tensors; the arithmetic runs in libsurfatt_gpu.so.
"""
from __future__ import annotations

import numpy as np

from . import _capi, surfker
from ._capi import default_context, ptr

R_EARTH = 6371.0
DEG2RAD = np.pi / 180.0


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def grid_topography(lon_raw, lat_raw, z_raw_km, x, y, ctx=None):
    """Topography::grid: z_raw (nlat, nlon) in km -> (ny, nx) CUDA tensor."""
    import torch
    ctx = ctx or default_context()
    lr, la, z = _c(lon_raw), _c(lat_raw), _c(z_raw_km)
    x, y = _c(x), _c(y)
    out = torch.empty((y.size, x.size), dtype=torch.float64, device="cuda")
    rc = _capi.lib().sa_grid_topography(ctx.h, lr.size, la.size, lr, la, z, x.size, y.size, x, y,
                                        ptr(out))
    _capi.check(ctx.h, rc)
    return out


def average_phase_velocity(zgrid, vs1d, periods, iwave=2, ctx=None):
    """surfker::surfdisp of the 1-D model (src/surf_grid.cpp:91-99)."""
    import torch
    vs = torch.as_tensor(_c(vs1d).reshape(1, 1, -1), device="cuda")
    sv, _ = surfker.fwdsurf(zgrid, vs, periods, iwave=iwave, ctx=ctx)
    return sv[:, 0, 0].cpu().numpy()


def sigma_deg(avg_svel, periods, wavelen_factor):
    """Wavelength-based smoothing width per period (src/surf_grid.cpp:116-119)."""
    out = []
    for c, t in zip(avg_svel, periods):
        sigma_km = c * t * wavelen_factor / (2.0 * np.pi)
        out.append(sigma_km / (R_EARTH * DEG2RAD))
    return np.array(out)


def build_media_with_topo(x, y, z_gridded, sig_deg, ctx=None, stream=None):
    """Per-period m11, m12, m22 and dip angle (degrees), each (nper, ny, nx)."""
    import torch
    ctx = ctx or default_context()
    x, y, s = _c(x), _c(y), _c(sig_deg).ravel()
    shp = (s.size, y.size, x.size)
    f = dict(dtype=torch.float64, device=z_gridded.device)
    m11, m12, m22, ang = (torch.empty(shp, **f) for _ in range(4))
    rc = _capi.lib().sa_topo_media(ctx.h, x.size, y.size, x, y, ptr(z_gridded.contiguous()),
                                   s.size, s, ptr(m11), ptr(m12), ptr(m22), ptr(ang), stream)
    _capi.check(ctx.h, rc)
    return m11, m12, m22, ang


def correct_depth_with_topo(zgrid, angle, sen_vs=None, sen_vp=None, sen_rho=None, ctx=None,
                            stream=None):
    """In place on (nx, ny, nz, nper) CUDA tensors."""
    ctx = ctx or default_context()
    z = _c(zgrid)
    ref = next(t for t in (sen_vs, sen_vp, sen_rho) if t is not None)
    nx, ny, nz, nper = ref.shape
    rc = _capi.lib().sa_correct_depth_with_topo(ctx.h, nx, ny, nz, nper, z, ptr(angle),
                                                ptr(sen_vs), ptr(sen_vp), ptr(sen_rho), stream)
    _capi.check(ctx.h, rc)
