"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` as the parity checker and the timed CPU
restatement of the reference.  The product (``surfattpp_b200``) never imports it.

Array conventions: 2-D fields are numpy arrays shaped (ny, nx) in C order, which
is the reference's Eigen column-major (nx x ny) layout, index ix + nx*iy.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
# The same restatement with the correctly rounded exp / log / sin / cos of
# surfattpp_b200/csrc/crmath.cuh in place of the C library's (omath.h): the
# device column kernels use those functions, so against this build they must
# agree bit for bit; against the default build they differ only where the C
# library misrounds.
_LIB_CR_PATH = os.path.join(_HERE, "_build", "liboracle_cr.so")
_lib = None
_lib_cr = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (g++ only, a few seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib_native = None


def _native_path() -> str:
    """Per-host location of the -march=native build (keyed by the CPU model
    and flags, so a library built on another host is never loaded)."""
    import hashlib
    try:
        with open("/proc/cpuinfo") as f:
            info = [ln for ln in f if ln.startswith(("model name", "flags"))][:2]
    except OSError:
        info = []
    tag = hashlib.sha1("".join(info).encode()).hexdigest()[:12]
    return os.path.join(_HERE, "_build", f"native-{tag}", "liboracle_native.so")


def lib(math: str = "libc"):
    """The oracle library; math="cr" selects the correctly rounded libm build,
    math="native" the timing build with the reference's release flags
    (-O3 -march=native, built on first use on this host)."""
    global _lib, _lib_cr, _lib_native
    if math == "native":
        if _lib_native is None:
            path = _native_path()
            # make rebuilds it when a source is newer
            subprocess.run(["make", "-s", "-C", _HERE, f"NATIVE_OUT={path}", path], check=True)
            _lib_native = _declare(C.CDLL(path))
        return _lib_native
    if math == "cr":
        if _lib_cr is None:
            if not os.path.exists(_LIB_CR_PATH):
                build()
            _lib_cr = _declare(C.CDLL(_LIB_CR_PATH))
        return _lib_cr
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    _lib = _declare(C.CDLL(_LIB_PATH))
    return _lib


def _declare(L):
    i, d = C.c_int, C.c_double
    L.orc_eik_fwd.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, _dp, d, d, _dp, C.POINTER(i)]
    L.orc_eik_fwd.restype = i
    L.orc_eik_adj.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, _dp, i, _dp, _dp, _dp, _dp,
                              C.POINTER(i)]
    L.orc_eik_adj.restype = i
    L.orc_eik_fwd_tol.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, _dp, d, d, d, i, _dp,
                                  C.POINTER(i)]
    L.orc_eik_fwd_tol.restype = i
    L.orc_eik_discrete_grad.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, _dp, d, d, d, i, i, _dp,
                                        _dp, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(i)]
    L.orc_eik_discrete_grad.restype = i
    L.orc_discrete_for_events.argtypes = [i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, i, _dp, _dp,
                                          _ip, _ip, _ip, _dp, _dp, C.c_void_p, _dp, C.c_void_p,
                                          d, i, _dp, C.c_void_p, C.POINTER(d), _ip, i]
    L.orc_discrete_for_events.restype = i
    L.orc_dispersion_dcdm.argtypes = [_fp, _fp, _fp, _fp, i, i, _dp, _dp, _dp, _dp, _dp]
    L.orc_dispersion_dcdm.restype = i
    L.orc_mask_uniform_grid.argtypes = [i, i, _dp, _dp, _dp, d, d]
    L.orc_interp2d.argtypes = [i, i, _dp, _dp, _dp, i, _dp, _dp, _dp]
    L.orc_forward_for_events.argtypes = [i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, i, _dp, _dp,
                                         _ip, _ip, _ip, _dp, _dp, _dp, _dp, i, _dp, _dp,
                                         C.POINTER(d), _ip, _ip, i, C.c_void_p]
    L.orc_kernel_precondition.argtypes = [C.c_size_t, _dp, _dp]
    L.orc_slegn96.argtypes = [_fp, _fp, _fp, i, d, d, C.POINTER(d), _dp, _dp, i]
    L.orc_slegnpu.argtypes = [_fp, _fp, _fp, i, d, d, d, d, d, d, C.POINTER(d), _dp, _dp, i]
    L.orc_depthkernel_love.argtypes = [i, i, i, _dp, _dp, i, _dp, i, _dp, _dp, _ip, i]
    L.orc_multigrid_smooth.argtypes = [i, i, i, _dp, _dp, _dp, _ip, i, _dp, _dp]
    L.orc_multigrid_smooth.restype = i
    L.orc_combine_kernels_vs.argtypes = [i, i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
    for f in ("orc_vs2vp", "orc_vp2rho", "orc_dalpha_dbeta", "orc_drho_dalpha"):
        getattr(L, f).argtypes = [d]
        getattr(L, f).restype = d
    L.orc_surfdisp96.argtypes = [_fp, _fp, _fp, _fp, i, i, i, i, i, i, _dp, _dp]
    L.orc_surfdisp96.restype = i
    L.orc_sregn96_hti.argtypes = [_fp, _fp, _fp, _fp, i, _dp, _dp, _dp] + [_dp] * 10 + [i]
    L.orc_sregn96.argtypes = [_fp, _fp, _fp, _fp, i, _dp, _dp, _dp] + [_dp] * 8 + [i]
    L.orc_fwdsurf.argtypes = [i, i, i, _dp, _dp, i, _dp, i, i, _dp, _ip, i]
    L.orc_depthkernel_hti.argtypes = [i, i, i, _dp, _dp, i, _dp, _dp, _dp, _dp, _ip, i]
    L.orc_pde_smooth_nstep.argtypes = [i, d, d, d, d, d, d, d, C.POINTER(d), C.POINTER(d)]
    L.orc_pde_smooth_nstep.restype = i
    L.orc_pde_smooth.argtypes = [i, i, i, d, d, d, _dp, _dp, d, d, _dp, C.POINTER(i)]
    L.orc_pde_smooth.restype = i
    z = C.c_size_t
    L.orc_lbfgs_direction.argtypes = [z, i, C.POINTER(C.POINTER(d)), C.POINTER(C.POINTER(d)), _dp]
    L.orc_grad_normalization.argtypes = [z, _dp]
    L.orc_grad_normalization.restype = d
    L.orc_descent_angle.argtypes = [z, _dp, _dp]
    L.orc_descent_angle.restype = d
    L.orc_wolfe_condition.argtypes = [d, d, d, C.POINTER(d), C.POINTER(d), d, d, i, d, d, i, d,
                                      C.POINTER(d)]
    L.orc_wolfe_condition.restype = i
    L.orc_model_update_vs.argtypes = [z, _dp, _dp, d, _dp, _dp, _dp]
    L.orc_depthkernel_group.argtypes = [i, i, i, _dp, _dp, i, _dp, _dp, _dp, _dp, _ip, i]
    L.orc_sregnpu.argtypes = [_fp, _fp, _fp, _fp, i, d, d, d, d, d, d, C.POINTER(d)] + [_dp] * 8 + [i]
    L.orc_gaussian_smooth_geo_2.argtypes = [i, i, _dp, _dp, _dp, d, _dp]
    L.orc_gradient_2_geo.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp]
    L.orc_topo_media.argtypes = [i, i, _dp, _dp, _dp, i, _dp, _dp, _dp, _dp, _dp]
    L.orc_correct_depth_with_topo.argtypes = [i, i, i, i, _dp, _dp, _dp]
    return L


def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dtype=dt)


def eik_fwd(xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg, y0_deg):
    """eikonal::FSM_UW_PS_lonlat_2d. Fields (ny, nx). Returns (T, niter)."""
    xx, yy = _c(xx_deg), _c(yy_deg)
    nx, ny = xx.size, yy.size
    T = np.zeros((ny, nx))
    it = C.c_int(0)
    rc = lib().orc_eik_fwd(nx, ny, xx, yy, _c(spha), _c(sphb), _c(sphc), _c(fun),
                           float(x0_deg), float(y0_deg), T, C.byref(it))
    if rc != 0:
        raise ValueError("Grid must be at least 3x3")
    return T, it.value


def eik_fwd_tol(xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg, y0_deg, tol=0.0,
                maxiter=5000):
    """The forward solve with its stopping rule as a parameter (tol 0: to a
    fixed point).  Returns (T, niter)."""
    xx, yy = _c(xx_deg), _c(yy_deg)
    nx, ny = xx.size, yy.size
    T = np.zeros((ny, nx))
    it = C.c_int(0)
    rc = lib().orc_eik_fwd_tol(nx, ny, xx, yy, _c(spha), _c(sphb), _c(sphc), _c(fun),
                               float(x0_deg), float(y0_deg), float(tol), int(maxiter), T,
                               C.byref(it))
    if rc != 0:
        raise ValueError("Grid must be at least 3x3")
    return T, it.value


def eik_discrete_grad(xx_deg, yy_deg, spha, sphb, sphc, fun, x0_deg, y0_deg, xrec, yrec,
                      dchi_dT, tol=0.0, maxiter=5000):
    """Exact discrete adjoint of the forward solve: (syn [nr], dchi/dfun
    (ny, nx), niter) for the receiver-time sensitivities dchi_dT [nr]."""
    xx, yy = _c(xx_deg), _c(yy_deg)
    nx, ny = xx.size, yy.size
    xr, yr, dd = _c(xrec).ravel(), _c(yrec).ravel(), _c(dchi_dT).ravel()
    syn = np.zeros(max(xr.size, 1))
    g = np.zeros((ny, nx))
    it = C.c_int(0)
    rc = lib().orc_eik_discrete_grad(nx, ny, xx, yy, _c(spha), _c(sphb), _c(sphc), _c(fun),
                                     float(x0_deg), float(y0_deg), float(tol), int(maxiter),
                                     xr.size, xr if xr.size else np.zeros(1),
                                     yr if yr.size else np.zeros(1),
                                     dd.ctypes.data if dd.size else None, syn.ctypes.data,
                                     g.ctypes.data, C.byref(it))
    if rc == -1:
        raise ValueError("Grid must be at least 3x3")
    if rc == -2:
        raise RuntimeError("forward solve did not reach its stopping rule")
    return syn[:xr.size], g, it.value


def discrete_for_events(xx_deg, yy_deg, svel, m11, m12, m22, ev, tol=0.0, maxiter=5000,
                        grad=True, sadj=None, nthreads=1):
    """The event batch with the exact discrete gradient: dict(syn, chi,
    grad_svel (nper, ny, nx) = dchi/dsvel, fwd_iters).  With sadj [npair],
    grad_svel is the vector-Jacobian product of the receiver times with it."""
    xx, yy = _c(xx_deg), _c(yy_deg)
    nper, ny, nx = svel.shape
    ne = len(ev["evlo"])
    nrec = int(ev["rec_ptr"][-1])
    syn = np.zeros(max(nrec, 1))
    g = np.zeros((nper, ny, nx)) if grad else None
    chi = C.c_double(0.0)
    fi = np.zeros(max(ne, 1), np.int32)
    tt = _c(ev["tt_obs"]) if ev.get("tt_obs") is not None else None
    sa = _c(sadj) if sadj is not None else None
    rc = lib().orc_discrete_for_events(
        nx, ny, nper, xx, yy, _c(svel), _c(m11), _c(m12), _c(m22), ne, _c(ev["evlo"]),
        _c(ev["evla"]), _c(ev["iper"], np.int32), _c(ev["rec_ptr"], np.int32),
        _c(ev["rec_idx"], np.int32), _c(ev["stlo"]), _c(ev["stla"]),
        tt.ctypes.data if tt is not None else None, _c(ev["weight"]),
        sa.ctypes.data if sa is not None else None, float(tol), int(maxiter), syn,
        g.ctypes.data if g is not None else None, C.byref(chi), fi, int(nthreads))
    if rc == -2:
        raise RuntimeError("forward solve did not reach its stopping rule")
    return dict(syn=syn[:nrec], chi=chi.value, grad_svel=g, fwd_iters=fi[:ne])


def eik_adj(xx_deg, yy_deg, spha, sphb, sphc, T, xrec, yrec, sadj):
    """eikonal::FSM_O1_JSE_lonlat_2d. Returns (Ta, niter)."""
    xx, yy = _c(xx_deg), _c(yy_deg)
    nx, ny = xx.size, yy.size
    Ta = np.zeros((ny, nx))
    it = C.c_int(0)
    xr, yr, sa = _c(xrec).ravel(), _c(yrec).ravel(), _c(sadj).ravel()
    lib().orc_eik_adj(nx, ny, xx, yy, _c(spha), _c(sphb), _c(sphc), _c(T), xr.size,
                      xr if xr.size else np.zeros(1), yr if yr.size else np.zeros(1),
                      sa if sa.size else np.zeros(1), Ta, C.byref(it))
    return Ta, it.value


def mask_uniform_grid(xx_deg, yy_deg, table, x0, y0):
    t = _c(table).copy()
    xx, yy = _c(xx_deg), _c(yy_deg)
    lib().orc_mask_uniform_grid(xx.size, yy.size, xx, yy, t, float(x0), float(y0))
    return t


def interp2d(xgrid, ygrid, z, xq, yq):
    xg, yg = _c(xgrid), _c(ygrid)
    xq, yq = _c(xq).ravel(), _c(yq).ravel()
    out = np.zeros(xq.size)
    lib().orc_interp2d(xg.size, yg.size, xg, yg, _c(z), xq.size, xq, yq, out)
    return out


def forward_for_events(xx_deg, yy_deg, svel, m11, m12, m22, ev, calc_adj=True, nthreads=1,
                       math="libc", kden=False):
    """preproc::forward_for_event over an event set.

    svel/m11/m12/m22: (nper, ny, nx).  ``ev`` is a dict with evlo, evla, iper,
    rec_ptr, rec_idx, stlo, stla, tt_obs, weight (see tests/workloads.py).
    math: which build runs it (see lib()).  kden: also the kernel-density
    adjoint (is_kden, src/preproc.cpp:128-137), returned as kden_s.
    Returns dict(syn, adj_s, chi, fwd_iters, adj_iters[, kden_s]).
    """
    xx, yy = _c(xx_deg), _c(yy_deg)
    nper, ny, nx = svel.shape
    ne = len(ev["evlo"])
    nrec = int(ev["rec_ptr"][-1])
    syn = np.zeros(max(nrec, 1))
    adj_s = np.zeros((nper, ny, nx))
    kden_s = np.zeros((nper, ny, nx)) if kden else None
    chi = C.c_double(0.0)
    fi = np.zeros(max(ne, 1), np.int32)
    ai = np.zeros(max(ne, 1), np.int32)
    lib(math).orc_forward_for_events(
        nx, ny, nper, xx, yy, _c(svel), _c(m11), _c(m12), _c(m22), ne,
        _c(ev["evlo"]), _c(ev["evla"]), _c(ev["iper"], np.int32), _c(ev["rec_ptr"], np.int32),
        _c(ev["rec_idx"], np.int32), _c(ev["stlo"]), _c(ev["stla"]), _c(ev["tt_obs"]),
        _c(ev["weight"]), int(calc_adj), syn, adj_s, C.byref(chi), fi, ai, int(nthreads),
        kden_s.ctypes.data if kden_s is not None else None)
    out = dict(syn=syn[:nrec], adj_s=adj_s, chi=chi.value, fwd_iters=fi[:ne], adj_iters=ai[:ne])
    if kden_s is not None:
        out["kden_s"] = kden_s
    return out


def kernel_precondition(ker_den, ker):
    """postproc::kernel_precondition: a preconditioned copy of ker."""
    out = _c(ker).copy()
    lib().orc_kernel_precondition(out.size, _c(ker_den), out)
    return out


def combine_kernels_vs(adj_s, vs3d, vp3d, sen_vs, sen_vp, sen_rho):
    nper, ny, nx = adj_s.shape
    nz = vs3d.shape[2]
    ker = np.zeros((nx, ny, nz))
    lib().orc_combine_kernels_vs(nx, ny, nz, nper, _c(adj_s), _c(vs3d), _c(vp3d), _c(sen_vs),
                                 _c(sen_vp), _c(sen_rho), ker)
    return ker


def vs2vp(vs):
    return lib().orc_vs2vp(float(vs))


def vp2rho(vp):
    return lib().orc_vp2rho(float(vp))


def dalpha_dbeta(vs):
    return lib().orc_dalpha_dbeta(float(vs))


def drho_dalpha(vp):
    return lib().orc_drho_dalpha(float(vp))


def surfdisp96(thk, vp, vs, rho, periods, iflsph=1, iwave=2, mode=1, igr=0):
    """surfdisp96_c. Returns (velocities, status)."""
    t = _c(periods)
    cg = np.zeros(t.size)
    st = lib().orc_surfdisp96(_c(thk, np.float32), _c(vp, np.float32), _c(vs, np.float32),
                              _c(rho, np.float32), len(thk), iflsph, iwave, mode, igr, t.size,
                              t, cg)
    return cg, st


def dispersion_dcdm(thk, vp, vs, rho, periods, c):
    """dc/d(vs, vp, rho) of surfdisp96's Rayleigh phase velocities c at
    `periods` for every layer: three arrays (nper, nlayer)."""
    t, cc = _c(periods), _c(c)
    n = len(thk)
    out = [np.zeros((t.size, n)) for _ in range(3)]
    rc = lib().orc_dispersion_dcdm(_c(thk, np.float32), _c(vp, np.float32), _c(vs, np.float32),
                                   _c(rho, np.float32), n, t.size, t, cc, *out)
    if rc:
        raise ValueError("water layers are not supported")
    return tuple(out)


def sregn96_hti(thk, vp, vs, rho, t, cp, iflsph=1):
    """sregn96_hti_c for one period. Returns dict of outputs."""
    n = len(thk)
    outs = {k: np.zeros(n) for k in ("dispu", "dispw", "stressu", "stressw", "dc2da", "dc2db",
                                      "dc2dh", "dc2dr", "dc2dgc", "dc2dgs")}
    tt, cpp, cg = np.array([float(t)]), np.array([float(cp)]), np.zeros(1)
    lib().orc_sregn96_hti(_c(thk, np.float32), _c(vp, np.float32), _c(vs, np.float32),
                          _c(rho, np.float32), n, tt, cpp, cg, *outs.values(), iflsph)
    outs["cp"], outs["cg"] = cpp[0], cg[0]
    return outs


def fwdsurf(zgrid, vs3d, periods, iwave=2, igr=0, nthreads=1, math="libc"):
    """SurfGrid::fwdsurf: vs3d (nx, ny, nz) -> svel (nper, ny, nx), status (ny, nx)."""
    nx, ny, nz = vs3d.shape
    p = _c(periods)
    svel = np.zeros((p.size, ny, nx))
    st = np.zeros((ny, nx), np.int32)
    lib(math).orc_fwdsurf(nx, ny, nz, _c(zgrid), _c(vs3d), p.size, p, iwave, igr, svel, st,
                      int(nthreads))
    return svel, st


def depthkernel_hti(zgrid, vs3d, periods, nthreads=1, math="libc"):
    """compute_dispersion_kernel (PH): returns sen_vs, sen_vp, sen_rho (nx,ny,nz,nper), status."""
    nx, ny, nz = vs3d.shape
    p = _c(periods)
    shp = (nx, ny, nz, p.size)
    sv, sp, sr = np.zeros(shp), np.zeros(shp), np.zeros(shp)
    st = np.zeros((ny, nx), np.int32)
    lib(math).orc_depthkernel_hti(nx, ny, nz, _c(zgrid), _c(vs3d), p.size, p, sv, sp, sr, st,
                              int(nthreads))
    return sv, sp, sr, st


def pde_smooth_nstep(ny, dx, dy, dz, y_first, y_last, sigma_h, sigma_v):
    """(nstep, ch, cv) of PostProc::pde_smooth (src/postproc.cpp:407-434)."""
    ch, cv = C.c_double(), C.c_double()
    n = lib().orc_pde_smooth_nstep(ny, dx, dy, dz, y_first, y_last, sigma_h, sigma_v,
                                   C.byref(ch), C.byref(cv))
    return n, ch.value, cv.value


def pde_smooth(field, dx, dy, dz, ygrid, zgrid, sigma_h, sigma_v):
    """PostProc::pde_smooth on one rank: returns (smoothed copy, nstep)."""
    f = _c(field).copy()
    nx, ny, nz = f.shape
    ns = C.c_int(0)
    rc = lib().orc_pde_smooth(nx, ny, nz, dx, dy, dz, _c(ygrid), _c(zgrid), sigma_h, sigma_v, f,
                              C.byref(ns))
    if rc != 0:
        raise ValueError(f"orc_pde_smooth failed ({rc})")
    return f, ns.value


def lbfgs_direction(models, grads):
    """optimize::lbfgs_direction over consecutive iterates (oldest first, the
    current one last): returns H g."""
    ms = [_c(m).ravel() for m in models]
    gs = [_c(g).ravel() for g in grads]
    n = ms[-1].size
    P = C.POINTER(C.c_double)
    mp = (P * len(ms))(*[m.ctypes.data_as(P) for m in ms])
    gp = (P * len(gs))(*[g.ctypes.data_as(P) for g in gs])
    out = np.zeros(n)
    lib().orc_lbfgs_direction(n, len(ms) - 1, mp, gp, out)
    return out


def grad_normalization(g):
    g = _c(g).ravel().copy()
    m = lib().orc_grad_normalization(g.size, g)
    return g, m


def descent_angle(direction, grad):
    return lib().orc_descent_angle(_c(direction).size, _c(direction).ravel(), _c(grad).ravel())


def wolfe_condition(gd, kd, alpha, alpha_L, alpha_R, f0, f1, subiter, c1, c2, max_sub, alpha_init):
    aL, aR, nxt = C.c_double(alpha_L), C.c_double(alpha_R), C.c_double()
    st = lib().orc_wolfe_condition(gd, kd, alpha, C.byref(aL), C.byref(aR), f0, f1, subiter, c1,
                                   c2, max_sub, alpha_init, C.byref(nxt))
    return st, nxt.value, aL.value, aR.value


def model_update_vs(vs, direction, alpha):
    v = _c(vs).ravel()
    n = v.size
    o1, o2, o3 = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().orc_model_update_vs(n, v, _c(direction).ravel(), alpha, o1, o2, o3)
    return o1, o2, o3


def gaussian_smooth_geo_2(data, lons, lats, sigma):
    """data (ny, nx) planes as elsewhere in this module ([iy][ix])."""
    d = _c(data)
    ny, nx = d.shape
    out = np.zeros((ny, nx))
    lib().orc_gaussian_smooth_geo_2(nx, ny, d, _c(lons), _c(lats), float(sigma), out)
    return out


def gradient_2_geo(f, lon, lat):
    d = _c(f)
    ny, nx = d.shape
    tx, ty = np.zeros((ny, nx)), np.zeros((ny, nx))
    lib().orc_gradient_2_geo(nx, ny, d, _c(lon), _c(lat), tx, ty)
    return tx, ty


def topo_media(lon, lat, z_gridded, sigma_deg):
    """Per-period media (m11, m12, m22, angle), each (nper, ny, nx)."""
    z = _c(z_gridded)
    ny, nx = z.shape
    s = _c(sigma_deg).ravel()
    shp = (s.size, ny, nx)
    m11, m12, m22, ang = np.zeros(shp), np.zeros(shp), np.zeros(shp), np.zeros(shp)
    lib().orc_topo_media(nx, ny, _c(lon), _c(lat), z, s.size, s, m11, m12, m22, ang)
    return m11, m12, m22, ang


def correct_depth_with_topo(zgrid, angle, ker):
    """ker (nx, ny, nz, nper) corrected copy; angle (nper, ny, nx)."""
    k = _c(ker).copy()
    nx, ny, nz, nper = k.shape
    lib().orc_correct_depth_with_topo(nx, ny, nz, nper, _c(zgrid), _c(angle), k)
    return k


def depthkernel_group(zgrid, vs3d, periods, nthreads=1, math="libc"):
    """Rayleigh group-velocity depth kernels: sen_vs, sen_vp, sen_rho (nx,ny,nz,nper), status."""
    nx, ny, nz = vs3d.shape
    p = _c(periods)
    shp = (nx, ny, nz, p.size)
    sv, sp, sr = np.zeros(shp), np.zeros(shp), np.zeros(shp)
    st = np.zeros((ny, nx), np.int32)
    lib(math).orc_depthkernel_group(nx, ny, nz, _c(zgrid), _c(vs3d), p.size, p, sv, sp, sr, st,
                                int(nthreads))
    return sv, sp, sr, st


def depthkernel_love(zgrid, vs3d, periods, igr=0, nthreads=1, math="libc"):
    """Love-wave depth kernels (depthkernel_love_phase / _group): sen_vs,
    sen_rho (nx, ny, nz, nper), status (ny, nx)."""
    nx, ny, nz = vs3d.shape
    p = _c(periods)
    shp = (nx, ny, nz, p.size)
    sv, sr = np.zeros(shp), np.zeros(shp)
    st = np.zeros((ny, nx), np.int32)
    lib(math).orc_depthkernel_love(nx, ny, nz, _c(zgrid), _c(vs3d), p.size, p, int(igr), sv, sr,
                                   st, int(nthreads))
    return sv, sr, st


def slegn96(thk, vs, rho, t, cp, iflsph=1):
    """One slegn96 call: dict(dc2db, dc2dr, cg)."""
    n = len(thk)
    kb, kr, cg = np.zeros(n), np.zeros(n), C.c_double()
    f = lambda a: _c(a, np.float32)
    lib().orc_slegn96(f(thk), f(vs), f(rho), n, float(t), float(cp), C.byref(cg), kb, kr,
                      int(iflsph))
    return dict(dc2db=kb, dc2dr=kr, cg=cg.value)


def multigrid_smooth(field, x, y, z, n_inv, nset):
    """PostProc::smooth with smooth_method 1 on a (nx, ny, nz) field."""
    f = _c(field)
    out = np.zeros_like(f)
    rc = lib().orc_multigrid_smooth(f.shape[0], f.shape[1], f.shape[2], _c(x), _c(y), _c(z),
                                    _c(n_inv, np.int32), int(nset), f, out)
    if rc != 0:
        raise ValueError("a node lies outside a coarse grid")
    return out
