"""CPU assembly of the exact gradient of chi with respect to vs (test
helper): the discrete eikonal adjoint's dchi/dsvel per period plane times
the derivatives of surfdisp96's phase-velocity roots, layer j = node j and
the half-space layer (a copy of the deepest node) added to the deepest node."""
import numpy as np


def _vs2vp(b):
    return 0.9409 + 2.0947 * b - 0.8206 * b * b + 0.2683 * b ** 3 - 0.0251 * b ** 4


def _vp2rho(a):
    return 1.6612 * a - 0.4721 * a * a + 0.0671 * a ** 3 - 0.0043 * a ** 4 + 0.000106 * a ** 5


def _dab(b):
    return 2.0947 - 2 * 0.8206 * b + 3 * 0.2683 * b * b - 4 * 0.0251 * b ** 3


def _dra(a):
    return 1.6612 - 2 * 0.4721 * a + 3 * 0.0671 * a * a - 4 * 0.0043 * a ** 3 + 5 * 0.000106 * a ** 4


def layer_thickness(z):
    nz = z.size
    thk = np.zeros(nz + 1)
    for kk in range(nz):
        thk[kk] = thk[kk - 1] if kk == nz - 1 else z[kk + 1] - z[kk]
    return thk


def dcdvs_nodes(orc, z, vs3d, periods, svel):
    """dc/dvs (nx, ny, nz, nper) of every column from the root derivatives."""
    nx, ny, nz = vs3d.shape
    thk = layer_thickness(z)
    out = np.zeros((nx, ny, nz, len(periods)))
    for ix in range(nx):
        for iy in range(ny):
            lv = np.append(vs3d[ix, iy], vs3d[ix, iy, -1])
            la = _vs2vp(lv)
            lr = _vp2rho(la)
            db, da, dr = orc.dispersion_dcdm(thk, la, lv, lr, periods, svel[:, iy, ix])
            node = db + da * _dab(lv) + dr * _dra(la) * _dab(lv)
            node[:, nz - 1] += node[:, nz]
            out[ix, iy] = node[:, :nz].T
    return out


def chain_gradient(orc, w, ev, vs0, nthreads=16):
    m11, m12, m22 = w.media()
    sv0, _ = orc.fwdsurf(w.zgrid, vs0, w.periods, nthreads=nthreads)
    o = orc.discrete_for_events(w.xx_deg, w.yy_deg, sv0, m11, m12, m22, ev, tol=0.0,
                                nthreads=nthreads)
    d = dcdvs_nodes(orc, w.zgrid, vs0, w.periods, sv0)
    return np.einsum("pyx,xykp->xyk", o["grad_svel"], d)
