"""Seeded synthetic workloads for the forward + adjoint misfit-gradient path.

There is no public dataset for this path; every input is generated here from a
seed, with the shapes, sizes and value ranges of the reference's example
``examples/00_checkerboard_iso`` (25 stations, 2x3x2 checkerboard) scaled up
for the larger cases.

Layouts (same as the reference):
  vs3d        (nx, ny, nz) row-major, as ModelGrid::vs3d_loc(ix, iy, k)
  2-D fields  numpy (ny, nx), i.e. Eigen column-major nx x ny (index ix + nx*iy)
  per-period  (nper, ny, nx)
  events      CSR: rec_ptr[ne+1] over rec_idx (station indices); one event is
              one (source, period) pair as in SrcRec::events_local
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

R_EARTH = 6371.0


def vs2vp(vs):
    """Brocher (2005) Vp(Vs), scalar form of include/utils.h:185-187."""
    return 0.9409 + 2.0947 * vs - 0.8206 * vs * vs + 0.2683 * vs * vs * vs - 0.0251 * vs * vs * vs * vs


def vp2rho(vp):
    """Brocher (2005) rho(Vp), include/utils.h:223-225."""
    return (1.6612 * vp - 0.4721 * vp * vp + 0.0671 * vp * vp * vp - 0.0043 * vp * vp * vp * vp
            + 0.000106 * vp * vp * vp * vp * vp)


@dataclass
class Workload:
    name: str
    xx_deg: np.ndarray
    yy_deg: np.ndarray
    zgrid: np.ndarray
    vs3d: np.ndarray                 # (nx, ny, nz)
    periods: np.ndarray
    stlo: np.ndarray
    stla: np.ndarray
    evlo: np.ndarray
    evla: np.ndarray
    iper: np.ndarray
    rec_ptr: np.ndarray
    rec_idx: np.ndarray
    tt_obs: np.ndarray
    weight: np.ndarray
    m11: np.ndarray | None = None    # (nper, ny, nx); None means isotropic 1, 0, 1
    m12: np.ndarray | None = None
    m22: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def nx(self):
        return self.xx_deg.size

    @property
    def ny(self):
        return self.yy_deg.size

    @property
    def nz(self):
        return self.zgrid.size

    @property
    def nper(self):
        return self.periods.size

    @property
    def n_events(self):
        return self.evlo.size

    def media(self):
        """m11, m12, m22 planes (nper, ny, nx); isotropic flat surface if unset."""
        shp = (self.nper, self.ny, self.nx)
        if self.m11 is None:
            # SurfGrid::build_media without topography: a = b = 1, c = +0 and
            # m12 = -c = -0.0 (src/surf_grid.cpp:178-190)
            return np.ones(shp), np.full(shp, -0.0), np.ones(shp)
        return self.m11, self.m12, self.m22

    def events(self):
        return dict(evlo=self.evlo, evla=self.evla, iper=self.iper, rec_ptr=self.rec_ptr,
                    rec_idx=self.rec_idx, stlo=self.stlo, stla=self.stla,
                    tt_obs=self.tt_obs, weight=self.weight)


def _grid(lon0, lat0, n, d):
    return lon0 + d * np.arange(n[0]), lat0 + d * np.arange(n[1])


def _stations(rng, xx, yy, nsta, margin_cells=2):
    dx, dy = xx[1] - xx[0], yy[1] - yy[0]
    lo = rng.uniform(xx[0] + margin_cells * dx, xx[-1] - margin_cells * dx, nsta)
    la = rng.uniform(yy[0] + margin_cells * dy, yy[-1] - margin_cells * dy, nsta)
    return lo, la


def _all_pairs_events(stlo, stla, nper):
    """Every station is a source for every period (station-major, then
    period); all other stations, in order, are its receivers."""
    nsta = stlo.size
    ne = nsta * nper
    src = np.repeat(np.arange(nsta), nper)
    iper = np.tile(np.arange(nper, dtype=np.int32), nsta)
    ptr = (np.arange(ne + 1, dtype=np.int64) * (nsta - 1)).astype(np.int32)
    # receivers of source s: 0..s-1, s+1..nsta-1
    r = np.tile(np.arange(nsta - 1, dtype=np.int32), ne)
    idx = r + (r >= np.repeat(src, nsta - 1)).astype(np.int32)
    return (np.asarray(stlo)[src].astype(float), np.asarray(stla)[src].astype(float), iper, ptr,
            idx.astype(np.int32))


def checker_pattern(nx, ny, nz, nxw, nyw, nzw):
    """ModelGrid::build_perturbation_pattern with hmargin = 0, anom_size <= 0
    (src/model_grid.cpp:523-572)."""
    xp = np.sin(nxw * np.pi * np.arange(nx) / nx)
    yp = np.sin(nyw * np.pi * np.arange(ny) / ny)
    zp = np.sin(nzw * np.pi * np.arange(nz) / nz)
    return xp, yp, zp


def gradient_model(nx, ny, zgrid, v0=2.8, v1=4.6):
    z = np.asarray(zgrid)
    vs1d = v0 + (v1 - v0) * z / z[-1]
    return np.broadcast_to(vs1d, (nx, ny, z.size)).copy()


def add_checker(vs3d, pert, nxw, nyw, nzw):
    nx, ny, nz = vs3d.shape
    xp, yp, zp = checker_pattern(nx, ny, nz, nxw, nyw, nzw)
    amp = xp[:, None] * yp[None, :] * pert
    return vs3d * (1.0 + amp[:, :, None] * zp[None, None, :])


def grf_perturbation(rng, nx, ny, nz, dx_km, dz_km, corr_km, amp):
    """Gaussian random field: white noise filtered by a Gaussian of correlation
    length corr_km, scaled to unit std, times amp, clipped to +-amp."""
    w = rng.standard_normal((nx, ny, nz))
    kx = np.fft.fftfreq(nx, d=dx_km)[:, None, None]
    ky = np.fft.fftfreq(ny, d=dx_km)[None, :, None]
    kz = np.fft.fftfreq(nz, d=dz_km)[None, None, :]
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2) * corr_km ** 2)
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    f /= f.std()
    return np.clip(f * amp / 2.0, -amp, amp)


def config1(seed=1001):
    """Checkerboard forward case: 41x41x30 at 0.05 deg, 10 periods 4-40 s,
    25 stations as sources and receivers (250 solves)."""
    rng = np.random.default_rng(seed)
    xx, yy = _grid(102.0, 24.0, (41, 41), 0.05)
    z = np.arange(0.0, 58.0 + 1e-9, 2.0)
    vs0 = gradient_model(41, 41, z)
    vs = add_checker(vs0, 0.08, 2, 3, 2)
    periods = np.geomspace(4.0, 40.0, 10)
    stlo, stla = _stations(rng, xx, yy, 25)
    evlo, evla, iper, ptr, idx = _all_pairs_events(stlo, stla, periods.size)
    tt = np.zeros(idx.size)
    return Workload("C1 checkerboard 41x41x30, 10 periods, 250 solves", xx, yy, z, vs, periods,
                    stlo, stla, evlo, evla, iper, ptr, idx, tt, np.ones(idx.size),
                    meta=dict(vs_start=vs0))


def config3(seed=1003, nsta=400, nper=20, n=301):
    """Batched case: 301x301x40 at 0.01 deg, GRF +-6 % (15 km) on the gradient,
    400 stations, 20 periods 2-50 s: 8000 forward + adjoint solves.
    Observed times are straight-ray times at a per-period reference velocity
    with 2 % seeded noise."""
    rng = np.random.default_rng(seed)
    xx, yy = _grid(102.0, 24.0, (n, n), 0.01)
    z = np.arange(0.0, 78.0 + 1e-9, 2.0)
    vs0 = gradient_model(n, n, z)
    dx_km = 0.01 * np.pi / 180.0 * R_EARTH
    vs = vs0 * (1.0 + grf_perturbation(rng, n, n, z.size, dx_km, 2.0, 15.0, 0.06))
    periods = np.geomspace(2.0, 50.0, nper)
    stlo, stla = _stations(rng, xx, yy, nsta)
    evlo, evla, iper, ptr, idx = _all_pairs_events(stlo, stla, nper)
    cref = 2.9 + 0.9 * (np.log(periods) - np.log(2.0)) / (np.log(50.0) - np.log(2.0))
    ev_src = np.repeat(np.arange(nsta), nper)
    src_of_rec = np.repeat(ev_src, np.diff(ptr))
    per_of_rec = np.repeat(iper, np.diff(ptr))
    d = _gc_km(stlo[src_of_rec], stla[src_of_rec], stlo[idx], stla[idx])
    tt = d / cref[per_of_rec] * (1.0 + 0.02 * rng.standard_normal(idx.size))
    return Workload(f"C3 batched {n}x{n}x{z.size}, {nper} periods, {nsta} stations, "
                    f"{nsta * nper} solves", xx, yy, z, vs, periods, stlo, stla, evlo, evla,
                    iper, ptr, idx, tt, np.ones(idx.size), meta=dict(vs_start=vs0))


def config5(seed=1005, nsta=1000, nper=30, n=601):
    """Full-inversion case: 601x601x50 at 0.005 deg (0-98 km), GRF +-6 %
    (15 km) on the gradient, 1000 stations, 30 periods 1-60 s: 30000 forward +
    adjoint solves per misfit gradient.  tt_obs are straight-ray times at a
    per-period reference velocity (the inversion benchmark replaces them with
    the engine's synthetic times in the GRF model)."""
    rng = np.random.default_rng(seed)
    xx, yy = _grid(102.0, 24.0, (n, n), 0.005)
    z = np.arange(0.0, 98.0 + 1e-9, 2.0)
    vs0 = gradient_model(n, n, z)
    dx_km = 0.005 * np.pi / 180.0 * R_EARTH
    vs = vs0 * (1.0 + grf_perturbation(rng, n, n, z.size, dx_km, 2.0, 15.0, 0.06))
    periods = np.geomspace(1.0, 60.0, nper)
    stlo, stla = _stations(rng, xx, yy, nsta)
    evlo, evla, iper, ptr, idx = _all_pairs_events(stlo, stla, nper)
    cref = 2.9 + 0.9 * (np.log(periods) - np.log(1.0)) / (np.log(60.0) - np.log(1.0))
    src_of_rec = np.repeat(np.repeat(np.arange(nsta), nper), np.diff(ptr))
    per_of_rec = np.repeat(iper, np.diff(ptr))
    d = _gc_km(stlo[src_of_rec], stla[src_of_rec], stlo[idx], stla[idx])
    tt = d / cref[per_of_rec]
    return Workload(f"C5 inversion {n}x{n}x{z.size}, {nper} periods, {nsta} stations, "
                    f"{nsta * nper} solves per gradient", xx, yy, z, vs, periods, stlo, stla,
                    evlo, evla, iper, ptr, idx, tt, np.ones(idx.size), meta=dict(vs_start=vs0))


def fractal_topography(rng, lon, lat, relief_km=4.0, slope=-2.0):
    """Seeded fractal surface on a lon/lat grid: power spectrum ~ k^slope
    (FFT-filtered white noise), scaled to [0, relief_km].  Returns (nlat, nlon)."""
    nlat, nlon = lat.size, lon.size
    noise = rng.standard_normal((nlat, nlon))
    ky = np.fft.fftfreq(nlat)[:, None]
    kx = np.fft.fftfreq(nlon)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (slope / 2.0)
    amp[0, 0] = 0.0
    z = np.real(np.fft.ifft2(np.fft.fft2(noise) * amp))
    z = (z - z.min()) / (z.max() - z.min())
    return relief_km * z


def config4(level=101, seed=1004, nsta=601, nper=15, lam=40.0, src_range=(50, 600),
            span_deg=2.0, wavelen_factor=2.5):
    """Topography case: level x level grid over a fixed span (101, 201 or 401
    nodes), fractal topography with 0-4 km relief and spectral slope -2, 15
    periods 4-40 s; per period a U{50..600} set of sources, each with a
    Poisson(lam) set of receivers (capped at nsta - 1).  The raw topography
    (0.005 deg, a margin beyond the model) is in meta["topo_raw"]."""
    rng = np.random.default_rng(seed)
    d = span_deg / (level - 1)
    xx, yy = _grid(102.0, 24.0, (level, level), d)
    z = np.arange(0.0, 58.0 + 1e-9, 2.0)
    vs = add_checker(gradient_model(level, level, z), 0.05, 2, 2, 2)
    periods = np.geomspace(4.0, 40.0, nper)
    stlo, stla = _stations(rng, xx, yy, nsta)
    evlo, evla, iper, ptr, idx = [], [], [], [0], []
    for ip in range(nper):
        ns = int(rng.integers(src_range[0], min(src_range[1], nsta) + 1))
        for s in rng.choice(nsta, size=ns, replace=False):
            nr = int(min(max(rng.poisson(lam), 1), nsta - 1))
            others = np.delete(np.arange(nsta), s)
            rec = np.sort(rng.choice(others, size=nr, replace=False))
            evlo.append(stlo[s])
            evla.append(stla[s])
            iper.append(ip)
            idx.extend(rec.tolist())
            ptr.append(len(idx))
    evlo, evla = np.array(evlo), np.array(evla)
    iper = np.array(iper, np.int32)
    ptr, idx = np.array(ptr, np.int32), np.array(idx, np.int32)
    cref = 2.9 + 0.9 * (np.log(periods) - np.log(4.0)) / (np.log(40.0) - np.log(4.0))
    ev_of = np.repeat(np.arange(evlo.size), np.diff(ptr))
    dist = _gc_km(evlo[ev_of], evla[ev_of], stlo[idx], stla[idx])
    tt = dist / cref[iper[ev_of]] * (1.0 + 0.02 * rng.standard_normal(idx.size))
    lon_raw = np.arange(101.8, 102.0 + span_deg + 0.2 + 1e-9, 0.005)
    lat_raw = np.arange(23.8, 24.0 + span_deg + 0.2 + 1e-9, 0.005)
    topo = fractal_topography(rng, lon_raw, lat_raw)
    return Workload(f"C4 topography {level}x{level}x{z.size}, {nper} periods, "
                    f"{evlo.size} solves", xx, yy, z, vs, periods, stlo, stla, evlo, evla, iper,
                    ptr, idx, tt, np.ones(idx.size),
                    meta=dict(topo_raw=(lon_raw, lat_raw, topo), wavelen_factor=wavelen_factor,
                              vs1d=vs.mean(axis=(0, 1))))


def _gc_km(lo1, la1, lo2, la2):
    r = np.pi / 180.0
    c = (np.sin(la1 * r) * np.sin(la2 * r)
         + np.cos(la1 * r) * np.cos(la2 * r) * np.cos((lo1 - lo2) * r))
    return np.arccos(np.clip(c, -1, 1)) * R_EARTH


def subset_events(w: Workload, keep) -> Workload:
    """Workload restricted to the events in ``keep`` (indices), receivers kept."""
    keep = np.asarray(keep)
    ptr = w.rec_ptr
    idx, tt, wt, newptr = [], [], [], [0]
    for e in keep:
        a, b = ptr[e], ptr[e + 1]
        idx.append(w.rec_idx[a:b])
        tt.append(w.tt_obs[a:b])
        wt.append(w.weight[a:b])
        newptr.append(newptr[-1] + (b - a))
    cat = (lambda v, dt: np.concatenate(v).astype(dt) if v else np.zeros(0, dt))
    return Workload(w.name + f" [subset {keep.size} events]", w.xx_deg, w.yy_deg, w.zgrid,
                    w.vs3d, w.periods, w.stlo, w.stla, w.evlo[keep], w.evla[keep],
                    w.iper[keep], np.array(newptr, np.int32), cat(idx, np.int32),
                    cat(tt, np.float64), cat(wt, np.float64), w.m11, w.m12, w.m22,
                    dict(w.meta))
