// Dispersion and depth-kernel kernels: surfdisp96 per surface column,
// sregn96_hti depth kernels per (column, period), the kernel combination of
// preproc::combine_kernels, and the host-side layer constants.  Compiled with
// -fmad=false (see surfker_dev.cuh).
// Out of line here, to shrink the instruction footprint: the eigenfunction
// routines and the complex division (the depth kernel 77 -> 72 -> 68 ms on
// C3) and dltar4 (the dispersion 141 -> 103 ms).  var, nevill and getsol stay inline (out of line on top of
// dltar4 they cost more in calls than they save: 107 / 137 / 179 ms).
#ifndef SK_NOINLINE_EIG
#define SK_NOINLINE_EIG __noinline__
#endif
#ifndef SK_ATTR_DLTAR4
#define SK_ATTR_DLTAR4 __noinline__
#endif
#ifndef SK_CDIV_ATTR
#define SK_CDIV_ATTR __noinline__
#endif
#include "surfker_dev.cuh"
#include "surfatt_gpu.h"

#include <algorithm>

namespace sa {

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
using sk::LayerConst;

// SurfGrid::fwdsurf per column (src/surf_grid.cpp:194-245): one thread per
// column, periods sequential (surfdisp96's bracket warm start).
// Resident 64-thread blocks per SM the register allocation is sized for.
// These kernels are latency-bound FP64 code with per-thread layer arrays in
// local memory: 10 blocks (96 registers, a few hundred bytes of spills) run
// the C3 dispersion 1.5x and the depth kernels 1.2x faster than the
// unconstrained allocation (128 / 202 registers), and put the 90,601 C3
// columns in one wave.
// Grids with more columns than one wave at 10 blocks per SM take the
// 16-block form (64 registers, a few more spills): with several waves the
// extra warps hide more FP64 latency (C5, 361,201 columns: 700 -> 659 ms),
// while a one-wave grid gains no warps and only pays the spills (C3: 122 ->
// 134 ms).  Both forms compute the same bits.
template <int MINB>
__global__ void __launch_bounds__(64, MINB)
surfdisp_columns_kernel(int nx, int ny, int nz, const double* __restrict__ vs3d, int nper,
                        const double* __restrict__ periods, int iflsph, int iwave, int igr,
                        const LayerConst* __restrict__ Lp, double* svel, int* status) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= nx * ny) return;
    const LayerConst& L = *Lp;
    const int ix = col / ny, iy = col % ny;
    float vp[sk::MMAX], vs[sk::MMAX], rho[sk::MMAX];
    sk::column_model(vs3d + (size_t)col * nz, nz, L, vp, vs, rho);
    double t[sk::KMAX], cg[sk::KMAX];
    for (int i = 0; i < nper; i++) {
        t[i] = periods[i];
        cg[i] = 0.0;
    }
    // SK_DISP_SERIAL builds the searches in the Fortran's call structure
    // (same bits; 1.2-1.3x slower, lanes diverge across the call sites)
#ifdef SK_DISP_SERIAL
    const int st = sk::surfdisp96(L, vp, vs, rho, iflsph, iwave, 1, igr, nper, t, cg);
#else
    const int st = sk::surfdisp96_lockstep(L, vp, vs, rho, iflsph, iwave, igr, nper, t, cg);
#endif
    if (status) status[ix + nx * iy] = st;
    for (int ip = 0; ip < nper; ip++) svel[(size_t)ip * nx * ny + ix + (size_t)nx * iy] = cg[ip];
}

// The correctly rounded transcendentals on device arrays (sa_math_eval):
// f = 0 exp, 1 log, 2 sin, 3 cos, 4 sincos (y holds sin, cos pairs), 5
// x^-3; exp,
// log and sincos through the same out-of-line routines the kernels call.
__global__ void math_eval_kernel(int f, size_t n, const double* __restrict__ x,
                                 double* __restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double v = x[i];
        switch (f) {
            case 0: y[i] = sk::sk_exp(v); break;
            case 1: y[i] = sk::sk_log(v); break;
            case 2: y[i] = cr::sin(v); break;
            case 3: y[i] = cr::cos(v); break;
            case 5: y[i] = cr::pow_m3(v); break;
            default: sk::sk_sincos(v, &y[2 * i], &y[2 * i + 1]); break;
        }
    }
}

// SurfGrid::compute_dispersion_kernel (src/surf_grid.cpp:247-305) through
// depthkernelHTI1d (src/surfdisp.cpp:481-547): one thread per (column, period)
// runs sregn96_hti at the column's phase velocity cp.
__global__ void SK_DEPTH_BOUNDS
depthkernel_kernel(int nx, int ny, int nz, const double* __restrict__ vs3d, int nper,
                   const double* __restrict__ periods, const double* __restrict__ cp_plane,
                   const LayerConst* __restrict__ Lp, double* sen_vs, double* sen_vp,
                   double* sen_rho, double* sen_hs) {
    long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool live = gid < (long long)nx * ny * nper;
    if (!live) {
        if (SK_DEPTH_PHASED == 0) return;
        gid = (long long)nx * ny * nper - 1;   // meets the barriers, stores nothing
    }
    // period-major: a warp takes 32 neighbouring columns at one period, whose
    // phase velocities stand alike against the layer velocities, so its lanes
    // take the same evanescent / oscillatory branches layer by layer
    const long long ncol = (long long)nx * ny;
    const int ip = (int)(gid / ncol);
    const int col = (int)(gid % ncol);
    const int ix = col / ny, iy = col % ny;
    const LayerConst& L = *Lp;
    float vp[sk::MMAX], vs[sk::MMAX], rho[sk::MMAX];
    sk::column_model(vs3d + (size_t)col * nz, nz, L, vp, vs, rho);
    sk::RW W;
    const int mmax = L.mmax;
    W.mmax = mmax;
    W.allfluid = true;
    for (int i = 0; i < mmax; i++) {
        W.zb[i] = vs[i];
        W.za[i] = vp[i];
        W.zrho[i] = rho[i];
        W.zd[i] = L.thk[i];
        W.iwat[i] = (W.zb[i] > 0.0) ? 0 : 1;
        if (W.zb[i] > 0.0) W.allfluid = false;
    }
    // bldsph (sregn96.f90:129-183), per-layer factors from the host
    for (int i = 0; i < mmax; i++) {
        W.za[i] = W.za[i] * L.rg_vtp[i];
        W.zb[i] = W.zb[i] * L.rg_vtp[i];
        W.zrho[i] = W.zrho[i] * L.rg_rtp[i];
        W.zd[i] = L.rg_zd[i];
    }
    for (int i = 0; i < mmax; i++) {
        W.xmu[i] = W.zrho[i] * (W.zb[i] * W.zb[i]);
        W.xlam[i] = W.zrho[i] * (W.za[i] * W.za[i]) - 2.0 * W.xmu[i];
    }
    const double pi = 3.1415926535897932384626433832795;
    const double twopi = 2.0 * pi;
    const double omega = twopi / periods[ip];
    double c = cp_plane[(size_t)ip * nx * ny + ix + (size_t)nx * iy];
    const double wvno = omega / c;
    sk::svfunc_phased(W, omega, wvno);
    double ugr, fac;
    sk::energy(W, omega, wvno, ugr, fac);
    if (!live) return;
    if (fabs(c) < 1.0e-36) c = 0.0;
    // sprayl (sregn96.f90:1592-1638): only the velocity and density kernels
    // are returned here
    const double ar = 6371.0;
    const double r = c / (2.0 * ar * omega);
    const double tm = sqrt(1.0 + r * r);
    const double tm3 = (tm * tm) * tm;
    for (int k = 0; k < nz; k++) {
        const size_t i4 = ((size_t)col * nz + k) * nper + ip;
        sen_vs[i4] = W.dcdb[k] * L.rg_vtp[k] / tm3;
        sen_vp[i4] = W.dcda[k] * L.rg_vtp[k] / tm3;
        sen_rho[i4] = W.dcdr[k] * L.rg_rtp[k] / tm3;
    }
    // the half-space layer (index nz), which the reference drops: its
    // velocities are the deepest node's, so a derivative with respect to that
    // node includes it.  Optional, [(col * nper + ip) * 3 + {vs, vp, rho}].
    if (sen_hs) {
        double* h = sen_hs + ((size_t)col * nper + ip) * 3;
        h[0] = W.dcdb[nz] * L.rg_vtp[nz] / tm3;
        h[1] = W.dcda[nz] * L.rg_vtp[nz] / tm3;
        h[2] = W.dcdr[nz] * L.rg_rtp[nz] / tm3;
    }
}

// Love-wave depth kernels, one thread per (column, period):
// surfker::depthkernel_love_phase (src/surfdisp.cpp:295-349) through slegn96
// (src/surfker/slegn96.f90:672-783) when igr = 0, depthkernel_love_group
// (:351-426) through slegnpu (:785-919) when igr = 1 (phase velocities at t,
// t1 = t(1 + 0.005), t2 = t(1 - 0.005) from cp, cp1, cp2).  sen_vs = dc/db
// (du/db), sen_rho = dc/drho (du/drho) of the first nz layers,
// earth-flattening corrected (splove, :631-670).  Models without water.
__global__ void SK_DEPTH_BOUNDS
depthkernel_love_kernel(int nx, int ny, int nz, const double* __restrict__ vs3d, int nper,
                        const double* __restrict__ periods, const double* __restrict__ p1,
                        const double* __restrict__ p2, const double* __restrict__ cp_plane,
                        const double* __restrict__ cp1_plane,
                        const double* __restrict__ cp2_plane, int igr,
                        const LayerConst* __restrict__ Lp, double* sen_vs, double* sen_rho) {
    long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool live = gid < (long long)nx * ny * nper;
    if (!live) {
        if (SK_DEPTH_PHASED == 0) return;
        gid = (long long)nx * ny * nper - 1;   // meets the barriers, stores nothing
    }
    // period-major: a warp takes 32 neighbouring columns at one period, whose
    // phase velocities stand alike against the layer velocities, so its lanes
    // take the same evanescent / oscillatory branches layer by layer
    const long long ncol = (long long)nx * ny;
    const int ip = (int)(gid / ncol);
    const int col = (int)(gid % ncol);
    const int ix = col / ny, iy = col % ny;
    const LayerConst& L = *Lp;
    float vp[sk::MMAX], vs[sk::MMAX], rho[sk::MMAX];
    sk::column_model(vs3d + (size_t)col * nz, nz, L, vp, vs, rho);
    sk::LW W;
    sk::lv_model(W, vs, rho, L);
    const double twopi = 2.0 * sk::kLovePiF;
    const double ar = 6371.0;
    const size_t pix = (size_t)ip * nx * ny + ix + (size_t)nx * iy;
    const double t = periods[ip], cp = cp_plane[pix];
    double omega = twopi / t;
    SK_PHASE();
    sk::lv_shfunc(W, omega, omega / cp);
    SK_PHASE();
    sk::lv_energy(W, omega, omega / cp);
    if (!igr) {
        if (!live) return;
        const double x = (3.0 * cp) / ((2.0 * ar) * omega);
        const double tm = sqrt(1.0 + x * x);
        const double tm3 = tm * tm * tm;
        for (int k = 0; k < nz; k++) {
            const size_t i4 = ((size_t)col * nz + k) * nper + ip;
            sen_vs[i4] = W.dcdb[k] * L.rg_vtp[k] / tm3;
            sen_rho[i4] = W.dcdr[k] * L.lv_rtp[k] / tm3;
        }
        return;
    }
    const double cg = W.ugr;
    double b0[sk::MMAX], r0[sk::MMAX], b1[sk::MMAX], r1[sk::MMAX];
    for (int k = 0; k < nz; k++) {
        b0[k] = W.dcdb[k];
        r0[k] = W.dcdr[k];
    }
    const double t1 = p1[ip], t2 = p2[ip];
    omega = twopi / t1;
    const double c1 = cp1_plane[pix];
    SK_PHASE();
    sk::lv_shfunc(W, omega, omega / c1);
    SK_PHASE();
    sk::lv_energy(W, omega, omega / c1);
    for (int k = 0; k < nz; k++) {
        b1[k] = W.dcdb[k];
        r1[k] = W.dcdr[k];
    }
    omega = twopi / t2;
    const double c2 = cp2_plane[pix];
    SK_PHASE();
    sk::lv_shfunc(W, omega, omega / c2);
    SK_PHASE();
    sk::lv_energy(W, omega, omega / c2);   // W.dc* now hold this evaluation
    if (!live) return;
    const double uc1 = cg / cp;
    omega = twopi / t;
    const double x = (3.0 * cp) / ((2.0 * ar) * omega);
    const double tm = sqrt(1.0 + x * x);
    const double y = 1.5 / (ar * omega);
    const double tm1 = (y * y) / tm;
    for (int k = 0; k < nz; k++) {
        const double dub = uc1 * (2.0 - uc1) * W.dcdb[k] - uc1 * uc1 * t * (W.dcdb[k] - b1[k]) / (t2 - t1);
        const double dur = uc1 * (2.0 - uc1) * W.dcdr[k] - uc1 * uc1 * t * (W.dcdr[k] - r1[k]) / (t2 - t1);
        const size_t i4 = ((size_t)col * nz + k) * nper + ip;
        sen_vs[i4] = (tm * dub + cg * cp * b0[k] * tm1) * L.rg_vtp[k];
        sen_rho[i4] = (tm * dur + cg * cp * r0[k] * tm1) * L.lv_rtp[k];
    }
}

cudaError_t launch_depthkernel_love(int nx, int ny, int nz, const double* vs3d, int nper,
                                    const double* periods, const double* p1, const double* p2,
                                    const double* cp, const double* cp1, const double* cp2,
                                    int igr, const void* layer_const, double* sen_vs,
                                    double* sen_rho, cudaStream_t st) {
    const long long n = (long long)nx * ny * nper;
    depthkernel_love_kernel<<<(unsigned)((n + SK_DEPTH_BLOCK - 1) / SK_DEPTH_BLOCK), SK_DEPTH_BLOCK, 0,
                              st>>>(
        nx, ny, nz, vs3d, nper, periods, p1, p2, cp, cp1, cp2, igr,
        reinterpret_cast<const LayerConst*>(layer_const), sen_vs, sen_rho);
    return cudaGetLastError();
}

// preproc::combine_kernels, vs-only branch (src/preproc.cpp:276-304): one
// thread per (ix, iy, k), periods accumulated in order from zero.
__global__ void combine_vs_kernel(int nx, int ny, int nz, int nper, const double* __restrict__ adj_s,
                                  const double* __restrict__ vs3d, const double* __restrict__ vp3d,
                                  const double* __restrict__ sen_vs,
                                  const double* __restrict__ sen_vp,
                                  const double* __restrict__ sen_rho, double* ker_vs) {
    const size_t i3 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i3 >= (size_t)nx * ny * nz) return;
    const int col = (int)(i3 / nz);
    const int ix = col / ny, iy = col % ny;
    const double vs = vs3d[i3];
    // vp3d NULL: vp = vs2vp(vs), as ModelGrid keeps it for vs-only
    // parametrisations (src/model_grid.cpp:594-596)
    const double vp = vp3d ? vp3d[i3] : sk::vs2vp(vs);
    const double dab = sk::dalpha_dbeta(vs);
    const double dra = sk::drho_dalpha(vp);
    double k = 0.0;
    for (int ip = 0; ip < nper; ip++) {
        const double att = adj_s[(size_t)ip * nx * ny + ix + (size_t)nx * iy];
        const size_t i4 = i3 * nper + ip;
        k -= att * (sen_vs[i4] + sen_vp[i4] * dab + sen_rho[i4] * dra * dab);
    }
    ker_vs[i3] = k;
}

// The vs gradient as a derivative (no counterpart in the reference, whose
// combine_kernels above is an area density built from dimensionless
// kernels): per (ix, iy, k)
//   g = -sum_iper adj_s * dA(iy) * dc/dvs,
//   dc/dvs = K_b / b + K_a / a * da/db + (K_r' / rho) * drho/da * da/db,
// with K_b, K_a, K_r the sregn96 outputs (b dc/db, a dc/da and its density
// kernel), dA = dx R cos(lat) dy R the cell area (the adjoint source is
// divided by it, src/eikonal_solver.cpp:366-367), and K_r' = rho dc/drho:
// sregn96's dcdr carries the flattened velocities once more on its elastic
// terms (src/surfker/sregn96.f90:1132, :1176, where facah, facav, facbv are
// already a dc/da and b dc/db), so K_r' = K_r - (rtp/vtp)/2 *
// ((a_f - 1) K_a + (b_f - 1) K_b), a_f, b_f the flattened velocities.  The
// deepest node also takes the half-space layer's terms (sen_hs).
__device__ inline double dcdvs_term(double kb, double ka, double kr, double vs, double vp,
                                    double rho, double dab, double dra, double vtp, double rtp) {
    const double af = vp * vtp, bf = vs * vtp;
    const double krho = kr - 0.5 * (rtp / vtp) * ((af - 1.0) * ka + (bf - 1.0) * kb);
    return kb / vs + ka / vp * dab + krho / rho * dra * dab;
}

__global__ void combine_vs_derivative_kernel(int nx, int ny, int nz, int nper,
                                             const double* __restrict__ adj_s,
                                             const double* __restrict__ vs3d,
                                             const double* __restrict__ vp3d,
                                             const double* __restrict__ sen_vs,
                                             const double* __restrict__ sen_vp,
                                             const double* __restrict__ sen_rho,
                                             const double* __restrict__ sen_hs,
                                             const double* __restrict__ area_row,
                                             const LayerConst* __restrict__ Lp, double* grad) {
    const size_t i3 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i3 >= (size_t)nx * ny * nz) return;
    const LayerConst& L = *Lp;
    const int col = (int)(i3 / nz);
    const int k = (int)(i3 % nz);
    const int ix = col / ny, iy = col % ny;
    const double vs = vs3d[i3];
    const double vp = vp3d ? vp3d[i3] : sk::vs2vp(vs);
    const double rho = sk::vp2rho(vp);
    const double dab = sk::dalpha_dbeta(vs);
    const double dra = sk::drho_dalpha(vp);
    double g = 0.0;
    for (int ip = 0; ip < nper; ip++) {
        const double att = adj_s[(size_t)ip * nx * ny + ix + (size_t)nx * iy];
        const size_t i4 = i3 * nper + ip;
        double d = dcdvs_term(sen_vs[i4], sen_vp[i4], sen_rho[i4], vs, vp, rho, dab, dra,
                              L.rg_vtp[k], L.rg_rtp[k]);
        if (k == nz - 1 && sen_hs) {
            const double* h = sen_hs + ((size_t)col * nper + ip) * 3;
            d += dcdvs_term(h[0], h[1], h[2], vs, vp, rho, dab, dra, L.rg_vtp[nz], L.rg_rtp[nz]);
        }
        g -= att * area_row[iy] * d;
    }
    grad[i3] = g;
}

// Exact dc/dvs of every node (no reference counterpart): one thread per
// (column, period); the derivatives of surfdisp96's Rayleigh phase-velocity
// root c (from the svel plane) with respect to each flattened layer's b, a,
// rho (sk::root_dcdm), chained through the flattening (b_f = vs tmp, a_f =
// vp tmp, rho_f = rho rhofac, sphere of surfdisp96.f:502-574) and the
// Brocher relations (vp(vs), rho(vp)); the half-space layer, a copy of the
// deepest node, adds to that node.  dcdvs [(col * nz + k) * nper + ip].
__global__ void __launch_bounds__(64)
dispersion_dcdvs_kernel(int nx, int ny, int nz, const double* __restrict__ vs3d, int nper,
                        const double* __restrict__ periods, const double* __restrict__ svel,
                        const LayerConst* __restrict__ Lp, double* dcdvs) {
    const long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (gid >= (long long)nx * ny * nper) return;
    // period-major: a warp takes 32 neighbouring columns at one period, whose
    // phase velocities stand alike against the layer velocities, so its lanes
    // take the same evanescent / oscillatory branches layer by layer
    const long long ncol = (long long)nx * ny;
    const int ip = (int)(gid / ncol);
    const int col = (int)(gid % ncol);
    const int ix = col / ny, iy = col % ny;
    const LayerConst& L = *Lp;
    float vp[sk::MMAX], vs[sk::MMAX], rho[sk::MMAX];
    const double* v1 = vs3d + (size_t)col * nz;
    sk::column_model(v1, nz, L, vp, vs, rho);
    sk::SDModel M;
    const int mmax = L.mmax;
    M.mmax = mmax;
    M.llw = 1;
    for (int i = 0; i < mmax; i++) {
        M.d[i] = L.sd_d[i];
        M.a[i] = (float)(vp[i] * L.sd_tmp[i]);
        M.b[i] = (float)(vs[i] * L.sd_tmp[i]);
        M.rho[i] = rho[i] * L.sd_rhofac[i];
    }
    M.del1st = 0.0;
    double ein[5 * sk::MMAX], logn[sk::MMAX], db[sk::MMAX], da[sk::MMAX], dr[sk::MMAX];
    const double c = svel[(size_t)ip * nx * ny + ix + (size_t)nx * iy];
    sk::root_dcdm(M, periods[ip], c, db, da, dr, ein, logn);
    for (int k = 0; k < nz; k++) {
        const double b = v1[k];
        const double a = sk::vs2vp(b);
        const double dab = sk::dalpha_dbeta(b), dra = sk::drho_dalpha(a);
        auto node = [&](int m) {
            return db[m] * L.sd_tmp[m] + da[m] * L.sd_tmp[m] * dab
                   + dr[m] * (double)L.sd_rhofac[m] * dra * dab;
        };
        double d = node(k);
        if (k == nz - 1) d += node(nz);
        dcdvs[((size_t)col * nz + k) * nper + ip] = d;
    }
}

// grad(ix, iy, k) = sum_iper dchi/dsvel(iper, iy, ix) * dc/dvs(ix, iy, k, iper),
// periods in order.
__global__ void combine_exact_kernel(int nx, int ny, int nz, int nper,
                                     const double* __restrict__ dchi_dsvel,
                                     const double* __restrict__ dcdvs, double* grad) {
    const size_t i3 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i3 >= (size_t)nx * ny * nz) return;
    const int col = (int)(i3 / nz);
    const int ix = col / ny, iy = col % ny;
    double g = 0.0;
    for (int ip = 0; ip < nper; ip++)
        g += dchi_dsvel[(size_t)ip * nx * ny + ix + (size_t)nx * iy] * dcdvs[i3 * nper + ip];
    grad[i3] = g;
}

cudaError_t launch_dispersion_dcdvs(int nx, int ny, int nz, const double* vs3d, int nper,
                                    const double* periods, const double* svel,
                                    const void* layer_const, double* dcdvs, cudaStream_t st) {
    const long long n = (long long)nx * ny * nper;
    dispersion_dcdvs_kernel<<<(unsigned)((n + 63) / 64), 64, 0, st>>>(
        nx, ny, nz, vs3d, nper, periods, svel, reinterpret_cast<const LayerConst*>(layer_const),
        dcdvs);
    return cudaGetLastError();
}

cudaError_t launch_combine_exact(int nx, int ny, int nz, int nper, const double* dchi_dsvel,
                                 const double* dcdvs, double* grad, cudaStream_t st) {
    const size_t n = (size_t)nx * ny * nz;
    combine_exact_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(nx, ny, nz, nper,
                                                                       dchi_dsvel, dcdvs, grad);
    return cudaGetLastError();
}

cudaError_t launch_combine_vs_derivative(int nx, int ny, int nz, int nper, const double* adj_s,
                                         const double* vs3d, const double* vp3d,
                                         const double* sen_vs, const double* sen_vp,
                                         const double* sen_rho, const double* sen_hs,
                                         const double* area_row, const void* layer_const,
                                         double* grad, cudaStream_t st) {
    const size_t n = (size_t)nx * ny * nz;
    combine_vs_derivative_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
        nx, ny, nz, nper, adj_s, vs3d, vp3d, sen_vs, sen_vp, sen_rho, sen_hs, area_row,
        reinterpret_cast<const LayerConst*>(layer_const), grad);
    return cudaGetLastError();
}

cudaError_t launch_surfdisp_columns(int nx, int ny, int nz, const double* vs3d, int nper,
                                    const double* periods, int iflsph, int iwave, int igr,
                                    const void* layer_const, double* svel, int* status,
                                    cudaStream_t st) {
    const int n = nx * ny;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const LayerConst* Lp = reinterpret_cast<const LayerConst*>(layer_const);
    if (n > nsm * 10 * 64)
        surfdisp_columns_kernel<16><<<(n + 63) / 64, 64, 0, st>>>(
            nx, ny, nz, vs3d, nper, periods, iflsph, iwave, igr, Lp, svel, status);
    else
        surfdisp_columns_kernel<10><<<(n + 63) / 64, 64, 0, st>>>(
            nx, ny, nz, vs3d, nper, periods, iflsph, iwave, igr, Lp, svel, status);
    return cudaGetLastError();
}

cudaError_t launch_depthkernel(int nx, int ny, int nz, const double* vs3d, int nper,
                               const double* periods, const double* cp, const void* layer_const,
                               double* sen_vs, double* sen_vp, double* sen_rho, cudaStream_t st,
                               double* sen_hs) {
    const long long n = (long long)nx * ny * nper;
    depthkernel_kernel<<<(unsigned)((n + SK_DEPTH_BLOCK - 1) / SK_DEPTH_BLOCK), SK_DEPTH_BLOCK, 0, st>>>(
        nx, ny, nz, vs3d, nper, periods, cp, reinterpret_cast<const LayerConst*>(layer_const),
        sen_vs, sen_vp, sen_rho, sen_hs);
    return cudaGetLastError();
}

cudaError_t launch_combine_vs(int nx, int ny, int nz, int nper, const double* adj_s,
                              const double* vs3d, const double* vp3d, const double* sen_vs,
                              const double* sen_vp, const double* sen_rho, double* ker_vs,
                              cudaStream_t st) {
    const size_t n = (size_t)nx * ny * nz;
    combine_vs_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        nx, ny, nz, nper, adj_s, vs3d, vp3d, sen_vs, sen_vp, sen_rho, ker_vs);
    return cudaGetLastError();
}

size_t layer_const_bytes() { return sizeof(LayerConst); }

// Host: the per-layer earth-flattening constants (C library arithmetic).
int build_layer_const(int nz, const double* zgrid, void* out) {
    LayerConst& L = *reinterpret_cast<LayerConst*>(out);
    const int mmax = nz + 1;
    if (mmax > sk::MMAX || nz < 1) return -1;
    L.mmax = mmax;
    // thickness (src/surfdisp.cpp:91-102)
    double thk[sk::MMAX];
    for (int kk = 0; kk < nz; ++kk) {
        if (kk == nz - 1) thk[kk] = (nz > 1) ? thk[kk - 1] : 0.0;
        else thk[kk] = zgrid[kk + 1] - zgrid[kk];
    }
    thk[mmax - 1] = 0.0;
    for (int i = 0; i < mmax; i++) L.thk[i] = (float)thk[i];
    // surfdisp96 sphere(0,0) and the Rayleigh/Love density factors
    {
        float d[sk::MMAX];
        for (int i = 0; i < mmax; i++) d[i] = L.thk[i];
        d[mmax - 1] = 1.0f;
        const double ar = 6370.0;
        double dr = 0.0, r0 = ar;
        for (int i = 0; i < mmax; i++) {
            dr = dr + (double)d[i];
            const double r1 = ar - dr;
            const double z0 = ar * std::log(ar / r0);
            const double z1 = ar * std::log(ar / r1);
            L.sd_d[i] = (float)(z1 - z0);
            const double tmp = (ar + ar) / (r0 + r1);
            L.sd_tmp[i] = tmp;
            const float btp = (float)tmp;
            L.sd_rhofac[i] = std::pow(btp, -2.275f);
            const float x2 = btp * btp, x3 = x2 * btp, x5 = x3 * x2;
            L.sd_rhofac_love[i] = 1.0f / x5;
            r0 = r1;
        }
        L.sd_d[mmax - 1] = 0.0f;
    }
    // sregn96 bldsph
    {
        const double ar = 6371.0;
        double dr = 0.0, r0 = ar;
        const double expo = (double)(-2.275f);
        for (int i = 1; i <= mmax; i++) {
            if (i == mmax) dr = dr + 1.0;
            else dr = dr + (double)L.thk[i - 1];
            const double r1 = ar - dr;
            const double z0 = ar * std::log(ar / r0);
            const double z1 = ar * std::log(ar / r1);
            const double tmp = (2.0 * ar) / (r0 + r1);
            L.rg_vtp[i - 1] = tmp;
            L.rg_rtp[i - 1] = std::pow(tmp, expo);
            // slegn96 bldsph: tmp**(-5) as gfortran expands it (x^3 x^2, inverse)
            const double x2 = tmp * tmp, x3 = x2 * tmp, x5 = x3 * x2;
            L.lv_rtp[i - 1] = 1.0 / x5;
            L.rg_dtp[i - 1] = ar / r0;
            L.rg_zd[i - 1] = z1 - z0;
            r0 = r1;
        }
        L.rg_zd[mmax - 1] = 0.0;
    }
    return 0;
}

}  // namespace sa

extern "C" int sa_math_eval(int f, size_t n, const double* x, double* y, void* stream) {
    if (f < 0 || f > 5 || (n > 0 && (!x || !y))) return SA_ERR_ARG;
    if (n == 0) return SA_OK;
    const int threads = 256;
    const size_t blocks = std::min<size_t>((n + threads - 1) / threads, 148 * 16);
    sa::math_eval_kernel<<<(unsigned)blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        f, n, x, y);
    return cudaGetLastError() == cudaSuccess ? SA_OK : SA_ERR_CUDA;
}
