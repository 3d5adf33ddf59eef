// Device routines of the dispersion and depth-kernel engine, shared by
// surfker.cu and surfker_group.cu.
//
// Dispersion and depth-kernel engine: surfdisp96 (Rayleigh/Love phase or
// group velocity root search) per surface column and sregn96_hti (Rayleigh
// eigenfunctions and depth kernels) per (column, period), plus the kernel
// combination of preproc::combine_kernels.
//
// Compiled with -fmad=false and IEEE division/sqrt: the FP64 and REAL*4
// arithmetic of src/surfker/surfdisp96.f and src/surfker/sregn96.f90 is kept
// operation for operation, including the REAL*4 islands (model arrays, gtsolh,
// sngl() arguments, default-kind literals).  exp, log, sin and cos are the
// correctly rounded ones of crmath.cuh, which agree with the C library the
// reference calls except where the C library itself misrounds (about 0.1 %
// of arguments); the layer flattening factors that involve REAL*4 powers are
// precomputed per layer on the host.
#pragma once
#include <cmath>

#include "crmath.cuh"
#include "launch.h"

namespace sa {
namespace sk {

constexpr int MMAX = 64;     // layers (nz + 1) supported per column
constexpr int KMAX = 64;     // periods per column

// Per-layer constants of the earth-flattening transforms.  They depend on
// the layer thicknesses only, which every column shares.
struct LayerConst {
    int mmax;
    // surfdisp96 sphere() (surfdisp96.f:502-574)
    float sd_d[MMAX];        // flattened thickness (d(mmax) = 0 afterwards)
    double sd_tmp[MMAX];     // velocity factor (ar+ar)/(r0+r1)
    float sd_rhofac[MMAX];   // btp**(-2.275) (Rayleigh), REAL*4 power
    float sd_rhofac_love[MMAX];  // btp**(-5) (Love)
    // sregn96 bldsph() (sregn96.f90:129-183)
    double rg_zd[MMAX];      // flattened thickness (zd(mmax) = 0)
    double rg_vtp[MMAX];
    double rg_rtp[MMAX];     // tmp**(-2.275), FP64 power
    double lv_rtp[MMAX];     // tmp**(-5) of slegn96's bldsph (Love density factor)
    double rg_dtp[MMAX];
    float thk[MMAX];         // unflattened float thickness (build_disp_req)
};

// Inlining of the routines reached from several call sites.  Each unit that
// includes this header picks per group: surfker.cu takes the transcendentals,
// dltar4, the eigenfunction routines and the complex division out of line
// (smaller instruction footprint, bit-identical results); surfker_group.cu
// keeps everything inline, because with layer_integrals out of line the
// group-velocity kernel's saved first-evaluation kernels come back
// overwritten on the device (see surfker_group.cu).  SK_NOINLINE marks the
// routines that stay inline everywhere
// (dltar1, nevill, getsol: out of line they cost more than they save).
#ifndef SK_NOINLINE
#define SK_NOINLINE inline
#endif
// The eigenfunction routines (varsv, dnka_rg, evalg, layer_integrals): out of
// line in surfker.cu (SK_NOINLINE_EIG set there), inline elsewhere.
#ifndef SK_NOINLINE_EIG
#define SK_NOINLINE_EIG inline
#endif
// dltar4: out of line in surfker.cu (SK_ATTR_DLTAR4 set there).
#ifndef SK_ATTR_DLTAR4
#define SK_ATTR_DLTAR4 inline
#endif

// One out-of-line copy each of the FP64 transcendentals.  The column kernels
// reach them from dozens of inlined call sites, and inline copies of the
// library routines made those kernels stall on instruction fetch
// (`no_instruction` about 8 cycles per issued instruction): out of line, the
// C3 dispersion runs 175 -> 141 ms with bit-identical results.  The group
// kernels (surfker_group.cu) keep them inline (SK_MATH_NOINLINE 0).
#ifndef SK_MATH_NOINLINE
#define SK_MATH_NOINLINE 1
#endif
#if SK_MATH_NOINLINE
#define SK_MATH_ATTR __noinline__
#else
#define SK_MATH_ATTR __forceinline__
#endif
static __device__ SK_MATH_ATTR void sk_sincos(double x, double* s, double* c) { cr::sincos(x, s, c); }
static __device__ SK_MATH_ATTR double sk_exp(double x) { return cr::exp(x); }
static __device__ SK_MATH_ATTR double sk_log(double x) { return cr::log(x); }

__device__ __forceinline__ double dsign1(double x) { return copysign(1.0, x); }

// Brocher relations, scalar forms (include/utils.h:185-187, :223-225)
__device__ __forceinline__ double vs2vp(double vs) {
    return 0.9409 + 2.0947 * vs - 0.8206 * vs * vs + 0.2683 * vs * vs * vs - 0.0251 * vs * vs * vs * vs;
}
__device__ __forceinline__ double vp2rho(double vp) {
    return 1.6612 * vp - 0.4721 * vp * vp + 0.0671 * vp * vp * vp - 0.0043 * vp * vp * vp * vp
         + 0.000106 * vp * vp * vp * vp * vp;
}
// include/utils.h:198-212
__device__ __forceinline__ double drho_dalpha(double vp) {
    return 1.6612 - 2 * 0.4721 * vp + 3 * 0.0671 * vp * vp - 4 * 0.0043 * vp * vp * vp
         + 5 * 0.000106 * vp * vp * vp * vp;
}
__device__ __forceinline__ double dalpha_dbeta(double vs) {
    return 2.0947 - 2 * 0.8206 * vs + 3 * 0.2683 * vs * vs - 4 * 0.0251 * vs * vs * vs;
}

// Float layer model of one column: build_disp_req (src/surfdisp.cpp:60-108)
// with the Brocher branch of SurfGrid::fwdsurf (src/surf_grid.cpp:214-226).
__device__ inline void column_model(const double* vs1d, int nz, const LayerConst& L, float* vp,
                                    float* vs, float* rho) {
    for (int kk = 0; kk < nz; ++kk) {
        const double b = vs1d[kk];
        const double a = vs2vp(b);
        const double r = vp2rho(a);
        vs[kk] = (float)b;
        vp[kk] = (float)a;
        rho[kk] = (float)r;
    }
    vs[nz] = vs[nz - 1];
    vp[nz] = vp[nz - 1];
    rho[nz] = rho[nz - 1];
}

// ---------------------------------------------------------------------------
// surfdisp96
// ---------------------------------------------------------------------------
struct SDModel {
    int mmax, llw;
    float d[MMAX], a[MMAX], b[MMAX], rho[MMAX];
    double del1st;
};

struct VarOut {
    double w, cosp, exa, a0, cpcq, cpy, cpz, cqw, cqx, xy, xz, wy, wz;
};

// surfdisp96.f:904-1021
__device__ inline VarOut var(double p, double q, double ra, double rb, double wvno, double xka,
                             double xkb, double dpth) {
    VarOut o;
    double pex = 0.0, sex = 0.0;
    double sinp = 0.0, w = 0.0, x = 0.0, cosp = 0.0;
    double sinq = 0.0, y = 0.0, z = 0.0, cosq = 0.0;
    if (wvno < xka) {
        sk_sincos(p, &sinp, &cosp);
        w = sinp / ra;
        x = -(ra * sinp);
    } else if (wvno == xka) {
        cosp = 1.0;
        w = dpth;
        x = 0.0;
    } else if (wvno > xka) {
        pex = p;
        double fac = 0.0;
        if (p < 16) fac = sk_exp(-2.0 * p);
        cosp = (1.0 + fac) * 0.5;
        sinp = (1.0 - fac) * 0.5;
        w = sinp / ra;
        x = ra * sinp;
    }
    if (wvno < xkb) {
        sk_sincos(q, &sinq, &cosq);
        y = sinq / rb;
        z = -(rb * sinq);
    } else if (wvno == xkb) {
        cosq = 1.0;
        y = dpth;
        z = 0.0;
    } else if (wvno > xkb) {
        sex = q;
        double fac = 0.0;
        if (q < 16) fac = sk_exp(-2.0 * q);
        cosq = (1.0 + fac) * 0.5;
        sinq = (1.0 - fac) * 0.5;
        y = sinq / rb;
        z = rb * sinq;
    }
    o.exa = pex + sex;
    o.a0 = 0.0;
    if (o.exa < 60.0) o.a0 = sk_exp(-o.exa);
    o.cpcq = cosp * cosq;
    o.cpy = cosp * y;
    o.cpz = cosp * z;
    o.cqw = cosq * w;
    o.cqx = cosq * x;
    o.xy = x * y;
    o.xz = x * z;
    o.wy = w * y;
    o.wz = w * z;
    o.w = w;
    o.cosp = cosp;
    return o;
}

// surfdisp96.f:1054-1098: the 5x5 compound layer matrix, ca[j][i] holding
// the Fortran ca(j+1, i+1).
__device__ inline void dnka_matrix(double ca[5][5], double wvno2, double gam, double gammk,
                                   double rho, const VarOut& v) {
    const double one = 1.0, two = 2.0;
    const double gamm1 = gam - one;
    const double twgm1 = gam + gamm1;
    const double gmgmk = gam * gammk;
    const double gmgm1 = gam * gamm1;
    const double gm1sq = gamm1 * gamm1;
    const double rho2 = rho * rho;
    const double a0pq = v.a0 - v.cpcq;
    ca[0][0] = v.cpcq - two * gmgm1 * a0pq - gmgmk * v.xz - wvno2 * gm1sq * v.wy;
    ca[0][1] = (wvno2 * v.cpy - v.cqx) / rho;
    ca[0][2] = -((twgm1 * a0pq + gammk * v.xz + wvno2 * gamm1 * v.wy) / rho);
    ca[0][3] = (v.cpz - wvno2 * v.cqw) / rho;
    ca[0][4] = -((two * wvno2 * a0pq + v.xz + wvno2 * wvno2 * v.wy) / rho2);
    ca[1][0] = (gmgmk * v.cpz - gm1sq * v.cqw) * rho;
    ca[1][1] = v.cpcq;
    ca[1][2] = gammk * v.cpz - gamm1 * v.cqw;
    ca[1][3] = -v.wz;
    ca[1][4] = ca[0][3];
    ca[3][0] = (gm1sq * v.cpy - gmgmk * v.cqx) * rho;
    ca[3][1] = -v.xy;
    ca[3][2] = gamm1 * v.cpy - gammk * v.cqx;
    ca[3][3] = ca[1][1];
    ca[3][4] = ca[0][1];
    ca[4][0] = -((two * gmgmk * gm1sq * a0pq + gmgmk * gmgmk * v.xz + gm1sq * gm1sq * v.wy) * rho2);
    ca[4][1] = ca[3][0];
    ca[4][2] = -((gammk * gamm1 * twgm1 * a0pq + gam * gammk * gammk * v.xz + gamm1 * gm1sq * v.wy) * rho);
    ca[4][3] = ca[1][0];
    ca[4][4] = ca[0][0];
    const double t = -two * wvno2;
    ca[2][0] = t * ca[4][2];
    ca[2][1] = t * ca[3][2];
    ca[2][2] = v.a0 + two * (v.cpcq - ca[0][0]);
    ca[2][3] = t * ca[1][2];
    ca[2][4] = t * ca[0][2];
}

// dnka followed by the row-vector product of dltar4 (ee(i) = sum_j
// e(j)*ca(j,i), surfdisp96.f:868-874).
__device__ inline void dnka_apply(const double* e, double* ee, double wvno2, double gam,
                                  double gammk, double rho, const VarOut& v) {
    double ca[5][5];
    dnka_matrix(ca, wvno2, gam, gammk, rho, v);
#pragma unroll
    for (int i = 0; i < 5; i++) {
        double cr = 0.0;
#pragma unroll
        for (int j = 0; j < 5; j++) cr = cr + e[j] * ca[j][i];
        ee[i] = cr;
    }
}

// surfdisp96.f:1025-1050
__device__ __forceinline__ void normc(double* ee, int n) {
    double t1 = 0.0;
    for (int i = 0; i < n; i++)
        if (fabs(ee[i]) > t1) t1 = fabs(ee[i]);
    if (t1 < 1.e-40) t1 = 1.0;
    for (int i = 0; i < n; i++) {
        double t2 = ee[i];
        t2 = t2 / t1;
        ee[i] = t2;
    }
}

// surfdisp96.f:801-901
static __device__ SK_ATTR_DLTAR4 double dltar4(const SDModel& M, double wvno, double omga) {
    const int mmax = M.mmax;
    double omega = omga;
    if (omega < 1.0e-4) omega = 1.0e-4;
    const double wvno2 = wvno * wvno;
    double xka = omega / (double)M.a[mmax - 1];
    double xkb = omega / (double)M.b[mmax - 1];
    double wvnop = wvno + xka;
    double wvnom = fabs(wvno - xka);
    double ra = sqrt(wvnop * wvnom);
    wvnop = wvno + xkb;
    wvnom = fabs(wvno - xkb);
    double rb = sqrt(wvnop * wvnom);
    double t = (double)M.b[mmax - 1] / omega;
    double gammk = 2.0 * t * t;
    double gam = gammk * wvno2;
    const double gamm1 = gam - 1.0;
    double rho1 = (double)M.rho[mmax - 1];
    double e[5], ee[5];
    e[0] = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
    e[1] = -(rho1 * ra);
    e[2] = rho1 * (gamm1 - gammk * ra * rb);
    e[3] = rho1 * rb;
    e[4] = wvno2 - ra * rb;
    for (int m = mmax - 2; m >= M.llw - 1; m--) {
        xka = omega / (double)M.a[m];
        xkb = omega / (double)M.b[m];
        t = (double)M.b[m] / omega;
        gammk = 2.0 * t * t;
        gam = gammk * wvno2;
        wvnop = wvno + xka;
        wvnom = fabs(wvno - xka);
        ra = sqrt(wvnop * wvnom);
        wvnop = wvno + xkb;
        wvnom = fabs(wvno - xkb);
        rb = sqrt(wvnop * wvnom);
        const double dpth = (double)M.d[m];
        rho1 = (double)M.rho[m];
        const double p = ra * dpth;
        const double q = rb * dpth;
        const VarOut v = var(p, q, ra, rb, wvno, xka, xkb, dpth);
        dnka_apply(e, ee, wvno2, gam, gammk, rho1, v);
        normc(ee, 5);
        for (int i = 0; i < 5; i++) e[i] = ee[i];
    }
    if (M.llw != 1) {
        xka = omega / (double)M.a[0];
        wvnop = wvno + xka;
        wvnom = fabs(wvno - xka);
        ra = sqrt(wvnop * wvnom);
        const double dpth = (double)M.d[0];
        rho1 = (double)M.rho[0];
        const double p = ra * dpth;
        const double znul = 1.0e-05;
        const VarOut v = var(p, znul, ra, znul, wvno, xka, znul, dpth);
        const double w0 = -(rho1 * v.w);
        return v.cosp * e[0] + w0 * e[1];
    }
    return e[0];
}

// surfdisp96.f:737-797
__device__ SK_NOINLINE double dltar1(const SDModel& M, double wvno, double omega) {
    const int mmax = M.mmax;
    double beta1 = (double)M.b[mmax - 1];
    double rho1 = (double)M.rho[mmax - 1];
    double xkb = omega / beta1;
    double wvnop = wvno + xkb;
    double wvnom = fabs(wvno - xkb);
    double rb = sqrt(wvnop * wvnom);
    double e1 = rho1 * rb;
    double e2 = 1.0 / (beta1 * beta1);
    for (int m = mmax - 2; m >= M.llw - 1; m--) {
        beta1 = (double)M.b[m];
        rho1 = (double)M.rho[m];
        const double xmu = rho1 * beta1 * beta1;
        xkb = omega / beta1;
        wvnop = wvno + xkb;
        wvnom = fabs(wvno - xkb);
        rb = sqrt(wvnop * wvnom);
        const double q = (double)M.d[m] * rb;
        double sinq, y, z, cosq;
        if (wvno < xkb) {
            sk_sincos(q, &sinq, &cosq);
            y = sinq / rb;
            z = -(rb * sinq);
        } else if (wvno == xkb) {
            cosq = 1.0;
            y = (double)M.d[m];
            z = 0.0;
        } else {
            double fac = 0.0;
            if (q < 16) fac = sk_exp(-2.0 * q);
            cosq = (1.0 + fac) * 0.5;
            sinq = (1.0 - fac) * 0.5;
            y = sinq / rb;
            z = rb * sinq;
        }
        const double e10 = e1 * cosq + e2 * xmu * z;
        const double e20 = e1 * y / xmu + e2 * cosq;
        double xnor = fabs(e10);
        const double ynor = fabs(e20);
        if (ynor > xnor) xnor = ynor;
        if (xnor < 1.e-40) xnor = 1.0;
        e1 = e10 / xnor;
        e2 = e20 / xnor;
    }
    return e1;
}

// ---------------------------------------------------------------------------
// Derivatives of the Rayleigh phase-velocity root (no reference counterpart:
// the reference's depth kernels come from sregn96's energy integrals, which
// agree with differences of surfdisp96's phase velocities only to about
// 1e-3).  dltar4's secular function is F = e_hs CA_{n} ... CA_0 u / N
// (e_hs the half-space row vector, CA_m the compound layer matrices, u the
// first unit vector, N the product of the normc scalings).  At the root F = 0,
// so with B_m = CA_{m-1} ... CA_0 u and e_{m+1} the normalised row vector
// entering layer m,
//   dF/dp_m = e_{m+1} (dCA_m/dp_m) B_m / (n_m ... n_0),   dc/dp = -F_p / F_c,
// dCA_m/dp_m and de_hs/dp by central differences of the one layer's matrix
// (relative step 1e-6), F_c by central differences of dltar4.
// ---------------------------------------------------------------------------
__device__ inline void layer_matrix(double a, double b, double rho, double d, double wvno,
                                    double omega, double ca[5][5]) {
    const double wvno2 = wvno * wvno;
    const double xka = omega / a, xkb = omega / b;
    const double t = b / omega;
    const double gammk = 2.0 * t * t;
    const double gam = gammk * wvno2;
    const double ra = sqrt((wvno + xka) * fabs(wvno - xka));
    const double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    const VarOut v = var(ra * d, rb * d, ra, rb, wvno, xka, xkb, d);
    dnka_matrix(ca, wvno2, gam, gammk, rho, v);
}
__device__ inline void halfspace_vector(double a, double b, double rho, double wvno, double omega,
                                        double e[5]) {
    const double wvno2 = wvno * wvno;
    const double xka = omega / a, xkb = omega / b;
    const double ra = sqrt((wvno + xka) * fabs(wvno - xka));
    const double rb = sqrt((wvno + xkb) * fabs(wvno - xkb));
    const double t = b / omega;
    const double gammk = 2.0 * t * t;
    const double gam = gammk * wvno2;
    const double gamm1 = gam - 1.0;
    e[0] = rho * rho * (gamm1 * gamm1 - gam * gammk * ra * rb);
    e[1] = -(rho * ra);
    e[2] = rho * (gamm1 - gammk * ra * rb);
    e[3] = rho * rb;
    e[4] = wvno2 - ra * rb;
}

// dc/d(b, a, rho) of the flattened layers of M (no water layer) at the root
// c for period t; `ein` (5 * mmax) and `logn` (mmax) are scratch.
__device__ inline void root_dcdm(const SDModel& M, double t, double c, double* dcb, double* dca,
                                 double* dcr, double* ein, double* logn) {
    const int mmax = M.mmax;
    const double omega = fmax(2.0 * 3.141592653589793 / t, 1.0e-4);
    const double wvno = omega / c;
    double e[5], ca[5][5];
    halfspace_vector(M.a[mmax - 1], M.b[mmax - 1], M.rho[mmax - 1], wvno, omega, e);
    for (int m = mmax - 2; m >= 0; m--) {
        for (int i = 0; i < 5; i++) ein[5 * m + i] = e[i];
        layer_matrix(M.a[m], M.b[m], M.rho[m], M.d[m], wvno, omega, ca);
        double ee[5], t1 = 0.0;
        for (int i = 0; i < 5; i++) {
            double cr = 0.0;
            for (int j = 0; j < 5; j++) cr += e[j] * ca[j][i];
            ee[i] = cr;
            t1 = fmax(t1, fabs(cr));
        }
        if (t1 < 1.e-40) t1 = 1.0;
        for (int i = 0; i < 5; i++) e[i] = ee[i] / t1;
        logn[m] = sk_log(t1);
    }
    const double hc = 1e-7 * c;
    const double Fc = (dltar4(M, omega / (c + hc), omega) - dltar4(M, omega / (c - hc), omega))
                      / (2.0 * hc);
    double B[5] = {1.0, 0.0, 0.0, 0.0, 0.0};
    double LB = 0.0, LN = 0.0;
    for (int m = 0; m <= mmax - 1; m++) {
        const bool hs = m == mmax - 1;
        if (!hs) LN += logn[m];
        const double scale = sk_exp(LB - LN);
        const double p0[3] = {M.b[m], M.a[m], M.rho[m]};
        double out[3];
        for (int q = 0; q < 3; q++) {
            double pp[3] = {p0[0], p0[1], p0[2]}, pm[3] = {p0[0], p0[1], p0[2]};
            const double h = 1e-6 * p0[q];
            pp[q] += h;
            pm[q] -= h;
            double s = 0.0;
            if (hs) {
                double ep[5], em[5];
                halfspace_vector(pp[1], pp[0], pp[2], wvno, omega, ep);
                halfspace_vector(pm[1], pm[0], pm[2], wvno, omega, em);
                for (int i = 0; i < 5; i++) s += (ep[i] - em[i]) / (2.0 * h) * B[i];
            } else {
                double cp[5][5], cm[5][5];
                layer_matrix(pp[1], pp[0], pp[2], M.d[m], wvno, omega, cp);
                layer_matrix(pm[1], pm[0], pm[2], M.d[m], wvno, omega, cm);
                for (int i = 0; i < 5; i++) {
                    double r = 0.0;
                    for (int j = 0; j < 5; j++) r += (cp[i][j] - cm[i][j]) / (2.0 * h) * B[j];
                    s += ein[5 * m + i] * r;
                }
            }
            out[q] = -(s * scale) / Fc;
        }
        dcb[m] = out[0];
        dca[m] = out[1];
        dcr[m] = out[2];
        if (hs) break;
        layer_matrix(M.a[m], M.b[m], M.rho[m], M.d[m], wvno, omega, ca);
        double nb[5], bm = 0.0;
        for (int i = 0; i < 5; i++) {
            double r = 0.0;
            for (int j = 0; j < 5; j++) r += ca[i][j] * B[j];
            nb[i] = r;
            bm = fmax(bm, fabs(r));
        }
        if (bm < 1e-300) bm = 1.0;
        for (int i = 0; i < 5; i++) B[i] = nb[i] / bm;
        LB += sk_log(bm);
    }
}

__device__ __forceinline__ double dltar(const SDModel& M, double wvno, double omega, int kk) {
    return kk == 1 ? dltar1(M, wvno, omega) : dltar4(M, wvno, omega);
}

// surfdisp96.f:578-711 (nevill with half inlined)
__device__ SK_NOINLINE double nevill(const SDModel& M, double t, double c1, double c2, double del1,
                                double del2, int ifunc, double twopi) {
    double x[20], y[20];
    const double omega = twopi / t;
    double c3 = 0.5 * (c1 + c2);
    double del3 = dltar(M, omega / c3, omega, ifunc);
    int nev = 1;
    int nctrl = 1;
    int m = 1;
    const double p01 = (double)0.01f;
    for (;;) {
        nctrl = nctrl + 1;
        if (nctrl >= 100) break;
        if (c3 < fmin(c1, c2) || c3 > fmax(c1, c2)) {
            nev = 0;
            c3 = 0.5 * (c1 + c2);
            del3 = dltar(M, omega / c3, omega, ifunc);
        }
        const double s13 = del1 - del3;
        const double s32 = del3 - del2;
        if (dsign1(del3) * dsign1(del1) < 0.0) {
            c2 = c3;
            del2 = del3;
        } else {
            c1 = c3;
            del1 = del3;
        }
        if (fabs(c1 - c2) <= 1.e-6 * c1) break;
        if (dsign1(s13) != dsign1(s32)) nev = 0;
        const double ss1 = fabs(del1);
        const double s1 = p01 * ss1;
        const double ss2 = fabs(del2);
        const double s2 = p01 * ss2;
        if (s1 > ss2 || s2 > ss1 || nev == 0) {
            c3 = 0.5 * (c1 + c2);
            del3 = dltar(M, omega / c3, omega, ifunc);
            nev = 1;
            m = 1;
        } else {
            if (nev == 2) {
                x[m] = c3;
                y[m] = del3;
            } else {
                x[0] = c1;
                y[0] = del1;
                x[1] = c2;
                y[1] = del2;
                m = 1;
            }
            bool bad = false;
            for (int kk = 1; kk <= m; kk++) {
                const int j = m - kk + 1;
                const double denom = y[m] - y[j - 1];
                if (fabs(denom) < 1.0e-10 * fabs(y[m])) {
                    bad = true;
                    break;
                }
                x[j - 1] = (-(y[j - 1] * x[j]) + y[m] * x[j - 1]) / denom;
            }
            if (!bad) {
                c3 = x[0];
                del3 = dltar(M, omega / c3, omega, ifunc);
                nev = 2;
                m = m + 1;
                if (m > 10) m = 10;
            } else {
                c3 = 0.5 * (c1 + c2);
                del3 = dltar(M, omega / c3, omega, ifunc);
                nev = 1;
                m = 1;
            }
        }
    }
    return c3;
}

// surfdisp96.f:403-498
__device__ SK_NOINLINE int getsol(SDModel& M, double t1, double& c1, double clow, double dc, double cm,
                             float betmx, int ifunc, int ifirst) {
    const double twopi = 2.0 * 3.141592653589793;
    double omega = twopi / t1;
    double wvno = omega / c1;
    double del1 = dltar(M, wvno, omega, ifunc);
    if (ifirst == 1) M.del1st = del1;
    const double plmn = dsign1(M.del1st) * dsign1(del1);
    int idir;
    if (ifirst == 1) idir = +1;
    else if (plmn >= 0.0) idir = +1;
    else idir = -1;
    for (int guard = 0; guard < 100000; guard++) {
        double c2;
        if (idir > 0) c2 = c1 + dc;
        else c2 = c1 - dc;
        if (c2 <= clow) {
            idir = +1;
            c1 = clow;
            continue;
        }
        omega = twopi / t1;
        wvno = omega / c2;
        const double del2 = dltar(M, wvno, omega, ifunc);
        if (dsign1(del1) != dsign1(del2)) {
            c1 = nevill(M, t1, c1, c2, del1, del2, ifunc, twopi);
            if (c1 > (double)betmx) return -1;
            return 1;
        }
        c1 = c2;
        del1 = del2;
        if (c1 < cm) return -1;
        if (c1 >= ((double)betmx + dc)) return -1;
    }
    return -1;
}

// surfdisp96.f:380-401 (REAL*4)
__device__ inline float gtsolh(float a, float b) {
    float c = 0.95f * b;
    for (int i = 0; i < 5; i++) {
        const float gamma = b / a;
        const float kappa = c / b;
        const float k2 = kappa * kappa;
        const float gk2 = (gamma * kappa) * (gamma * kappa);
        const float fac1 = sqrtf(1.0f - gk2);
        const float fac2 = sqrtf(1.0f - k2);
        const float t = 2.0f - k2;
        const float fr = t * t - 4.0f * fac1 * fac2;
        float frp = -(4.0f * (2.0f - k2) * kappa) + 4.0f * fac2 * gamma * gamma * kappa / fac1
                  + 4.0f * fac1 * kappa / fac2;
        frp = frp / b;
        c = c - fr / frp;
    }
    return c;
}

// surfdisp96.f:57-373 up to the root searches: the (flattened) layer model,
// the bracket step dc and the starting velocity cc of the first search.
__device__ inline void sd_setup(const LayerConst& L, const float* vpm, const float* vsm,
                                const float* rhom, int iflsph, int iwave, SDModel& M,
                                float& betmx, double& cc, double& dc) {
    const int mmax = L.mmax;
    M.mmax = mmax;
    float vmin = vsm[0];
    for (int i = 1; i < mmax; i++) vmin = fminf(vmin, vsm[i]);
    float ddc0;
    if (vmin < 1.0f) ddc0 = 0.001f;
    else if (vmin < 2.0f) ddc0 = 0.002f;
    else ddc0 = 0.005f;
    M.llw = 1;
    if (vsm[0] <= 0.0f) M.llw = 2;
    for (int i = 0; i < mmax; i++) {
        if (iflsph == 1) {   // sphere(0,0): velocities and thickness flattened
            M.d[i] = L.sd_d[i];
            M.a[i] = (float)(vpm[i] * L.sd_tmp[i]);
            M.b[i] = (float)(vsm[i] * L.sd_tmp[i]);
        } else {
            M.d[i] = L.thk[i];
            M.a[i] = vpm[i];
            M.b[i] = vsm[i];
        }
        M.rho[i] = rhom[i];
    }
    M.del1st = 0.0;
    int jmn = 1, jsol = 1;
    float betmn = 1.e20f;
    betmx = -1.e20f;
    for (int i = 0; i < mmax; i++) {
        if (M.b[i] > 0.01f && M.b[i] < betmn) {
            betmn = M.b[i];
            jmn = i + 1;
            jsol = 1;
        } else if (M.b[i] <= 0.01f && M.a[i] < betmn) {
            betmn = M.a[i];
            jmn = i + 1;
            jsol = 0;
        }
        if (M.b[i] > betmx) betmx = M.b[i];
    }
    const int ifunc = (iwave == 1) ? 1 : 2;
    if (iflsph == 1)   // sphere(ifunc,1): density mapping
        for (int i = 0; i < mmax; i++)
            M.rho[i] = rhom[i] * (ifunc == 1 ? L.sd_rhofac_love[i] : L.sd_rhofac[i]);
    const float ddc = ddc0;
    float cc1;
    if (jsol == 0) cc1 = betmn;
    else cc1 = gtsolh(M.a[jmn - 1], M.b[jmn - 1]);
    cc1 = 0.95f * cc1;
    cc1 = 0.90f * cc1;
    cc = (double)cc1;
    dc = fabs((double)ddc);
}

// surfdisp96.f:57-373 for one column, the searches in the reference's
// order.  vp/vs/rho: unflattened float model (mmax layers).  Returns 0, or
// 1 when the fundamental-mode search fails.
static __device__ int surfdisp96(const LayerConst& L, const float* vpm, const float* vsm,
                          const float* rhom, int iflsph, int iwave, int mode, int igr, int kmax,
                          const double* t, double* cg) {
    SDModel M;
    float betmx;
    double cc, dc;
    sd_setup(L, vpm, vsm, rhom, iflsph, iwave, M, betmx, cc, dc);
    const int ifunc = (iwave == 1) ? 1 : 2;
    const double one = 1.0e-2;
    const float sone = 1.500f;
    const float h = 0.005f;
    const double onea = (double)sone;
    double c[KMAX], cb[KMAX];
    double c1 = cc;
    const double cm = cc;
    double clow = cc;
    for (int i = 0; i < kmax; i++) {
        cb[i] = 0.0;
        c[i] = 0.0;
    }
    int ift = 999;
    for (int iq = 1; iq <= mode; iq++) {
        int kfail = -1;
        for (int k = 1; k <= kmax; k++) {
            if (k >= ift) {
                kfail = k;
                break;
            }
            double t1 = t[k - 1];
            float t1a, t1b = 0.0f;
            if (igr > 0) {
                t1a = (float)(t1 / (double)(1.0f + h));
                t1b = (float)(t1 / (double)(1.0f - h));
                t1 = (double)t1a;
            } else {
                t1a = (float)t1;
            }
            int ifirst;
            if (k == 1 && iq == 1) {
                c1 = cc;
                clow = cc;
                ifirst = 1;
            } else if (k == 1 && iq > 1) {
                c1 = c[0] + one * dc;
                clow = c1;
                ifirst = 1;
            } else if (k > 1 && iq > 1) {
                ifirst = 0;
                clow = c[k - 1] + one * dc;
                c1 = c[k - 2];
                if (c1 < clow) c1 = clow;
            } else {
                ifirst = 0;
                c1 = c[k - 2] - onea * dc;
                clow = cm;
            }
            int iret = getsol(M, t1, c1, clow, dc, cm, betmx, ifunc, ifirst);
            if (iret == -1) {
                kfail = k;
                break;
            }
            c[k - 1] = c1;
            if (igr > 0) {
                t1 = (double)t1b;
                ifirst = 0;
                clow = cb[k - 1] + one * dc;
                c1 = c1 - onea * dc;
                iret = getsol(M, t1, c1, clow, dc, cm, betmx, ifunc, ifirst);
                if (iret == -1) c1 = c[k - 1];
                cb[k - 1] = c1;
            } else {
                c1 = 0.0;
            }
            const float cc0 = (float)c[k - 1];
            const float ccg = (float)c1;
            if (igr == 0) {
                cg[k - 1] = cc0;
            } else {
                const float gvel =
                    (1.0f / t1a - 1.0f / t1b) / (1.0f / (t1a * cc0) - 1.0f / (t1b * ccg));
                cg[k - 1] = gvel;
            }
        }
        if (kfail < 0) continue;
        for (int i = kfail; i <= kmax; i++) cg[i - 1] = 0.0;
        if (iq <= 1) return 1;
        ift = kfail;
    }
    return 0;
}

// surfdisp96's fundamental-mode searches (getsol's bracket march, nevill's
// refinement, the period loop and the group velocity's second search) as a
// resumable state machine: advance() runs the control flow up to the next
// secular-function evaluation, leaves the requested (wvno, omega) in the
// state and returns true; the caller evaluates dltar there and passes the
// value back at the next advance().  Each lane's sequence of evaluations,
// and every operation on their values, are those of surfdisp96() above (the
// same trial velocities, brackets and Neville tables), so the results are
// bit-identical; what changes is that all lanes of a warp meet at one dltar
// call site, whichever period, march step or refinement step each is in,
// instead of running the march and the refinements of differently long
// brackets one after another.  Only mode 1 (the fundamental mode, what every
// caller here asks for).
struct RootSearch {
    enum : int { kStart = 0, kGsFirst, kGsMarch, kGsStep, kNvFirst, kNvTop, kNvTopEval,
                 kNvMid, kNvEnd, kDone };
    // per column
    double cc, dc, cm;
    float betmx;
    int igr, kmax;
    // progress
    int ph, k, stage, status;
    float t1a, t1b;
    double cprev;                      // c(k-1) of the period before
    double ck;                         // this period's phase velocity
    // getsol
    double t1, c1, clow, del1, c2;
    int idir, guard, ifirst;
    // nevill
    double n1, n2, nd1, nd2, c3, del3, nomega;
    int nev, nctrl, m;
    double x[11], y[11];
    // the requested evaluation
    double wvno, omega;
};

// surfdisp96.f:57-373 period loop, one step (see RootSearch).
__device__ inline bool root_advance(RootSearch& S, SDModel& M, double del, const double* t,
                                    double* cg) {
    const double twopi = 2.0 * 3.141592653589793;
    const double one = 1.0e-2;
    const double onea = (double)1.500f;
    const float h = 0.005f;
    for (;;) {
        switch (S.ph) {
            case RootSearch::kStart: {   // next period (surfdisp96.f:121-160)
                S.k++;
                if (S.k > S.kmax) {
                    S.ph = RootSearch::kDone;
                    S.status = 0;
                    return false;
                }
                double t1 = t[S.k - 1];
                S.t1b = 0.0f;
                if (S.igr > 0) {
                    S.t1a = (float)(t1 / (double)(1.0f + h));
                    S.t1b = (float)(t1 / (double)(1.0f - h));
                    t1 = (double)S.t1a;
                } else {
                    S.t1a = (float)t1;
                }
                if (S.k == 1) {
                    S.c1 = S.cc;
                    S.clow = S.cc;
                    S.ifirst = 1;
                } else {
                    S.ifirst = 0;
                    S.c1 = S.cprev - onea * S.dc;
                    S.clow = S.cm;
                }
                S.t1 = t1;
                S.stage = 0;
                // getsol entry: del1 at c1 (surfdisp96.f:413-416)
                S.omega = twopi / S.t1;
                S.wvno = S.omega / S.c1;
                S.ph = RootSearch::kGsFirst;
                return true;
            }
            case RootSearch::kGsFirst: {
                S.del1 = del;
                if (S.ifirst == 1) M.del1st = S.del1;
                const double plmn = dsign1(M.del1st) * dsign1(S.del1);
                if (S.ifirst == 1) S.idir = +1;
                else if (plmn >= 0.0) S.idir = +1;
                else S.idir = -1;
                S.guard = 0;
                S.ph = RootSearch::kGsMarch;
                break;
            }
            case RootSearch::kGsMarch: {   // next trial velocity (surfdisp96.f:431-446)
                if (S.guard >= 100000) goto getsol_fail;
                if (S.idir > 0) S.c2 = S.c1 + S.dc;
                else S.c2 = S.c1 - S.dc;
                if (S.c2 <= S.clow) {
                    S.idir = +1;
                    S.c1 = S.clow;
                    S.guard++;
                    break;
                }
                S.omega = twopi / S.t1;
                S.wvno = S.omega / S.c2;
                S.ph = RootSearch::kGsStep;
                return true;
            }
            case RootSearch::kGsStep: {
                const double del2 = del;
                if (dsign1(S.del1) != dsign1(del2)) {
                    // nevill entry (surfdisp96.f:578-590)
                    S.n1 = S.c1;
                    S.n2 = S.c2;
                    S.nd1 = S.del1;
                    S.nd2 = del2;
                    S.nomega = twopi / S.t1;
                    S.c3 = 0.5 * (S.n1 + S.n2);
                    S.omega = S.nomega;
                    S.wvno = S.nomega / S.c3;
                    S.ph = RootSearch::kNvFirst;
                    return true;
                }
                S.c1 = S.c2;
                S.del1 = del2;
                if (S.c1 < S.cm) goto getsol_fail;
                if (S.c1 >= ((double)S.betmx + S.dc)) goto getsol_fail;
                S.guard++;
                S.ph = RootSearch::kGsMarch;
                break;
            }
            case RootSearch::kNvFirst:
                S.del3 = del;
                S.nev = 1;
                S.nctrl = 1;
                S.m = 1;
                S.ph = RootSearch::kNvTop;
                break;
            case RootSearch::kNvTop:   // surfdisp96.f:593-600
                S.nctrl = S.nctrl + 1;
                if (S.nctrl >= 100) goto nevill_done;
                if (S.c3 < fmin(S.n1, S.n2) || S.c3 > fmax(S.n1, S.n2)) {
                    S.nev = 0;
                    S.c3 = 0.5 * (S.n1 + S.n2);
                    S.omega = S.nomega;
                    S.wvno = S.nomega / S.c3;
                    S.ph = RootSearch::kNvTopEval;
                    return true;
                }
                S.ph = RootSearch::kNvMid;
                break;
            case RootSearch::kNvTopEval:
                S.del3 = del;
                S.ph = RootSearch::kNvMid;
                break;
            case RootSearch::kNvMid: {   // surfdisp96.f:601-696
                const double s13 = S.nd1 - S.del3;
                const double s32 = S.del3 - S.nd2;
                if (dsign1(S.del3) * dsign1(S.nd1) < 0.0) {
                    S.n2 = S.c3;
                    S.nd2 = S.del3;
                } else {
                    S.n1 = S.c3;
                    S.nd1 = S.del3;
                }
                if (fabs(S.n1 - S.n2) <= 1.e-6 * S.n1) goto nevill_done;
                if (dsign1(s13) != dsign1(s32)) S.nev = 0;
                const double p01 = (double)0.01f;
                const double ss1 = fabs(S.nd1);
                const double s1 = p01 * ss1;
                const double ss2 = fabs(S.nd2);
                const double s2 = p01 * ss2;
                bool halve = s1 > ss2 || s2 > ss1 || S.nev == 0;
                if (!halve) {
                    int m = S.m;
                    if (S.nev == 2) {
                        S.x[m] = S.c3;
                        S.y[m] = S.del3;
                    } else {
                        S.x[0] = S.n1;
                        S.y[0] = S.nd1;
                        S.x[1] = S.n2;
                        S.y[1] = S.nd2;
                        m = 1;
                    }
                    bool bad = false;
                    for (int kk = 1; kk <= m; kk++) {
                        const int j = m - kk + 1;
                        const double denom = S.y[m] - S.y[j - 1];
                        if (fabs(denom) < 1.0e-10 * fabs(S.y[m])) {
                            bad = true;
                            break;
                        }
                        S.x[j - 1] = (-(S.y[j - 1] * S.x[j]) + S.y[m] * S.x[j - 1]) / denom;
                    }
                    if (!bad) {
                        S.c3 = S.x[0];
                        S.nev = 2;
                        m = m + 1;
                        if (m > 10) m = 10;
                        S.m = m;
                    } else {
                        halve = true;
                    }
                }
                if (halve) {
                    S.c3 = 0.5 * (S.n1 + S.n2);
                    S.nev = 1;
                    S.m = 1;
                }
                S.omega = S.nomega;
                S.wvno = S.nomega / S.c3;
                S.ph = RootSearch::kNvEnd;
                return true;
            }
            case RootSearch::kNvEnd:
                S.del3 = del;
                S.ph = RootSearch::kNvTop;
                break;
            default:
                return false;
        }
        continue;
    nevill_done:   // getsol after nevill (surfdisp96.f:455-459)
        S.c1 = S.c3;
        if (S.c1 > (double)S.betmx) goto getsol_fail;
        // getsol found its root: c1
        if (S.stage == 0) {
            S.ck = S.c1;
            if (S.igr > 0) {   // the group velocity's second search (surfdisp96.f:181-192)
                S.stage = 1;
                S.t1 = (double)S.t1b;
                S.ifirst = 0;
                S.clow = 0.0 + one * S.dc;   // cb(k) is still 0 in mode 1
                S.c1 = S.c1 - onea * S.dc;
                S.omega = twopi / S.t1;
                S.wvno = S.omega / S.c1;
                S.ph = RootSearch::kGsFirst;
                return true;
            }
            cg[S.k - 1] = (float)S.ck;
        } else {
            const float cc0 = (float)S.ck;
            const float ccg = (float)S.c1;
            cg[S.k - 1] = (1.0f / S.t1a - 1.0f / S.t1b) / (1.0f / (S.t1a * cc0) - 1.0f / (S.t1b * ccg));
        }
        S.cprev = S.ck;
        S.ph = RootSearch::kStart;
        continue;
    getsol_fail:
        if (S.stage == 0) {   // the fundamental mode fails from this period on
            for (int i = S.k; i <= S.kmax; i++) cg[i - 1] = 0.0;
            S.ph = RootSearch::kDone;
            S.status = 1;
            return false;
        }
        {   // the second search failed: the group velocity uses c itself
            const float cc0 = (float)S.ck;
            const float ccg = (float)S.ck;
            cg[S.k - 1] = (1.0f / S.t1a - 1.0f / S.t1b) / (1.0f / (S.t1a * cc0) - 1.0f / (S.t1b * ccg));
        }
        S.cprev = S.ck;
        S.ph = RootSearch::kStart;
    }
}

// surfdisp96() with the searches of all lanes meeting at one dltar call
// (see RootSearch); same arguments and results, mode 1.
static __device__ int surfdisp96_lockstep(const LayerConst& L, const float* vpm, const float* vsm,
                                          const float* rhom, int iflsph, int iwave, int igr,
                                          int kmax, const double* t, double* cg) {
    SDModel M;
    RootSearch S;
    sd_setup(L, vpm, vsm, rhom, iflsph, iwave, M, S.betmx, S.cc, S.dc);
    const int ifunc = (iwave == 1) ? 1 : 2;
    S.cm = S.cc;
    S.igr = igr;
    S.kmax = kmax;
    S.ph = RootSearch::kStart;
    S.k = 0;
    S.status = 0;
    S.cprev = 0.0;
    S.ck = 0.0;
    double del = 0.0;
    while (root_advance(S, M, del, t, cg)) del = dltar(M, S.wvno, S.omega, ifunc);
    return S.status;
}

// ---------------------------------------------------------------------------
// sregn96_hti (sregn96.f90:1745-1849), Rayleigh, no fluid layers required
// (the fluid branches are kept for completeness).
// ---------------------------------------------------------------------------
struct cx {
    double re, im;
};
__device__ __forceinline__ cx C(double r, double i = 0.0) { return {r, i}; }
__device__ __forceinline__ cx operator+(cx a, cx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cx operator-(cx a, cx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cx operator-(cx a) { return {-a.re, -a.im}; }
__device__ __forceinline__ cx operator*(cx a, cx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cx operator*(double s, cx a) { return {s * a.re, s * a.im}; }
__device__ __forceinline__ cx operator*(cx a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ cx operator-(double s, cx a) { return {s - a.re, -a.im}; }
__device__ __forceinline__ cx operator/(cx a, double s) { return {a.re / s, a.im / s}; }
// gfortran's range-reduced complex division
#ifndef SK_CDIV_ATTR
#define SK_CDIV_ATTR __forceinline__
#endif
static __device__ SK_CDIV_ATTR cx cdiv_(cx a, cx b) {
    const double ar = a.re, ai = a.im, br = b.re, bi = b.im;
    if (fabs(br) < fabs(bi)) {
        const double ratio = br / bi;
        const double div = (br * ratio) + bi;
        return {((ar * ratio) + ai) / div, ((ai * ratio) - ar) / div};
    }
    const double ratio = bi / br;
    const double div = (bi * ratio) + br;
    return {((ai * ratio) + ar) / div, (ai - (ar * ratio)) / div};
}
__device__ __forceinline__ cx operator/(cx a, cx b) { return cdiv_(a, b); }
__device__ __forceinline__ cx operator/(double s, cx b) { return C(s) / b; }
__device__ __forceinline__ double cabs_(cx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ cx csqrt_real(double x) {
    if (x < 0.0) return {0.0, sqrt(-x)};
    return {sqrt(x), 0.0};
}
__device__ __forceinline__ cx cexp_(cx a) {
    const double e = sk_exp(a.re);
    double sn, cs;
    sk_sincos(a.im, &sn, &cs);
    return {e * cs, e * sn};
}
__device__ __forceinline__ cx conj_(cx a) { return {a.re, -a.im}; }

struct RW {
    int mmax;
    bool allfluid;
    double zd[MMAX], zrho[MMAX], za[MMAX], zb[MMAX], xmu[MMAX], xlam[MMAX];
    double ur[MMAX], uz[MMAX], tz[MMAX], tr[MMAX];
    double dcda[MMAX], dcdb[MMAX], dcdr[MMAX], dcdh[MMAX], dcdgc[MMAX];
    double exe[MMAX], exa[MMAX];
    double cd[MMAX][5], vv[MMAX][4];
    unsigned char iwat[MMAX];
    cx ra, rb;
    cx e[4][4], einv[4][4];
};

struct VarSv {
    double cosp, cosq, rsinp, rsinq, sinpr, sinqr, pex, svex;
};
// sregn96.f90:827-911
static __device__ SK_NOINLINE_EIG VarSv varsv(cx p, cx q, cx rp, cx rsv, int iwat, double zd) {
    VarSv o;
    const double lim = (double)1.0e-5f;
    o.svex = 0.0;
    const double pr = p.re, pi = p.im, qr = q.re, qi = q.im;
    o.pex = pr;
    double spi, cpi;
    sk_sincos(pi, &spi, &cpi);
    const cx epp = C(cpi, spi) / 2.0;
    const cx epm = conj_(epp);
    const double pfac = (pr < 30.0) ? sk_exp(-(2.0 * pr)) : 0.0;
    o.cosp = (epp + pfac * epm).re;
    const cx sinp = epp - pfac * epm;
    o.rsinp = (rp * sinp).re;
    if (fabs(pr) < lim && cabs_(rp) < lim) o.sinpr = zd;
    else o.sinpr = (sinp / rp).re;
    if (iwat == 1) {
        o.cosq = 1.0;
        o.rsinq = 0.0;
        o.sinqr = 0.0;
    } else {
        o.svex = qr;
        double sqi, cqi;
        sk_sincos(qi, &sqi, &cqi);
        const cx eqp = C(cqi, sqi) / 2.0;
        const cx eqm = conj_(eqp);
        const double svfac = (qr < 30.0) ? sk_exp(-(2.0 * qr)) : 0.0;
        o.cosq = (eqp + svfac * eqm).re;
        const cx sinq = eqp - svfac * eqm;
        o.rsinq = (rsv * sinq).re;
        if (fabs(qr) < lim && cabs_(rsv) < lim) o.sinqr = zd;
        else o.sinqr = (sinq / rsv).re;
    }
    return o;
}

// sregn96.f90:491-647 fused with the product ee(i) = sum_j cd(m+1,j)*ca(j,i)
static __device__ SK_NOINLINE_EIG void dnka_rg(double ca[5][5], double cosp, double rsinp, double sinpr,
                               double cossv, double rsinsv, double sinsvr, float rho, float b,
                               int iwat, double ex, double exa, double wvno, double wvno2,
                               double om2) {
    if (iwat == 1) {
        for (int j = 0; j < 5; j++)
            for (int i = 0; i < 5; i++) ca[i][j] = 0.0;
        const double dfac = (ex > 35.0) ? 0.0 : sk_exp(-ex);
        ca[2][2] = dfac;
        ca[0][0] = cosp;
        ca[4][4] = cosp;
        ca[0][1] = -(rsinp / (rho * om2));
        ca[1][0] = -(rho * sinpr * om2);
        ca[1][1] = cosp;
        ca[3][3] = cosp;
        ca[3][4] = ca[0][1];
        ca[4][3] = ca[1][0];
        return;
    }
    const double a0 = (exa < 60.0) ? sk_exp(-exa) : 0.0;
    const double cpcq = cosp * cossv;
    const double cpy = cosp * sinsvr;
    const double cpz = cosp * rsinsv;
    const double cqw = cossv * sinpr;
    const double cqx = cossv * rsinp;
    const double xy = rsinp * sinsvr;
    const double xz = rsinp * rsinsv;
    const double wy = sinpr * sinsvr;
    const double wz = sinpr * rsinsv;
    const float rho2 = rho * rho;
    const double gam = (double)(2.0f * b * b) * wvno2 / om2;
    const double gam2 = gam * gam;
    const double gamm1 = gam - 1.0;
    const double gamm2 = gamm1 * gamm1;
    const double cqww2 = cqw * wvno2;
    const double cqxw2 = cqx / wvno2;
    const double gg1 = gam * gamm1;
    const double a0c = 2.0 * (a0 - cpcq);
    const double xz2 = xz / wvno2;
    const double gxz2 = gam * xz2;
    const double g2xz2 = gam2 * xz2;
    const double a0cgg1 = a0c * (gam + gamm1);
    const double wy2 = wy * wvno2;
    const double g2wy2 = gamm2 * wy2;
    const double g1wy2 = gamm1 * wy2;
    const double rom2 = (double)rho * om2;
    double temp = a0c * gg1 + g2xz2 + g2wy2;
    ca[2][2] = a0 + temp + temp;
    ca[0][0] = cpcq - temp;
    ca[0][1] = (-cqx + wvno2 * cpy) / rom2;
    temp = 0.5 * a0cgg1 + gxz2 + g1wy2;
    ca[0][2] = wvno * temp / rom2;
    ca[0][3] = (-cqww2 + cpz) / rom2;
    temp = wvno2 * (a0c + wy2) + xz;
    ca[0][4] = -(temp / ((double)rho2 * om2 * om2));
    ca[1][0] = (-(gamm2 * cqw) + gam2 * cpz / wvno2) * (double)rho * om2;
    ca[1][1] = cpcq;
    ca[1][2] = (gamm1 * cqww2 - gam * cpz) / wvno;
    ca[1][3] = -wz;
    ca[1][4] = ca[0][3];
    temp = 0.5 * a0cgg1 * gg1 + gam2 * gxz2 + gamm2 * g1wy2;
    ca[2][0] = -(2.0 * temp * (double)rho * om2 / wvno);
    ca[2][1] = -(wvno * (gam * cqxw2 - gamm1 * cpy) * 2.0);
    ca[2][3] = -2.0 * ca[1][2];
    ca[2][4] = -2.0 * ca[0][2];
    ca[3][0] = (-(gam2 * cqxw2) + gamm2 * cpy) * (double)rho * om2;
    ca[3][1] = -xy;
    ca[3][2] = -(ca[2][1] / 2.0);
    ca[3][3] = ca[1][1];
    ca[3][4] = ca[0][1];
    temp = gamm2 * (a0c * gam2 + g2wy2) + gam2 * g2xz2;
    ca[4][0] = -((double)rho2 * om2 * om2 * temp / wvno2);
    ca[4][1] = ca[3][0];
    ca[4][2] = -(ca[2][0] / 2.0);
    ca[4][3] = ca[1][0];
    ca[4][4] = ca[0][0];
}

// sregn96.f90:649-825 (jbdry = 0, inp = 1)
static __device__ SK_NOINLINE_EIG void evalg(RW& W, int m, cx* gbr, double wvno, double om, double om2,
                             double wvno2) {
    const double xka = om / W.za[m - 1];
    const double xkb = (W.zb[m - 1] > 0.0) ? om / W.zb[m - 1] : 0.0;
    W.ra = csqrt_real(wvno2 - xka * xka);
    W.rb = csqrt_real(wvno2 - xkb * xkb);
    const cx ra = W.ra, rb = W.rb;
    double gam = W.zb[m - 1] * wvno / om;
    gam = 2.0 * (gam * gam);
    const double gamm1 = gam - 1.0;
    const double zr = W.zrho[m - 1];
    cx(&E)[4][4] = W.e;
    cx(&EI)[4][4] = W.einv;
    if (W.iwat[m - 1] == 0) {
        E[0][0] = C(wvno);
        E[0][1] = rb;
        E[0][2] = C(wvno);
        E[0][3] = -rb;
        E[1][0] = ra;
        E[1][1] = C(wvno);
        E[1][2] = -ra;
        E[1][3] = C(wvno);
        E[2][0] = C(zr * om2 * gamm1);
        E[2][1] = (zr * om2 * gam) * rb / wvno;
        E[2][2] = C(zr * om2 * gamm1);
        E[2][3] = -((zr * om2 * gam) * rb / wvno);
        E[3][0] = (zr * om2 * gam) * ra / wvno;
        E[3][1] = C(zr * om2 * gamm1);
        E[3][2] = -((zr * om2 * gam) * ra / wvno);
        E[3][3] = C(zr * om2 * gamm1);
        EI[0][0] = C(0.5 * gam / wvno);
        EI[0][1] = -((0.5 * gamm1) / ra);
        EI[0][2] = C(-(0.5 / (zr * om2)));
        EI[0][3] = (0.5 * wvno) / ((zr * om2) * ra);
        EI[1][0] = -((0.5 * gamm1) / rb);
        EI[1][1] = C(0.5 * gam / wvno);
        EI[1][2] = (0.5 * wvno) / ((zr * om2) * rb);
        EI[1][3] = C(-(0.5 / (zr * om2)));
        EI[2][0] = C(0.5 * gam / wvno);
        EI[2][1] = (0.5 * gamm1) / ra;
        EI[2][2] = C(-(0.5 / (zr * om2)));
        EI[2][3] = -((0.5 * wvno) / ((zr * om2) * ra));
        EI[3][0] = (0.5 * gamm1) / rb;
        EI[3][1] = C(0.5 * gam / wvno);
        EI[3][2] = -((0.5 * wvno) / ((zr * om2) * rb));
        EI[3][3] = C(-(0.5 / (zr * om2)));
        if (gbr) {
            gbr[0] = ((zr * zr) * om2 * om2) * (-((gam * gam) * ra * rb) + C(wvno2 * gamm1 * gamm1));
            gbr[1] = -((zr * (wvno2 * ra)) * om2);
            gbr[2] = -(((zr * (-((gam * ra) * rb) + C(wvno2 * gamm1))) * om2) * wvno);
            gbr[3] = (zr * (wvno2 * rb)) * om2;
            gbr[4] = wvno2 * (C(wvno2) - ra * rb);
            const cx den = -((((zr * zr) * om2 * om2 * wvno2) * ra) * rb);
            for (int k = 0; k < 5; k++) gbr[k] = (0.25 * gbr[k]) / den;
        }
    } else {
        if (gbr) {
            if (W.allfluid) {
                gbr[0] = 0.5 / ra;
                gbr[1] = C(0.5) / C(-(zr * om2));
                gbr[2] = C(0.0);
                gbr[3] = C(0.0);
                gbr[4] = C(0.0);
            } else {
                gbr[0] = C(0.0);
                gbr[1] = C(0.0);
                gbr[2] = C(0.0);
                gbr[3] = ((0.5 * zr) * om2) / ra;
                gbr[4] = C(-0.5);
            }
        }
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
                E[i][j] = C(0.0);
                EI[i][j] = C(0.0);
            }
        E[0][0] = ra;
        E[0][1] = -ra;
        E[1][0] = C(-(zr * om2));
        E[1][1] = C(-(zr * om2));
        EI[0][0] = 0.5 / ra;
        EI[0][1] = C(-(0.5 / (zr * om2)));
        EI[1][0] = -(0.5 / ra);
        EI[1][1] = C(-(0.5 / (zr * om2)));
    }
}

__device__ __forceinline__ double normc_ex(double* ee, int nmat) {
    double t1 = 0.0;
    for (int i = 0; i < nmat; i++)
        if (fabs(ee[i]) > t1) t1 = fabs(ee[i]);
    if (t1 < 1.e-40) t1 = 1.0;
    for (int i = 0; i < nmat; i++) {
        double t2 = ee[i];
        t2 = t2 / t1;
        ee[i] = t2;
    }
    return sk_log(t1);
}

// sregn96.f90:401-489
__device__ inline void up(RW& W, double omega, double wvno) {
    const double wvno2 = wvno * wvno;
    const double om2 = omega * omega;
    cx gbr[5];
    evalg(W, W.mmax, gbr, wvno, omega, om2, wvno2);
    for (int j = 0; j < 5; j++) W.cd[W.mmax - 1][j] = gbr[j].re;
    W.exe[W.mmax - 1] = 0.0;
    double exsum = 0.0;
    double ca[5][5], ee[5];
    for (int m = W.mmax - 1; m >= 1; m--) {
        const double xka = omega / W.za[m - 1];
        const double xkb = (W.zb[m - 1] > 0.0) ? omega / W.zb[m - 1] : 0.0;
        const cx rp = csqrt_real(wvno2 - xka * xka);
        const cx rsv = csqrt_real(wvno2 - xkb * xkb);
        const VarSv v = varsv(rp * W.zd[m - 1], rsv * W.zd[m - 1], rp, rsv, W.iwat[m - 1],
                              W.zd[m - 1]);
        dnka_rg(ca, v.cosp, v.rsinp, v.sinpr, v.cosq, v.rsinq, v.sinqr, (float)W.zrho[m - 1],
                (float)W.zb[m - 1], W.iwat[m - 1], v.pex, v.pex + v.svex, wvno, wvno2, om2);
        for (int i = 0; i < 5; i++) {
            double cr = 0.0;
            for (int j = 0; j < 5; j++) cr = cr + W.cd[m][j] * ca[j][i];
            ee[i] = cr;
        }
        const double exn = normc_ex(ee, 5);
        exsum = exsum + v.pex + v.svex + exn;
        W.exe[m - 1] = exsum;
        for (int i = 0; i < 5; i++) W.cd[m - 1][i] = ee[i];
    }
}

// sregn96.f90:913-987
__device__ inline void hska(double AA[4][4], double cosp, double rsinp, double sinpr,
                            double tcossv, double trsinsv, double tsinsvr, float rho, float b,
                            int iwat, double pex, double svex, double wvno, double wvno2,
                            double om2) {
    const double rom2 = (double)rho * om2;
    if (iwat == 1) {
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) AA[i][j] = 0.0;
        const double dfac = (pex > 35.0) ? 0.0 : sk_exp(-pex);
        AA[0][0] = dfac;
        AA[3][3] = dfac;
        AA[1][1] = cosp;
        AA[2][2] = cosp;
        AA[1][2] = -(rsinp / rom2);
        AA[2][1] = -(rom2 * sinpr);
        return;
    }
    const double dfac = ((pex - svex) > 70.0) ? 0.0 : sk_exp(svex - pex);
    const double cossv = dfac * tcossv;
    const double rsinsv = dfac * trsinsv;
    const double sinsvr = dfac * tsinsvr;
    const double gam = (double)(2.0f * b * b) * wvno2 / om2;
    const double gamm1 = gam - 1.0;
    AA[0][0] = cossv + gam * (cosp - cossv);
    AA[0][1] = -(wvno * gamm1 * sinpr) + gam * rsinsv / wvno;
    AA[0][2] = -(wvno * (cosp - cossv) / rom2);
    AA[0][3] = (wvno2 * sinpr - rsinsv) / rom2;
    AA[1][0] = gam * rsinp / wvno - wvno * gamm1 * sinsvr;
    AA[1][1] = cosp - gam * (cosp - cossv);
    AA[1][2] = (-rsinp + wvno2 * sinsvr) / rom2;
    AA[1][3] = -AA[0][2];
    AA[2][0] = rom2 * gam * gamm1 * (cosp - cossv) / wvno;
    AA[2][1] = rom2 * (-(gamm1 * gamm1 * sinpr) + gam * gam * rsinsv / wvno2);
    AA[2][2] = AA[1][1];
    AA[2][3] = -AA[0][1];
    AA[3][0] = rom2 * (gam * gam * rsinp / wvno2 - gamm1 * gamm1 * sinsvr);
    AA[3][1] = -AA[2][0];
    AA[3][2] = -AA[1][0];
    AA[3][3] = AA[0][0];
}

// sregn96.f90:989-1059
__device__ inline void down(RW& W, double omega, double wvno) {
    const double om2 = omega * omega;
    const double wvno2 = wvno * wvno;
    for (int i = 0; i < 4; i++) W.vv[0][i] = (i == 0) ? 1.0 : 0.0;
    W.exa[0] = 0.0;
    double exsum = 0.0;
    double AA[4][4], aa0[4];
    for (int m = 1; m <= W.mmax - 1; m++) {
        const double xka = omega / W.za[m - 1];
        const double xkb = (W.zb[m - 1] > 0.0) ? omega / W.zb[m - 1] : 0.0;
        const cx rp = csqrt_real(wvno2 - xka * xka);
        const cx rsv = csqrt_real(wvno2 - xkb * xkb);
        const VarSv v = varsv(rp * W.zd[m - 1], rsv * W.zd[m - 1], rp, rsv, W.iwat[m - 1],
                              W.zd[m - 1]);
        hska(AA, v.cosp, v.rsinp, v.sinpr, v.cosq, v.rsinq, v.sinqr, (float)W.zrho[m - 1],
             (float)W.zb[m - 1], W.iwat[m - 1], v.pex, v.svex, wvno, wvno2, om2);
        for (int i = 0; i < 4; i++) {
            double cc = 0.0;
            for (int j = 0; j < 4; j++) cc = cc + AA[i][j] * W.vv[m - 1][j];
            aa0[i] = cc;
        }
        const double ex2 = normc_ex(aa0, 4);
        exsum = exsum + v.pex + ex2;
        W.exa[m] = exsum;
        for (int i = 0; i < 4; i++) W.vv[m][i] = aa0[i];
    }
}

// sregn96.f90:193-399
// svfunc after up() and down(): the eigenfunctions from the compound
// matrices and the propagator vectors.
__device__ inline void svfunc_combine(RW& W) {
    const double f1213 = -W.cd[0][1];
    W.ur[0] = W.cd[0][2] / W.cd[0][1];
    W.uz[0] = 1.0;
    W.tz[0] = 0.0;
    W.tr[0] = 0.0;
    for (int i = 2; i <= W.mmax; i++) {
        const double* cdi = W.cd[i - 1];
        const double cd1 = cdi[0], cd2 = cdi[1], cd3 = cdi[2], cd4 = -cdi[2], cd5 = cdi[3],
                     cd6 = cdi[4];
        const double* vvi = W.vv[i - 1];
        const double tz1 = -vvi[3], tz2 = -vvi[2], tz3 = vvi[1], tz4 = vvi[0];
        const double uu1 = tz2 * cd6 - tz3 * cd5 + tz4 * cd4;
        const double uu2 = -(tz1 * cd6) + tz3 * cd3 - tz4 * cd2;
        const double uu3 = tz1 * cd5 - tz2 * cd3 + tz4 * cd1;
        const double uu4 = -(tz1 * cd4) + tz2 * cd2 - tz3 * cd1;
        const double ext = W.exa[i - 1] + W.exe[i - 1] - W.exe[0];
        if (ext > -80.0 && ext < 80.0) {
            const double fact = sk_exp(ext);
            W.ur[i - 1] = uu1 * fact / f1213;
            W.uz[i - 1] = uu2 * fact / f1213;
            W.tz[i - 1] = uu3 * fact / f1213;
            W.tr[i - 1] = uu4 * fact / f1213;
        } else {
            W.ur[i - 1] = 0.0;
            W.uz[i - 1] = 0.0;
            W.tz[i - 1] = 0.0;
            W.tr[i - 1] = 0.0;
        }
    }
    if (!W.allfluid) {
        int jwat = 0;
        for (int i = 1; i <= W.mmax; i++) {
            if (W.iwat[i - 1] > 0) jwat = i;
            else break;
        }
        for (int i = 1; i <= jwat; i++) {
            W.ur[i - 1] = 0.0;
            W.tr[i - 1] = 0.0;
        }
    }
}

__device__ inline void svfunc(RW& W, double omega, double wvno) {
    up(W, omega, wvno);
    down(W, omega, wvno);
    svfunc_combine(W);
}

// The depth kernels run blocks of SK_DEPTH_PHASED threads, one block per SM
// (96 registers each), and a block barrier between the eigenfunction
// routines keeps all warps of an SM on the same routine: up, down, the
// eigenfunctions, the energy integrals.  Launched as 64-thread blocks at 10
// per SM without barriers (SK_DEPTH_PHASED 0), the blocks drift apart, every
// routine's code is in flight on an SM at once and the warps stall on
// instruction fetch (C3 Rayleigh phase kernels: 71.2 ms against 55.2 ms
// phased).  Threads past the last item repeat it, to meet the barriers, and
// store nothing.
#ifndef SK_DEPTH_PHASED
#define SK_DEPTH_PHASED 640
#endif
#if SK_DEPTH_PHASED > 0
#define SK_DEPTH_BLOCK SK_DEPTH_PHASED
#define SK_DEPTH_BOUNDS __launch_bounds__(SK_DEPTH_PHASED, 1)
#define SK_PHASE() __syncthreads()
#else
#define SK_DEPTH_BLOCK 64
#define SK_DEPTH_BOUNDS __launch_bounds__(64, 10)
#define SK_PHASE() ((void)0)
#endif
__device__ inline void svfunc_phased(RW& W, double omega, double wvno) {
    SK_PHASE();
    up(W, omega, wvno);
    SK_PHASE();
    down(W, omega, wvno);
    SK_PHASE();
    svfunc_combine(W);
    SK_PHASE();
}

// sregn96.f90:1326-1404
__device__ inline cx ffunc(cx nub, double dm) {
    if (cabs_(nub) < 1.0e-08) return C(dm);
    const cx argcd = nub * dm;
    const cx exqq = (argcd.re < 40.0) ? cexp_(-(2.0 * argcd)) : C(0.0);
    return (1.0 - exqq) / (2.0 * nub);
}
__device__ inline cx gfunc(cx nub, double dm) {
    const cx argcd = nub * dm;
    if (argcd.re < 75.0) return cexp_(-argcd) * dm;
    return C(0.0, 0.0);
}
__device__ inline cx h1func(cx nua, cx nub, double dm) {
    if (cabs_(nub + nua) < 1.0e-08) return C(dm);
    const cx argcd = (nua + nub) * dm;
    const cx exqq = (argcd.re < 40.0) ? cexp_(-argcd) : C(0.0);
    return (1.0 - exqq) / (nub + nua);
}
__device__ inline cx h2func(cx nua, cx nub, double dm) {
    if (cabs_(nub - nua) < 1.0e-08) return C(dm);
    cx argcd = nua * dm;
    const cx exqp = (argcd.re < 40.0) ? cexp_(-argcd) : C(0.0);
    argcd = nub * dm;
    const cx exqq = (argcd.re < 40.0) ? cexp_(-argcd) : C(0.0);
    return (exqq - exqp) / (nua - nub);
}

// The six energy integrals of one layer (sregn96.f90:1205-1324 called with
// (1,1),(1,3),(2,2),(2,4),(3,3),(4,4)); evalg is evaluated once per layer
// (its outputs are the same for every (i, j)).
static __device__ SK_NOINLINE_EIG void layer_integrals(RW& W, int m, int typelyr, double om, double om2,
                                       double wvno, double wvno2, double* I) {
    evalg(W, m, nullptr, wvno, om, om2, wvno2);
    const cx ra = W.ra, rb = W.rb;
    const double zd = W.zd[m - 1];
    auto e = [&](int a, int b) { return W.e[a - 1][b - 1]; };
    auto ei = [&](int a, int b) { return W.einv[a - 1][b - 1]; };
    const int II[6] = {1, 1, 2, 2, 3, 4};
    const int JJ[6] = {1, 3, 2, 4, 3, 4};
    if (W.iwat[m - 1] == 1) {
        cx kmpu = C(0.0), km1pd = C(0.0), FA = C(0.0), GA = C(0.0);
        if (typelyr < 0) {
            kmpu = ei(1, 1) * W.uz[m] + ei(1, 2) * W.tz[m];
        } else if (typelyr == 0) {
            km1pd = ei(2, 1) * W.uz[m - 1] + ei(2, 2) * W.tz[m - 1];
            kmpu = ei(1, 1) * W.uz[m] + ei(1, 2) * W.tz[m];
            FA = ffunc(ra, zd);
            GA = gfunc(ra, zd);
        } else {
            km1pd = ei(2, 1) * W.uz[m - 1] + ei(2, 2) * W.tz[m - 1];
        }
        for (int q = 0; q < 6; q++) {
            const int i = II[q], j = JJ[q];
            cx c;
            if (typelyr < 0) c = e(i, 1) * e(j, 1) * kmpu * kmpu / (2.0 * ra);
            else if (typelyr == 0)
                c = e(i, 1) * e(j, 1) * kmpu * kmpu * FA
                  + (e(i, 1) * e(j, 2) + e(i, 2) * e(j, 1)) * kmpu * km1pd * GA
                  + e(i, 2) * e(j, 2) * km1pd * km1pd * FA;
            else c = e(i, 2) * e(j, 2) * km1pd * km1pd / (2.0 * ra);
            I[q] = c.re;
        }
        return;
    }
    const double urm = W.ur[m - 1], uzm = W.uz[m - 1], tzm = W.tz[m - 1], trm = W.tr[m - 1];
    if (typelyr < 0) {
        const cx kmpu = ei(1, 1) * urm + ei(1, 2) * uzm + ei(1, 3) * tzm + ei(1, 4) * trm;
        const cx kmsu = ei(2, 1) * urm + ei(2, 2) * uzm + ei(2, 3) * tzm + ei(2, 4) * trm;
        for (int q = 0; q < 6; q++) {
            const int i = II[q], j = JJ[q];
            const cx c = e(i, 1) * e(j, 1) * kmpu * kmpu / (2.0 * ra)
                       + (e(i, 1) * e(j, 2) + e(i, 2) * e(j, 1)) * kmpu * kmsu / (ra + rb)
                       + e(i, 2) * e(j, 2) * kmsu * kmsu / (2.0 * rb);
            I[q] = c.re;
        }
    } else if (typelyr == 0) {
        const double urp = W.ur[m], uzp = W.uz[m], tzp = W.tz[m], trp = W.tr[m];
        const cx km1pd = ei(3, 1) * urm + ei(3, 2) * uzm + ei(3, 3) * tzm + ei(3, 4) * trm;
        const cx km1sd = ei(4, 1) * urm + ei(4, 2) * uzm + ei(4, 3) * tzm + ei(4, 4) * trm;
        const cx kmpu = ei(1, 1) * urp + ei(1, 2) * uzp + ei(1, 3) * tzp + ei(1, 4) * trp;
        const cx kmsu = ei(2, 1) * urp + ei(2, 2) * uzp + ei(2, 3) * tzp + ei(2, 4) * trp;
        const cx FA = ffunc(ra, zd);
        const cx GA = gfunc(ra, zd);
        const cx FB = ffunc(rb, zd);
        const cx GB = gfunc(rb, zd);
        const cx H1 = h1func(ra, rb, zd);
        const cx H2 = h2func(ra, rb, zd);
        for (int q = 0; q < 6; q++) {
            const int i = II[q], j = JJ[q];
            const cx c = e(i, 1) * e(j, 1) * kmpu * kmpu * FA
                       + e(i, 3) * e(j, 3) * km1pd * km1pd * FA
                       + e(i, 2) * e(j, 2) * kmsu * kmsu * FB
                       + e(i, 4) * e(j, 4) * km1sd * km1sd * FB
                       + H1 * ((e(i, 1) * e(j, 2) + e(i, 2) * e(j, 1)) * kmpu * kmsu
                               + (e(i, 3) * e(j, 4) + e(i, 4) * e(j, 3)) * km1pd * km1sd)
                       + H2 * ((e(i, 1) * e(j, 4) + e(i, 4) * e(j, 1)) * kmpu * km1sd
                               + (e(i, 2) * e(j, 3) + e(i, 3) * e(j, 2)) * km1pd * kmsu)
                       + GA * (e(i, 1) * e(j, 3) + e(i, 3) * e(j, 1)) * kmpu * km1pd
                       + GB * (e(i, 2) * e(j, 4) + e(i, 4) * e(j, 2)) * kmsu * km1sd;
            I[q] = c.re;
        }
    } else {
        const cx km1pd = ei(3, 1) * urm + ei(3, 2) * uzm + ei(3, 3) * tzm + ei(3, 4) * trm;
        const cx km1sd = ei(4, 1) * urm + ei(4, 2) * uzm + ei(4, 3) * tzm + ei(4, 4) * trm;
        for (int q = 0; q < 6; q++) {
            const int i = II[q], j = JJ[q];
            const cx c = e(i, 3) * e(j, 3) * km1pd * km1pd / (2.0 * ra)
                       + (e(i, 3) * e(j, 4) + e(i, 4) * e(j, 3)) * km1pd * km1sd / (ra + rb)
                       + e(i, 4) * e(j, 4) * km1sd * km1sd / (2.0 * rb);
            I[q] = c.re;
        }
    }
}

// sregn96.f90:1061-1203 (getmat :1538-1590) followed by the 1/(U I0) scaling.
__device__ inline double energy(RW& W, double om, double wvno, double& ugr, double& fac) {
    double sumi0 = 0.0, sumi1 = 0.0, sumi2 = 0.0, sumi3 = 0.0;
    const double c = om / wvno;
    const double om2 = om * om;
    const double wvno2 = wvno * wvno;
    for (int m = 1; m <= W.mmax; m++) {
        double a12 = 0, a14 = 0, a21 = 0, a23 = 0, ah, av, bv, eta, rho, TA, TC, TF, TL, TN;
        if (W.iwat[m - 1] == 1) {
            ah = W.za[m - 1];
            av = W.za[m - 1];
            bv = 0.0;
            rho = W.zrho[m - 1];
            eta = 1.0;
            TL = 0.0;
            TN = 0.0;
            TC = W.zrho[m - 1] * W.za[m - 1] * W.za[m - 1];
            TA = W.zrho[m - 1] * W.za[m - 1] * W.za[m - 1];
            TF = TA - 2.0 * TN;
            a12 = -(wvno * wvno - om * om / (ah * ah)) / (rho * om * om);
        } else {
            ah = W.za[m - 1];
            av = W.za[m - 1];
            bv = W.zb[m - 1];
            rho = W.zrho[m - 1];
            eta = 1.0;
            TL = W.zrho[m - 1] * W.zb[m - 1] * W.zb[m - 1];
            TN = W.zrho[m - 1] * W.zb[m - 1] * W.zb[m - 1];
            TC = W.zrho[m - 1] * W.za[m - 1] * W.za[m - 1];
            TA = W.zrho[m - 1] * W.za[m - 1] * W.za[m - 1];
            TF = TA - 2.0 * TN;
            a12 = -wvno;
            a14 = 1.0 / TL;
            a21 = wvno * TF / TC;
            a23 = 1.0 / TC;
        }
        const int typelyr = (m == W.mmax) ? 1 : 0;
        double I[6];
        layer_integrals(W, m, typelyr, om, om2, wvno, wvno2, I);
        const double INT11 = I[0], INT13 = I[1], INT22 = I[2], INT24 = I[3], INT33 = I[4],
                     INT44 = I[5];
        if (W.iwat[m - 1] == 1) {
            const double wr = wvno / (rho * om2);
            const double URUR = INT22 * (wr * wr);
            const double UZUZ = INT11;
            const double URDUZ = -(wvno / (rho * om2)) * a12 * INT22;
            const double DUZDUZ = a12 * a12 * INT22;
            sumi0 = sumi0 + rho * (URUR + UZUZ);
            sumi1 = sumi1 + TA * URUR;
            sumi2 = sumi2 - TF * URDUZ;
            sumi3 = sumi3 + TC * DUZDUZ;
            const double facah = rho * ah * ah * (URUR - 2.0 * eta * URDUZ / wvno);
            const double facav = rho * av * av * DUZDUZ / wvno2;
            W.dcda[m - 1] = facah + facav;
            W.dcdb[m - 1] = 0.0;
            const double facr = -(0.5 * c * c * (URUR + UZUZ));
            W.dcdr[m - 1] = 0.5 * (av * facav + ah * facah) + facr * rho;
            W.dcdgc[m - 1] = 0.0;
            W.ur[m - 1] = -(wvno * W.tz[m - 1]) / (rho * om2);
        } else {
            const double URUR = INT11;
            const double UZUZ = INT22;
            const double DURDUR = a12 * a12 * INT22 + 2.0 * a12 * a14 * INT24 + a14 * a14 * INT44;
            const double DUZDUZ = a21 * a21 * INT11 + 2.0 * a21 * a23 * INT13 + a23 * a23 * INT33;
            const double URDUZ = a21 * INT11 + a23 * INT13;
            const double UZDUR = a12 * INT22 + a14 * INT24;
            sumi0 = sumi0 + rho * (URUR + UZUZ);
            sumi1 = sumi1 + TL * UZUZ + TA * URUR;
            sumi2 = sumi2 + TL * UZDUR - TF * URDUZ;
            sumi3 = sumi3 + TL * DURDUR + TC * DUZDUZ;
            const double facah = rho * ah * ah * (URUR - 2.0 * eta * URDUZ / wvno);
            const double facav = rho * av * av * DUZDUZ / wvno2;
            const double facbh = 0.0;
            const double facbv =
                rho * bv * bv * (UZUZ + 2.0 * UZDUR / wvno + DURDUR / wvno2 + 4.0 * eta * URDUZ / wvno);
            W.dcda[m - 1] = facah + facav;
            W.dcdb[m - 1] = facbv + facbh;
            const double facr = -(0.5 * c * c * (URUR + UZUZ));
            W.dcdr[m - 1] = 0.5 * (av * facav + ah * facah + bv * facbv) + facr * rho;
            W.dcdgc[m - 1] = rho * bv * bv * (UZUZ + 2.0 * UZDUR / wvno + DURDUR / wvno2)
                           + rho * bv * bv * (URUR);
        }
    }
    ugr = (wvno * sumi1 + sumi2) / (om * sumi0);
    const double are = wvno / (2.0 * om * ugr * sumi0);
    fac = are * c / wvno2;
    for (int m = 0; m < W.mmax; m++) {
        W.dcda[m] = W.dcda[m] / (ugr * sumi0);
        W.dcdb[m] = W.dcdb[m] / (ugr * sumi0);
        W.dcdr[m] = W.dcdr[m] / (ugr * sumi0);
        W.dcdgc[m] = W.dcdgc[m] / (ugr * sumi0);
    }
    return sumi0;
}

// ---------------------------------------------------------------------------
// slegn96 / slegnpu: Love-wave eigenfunctions and depth kernels
// (src/surfker/slegn96.f90, modules LoveWaveModel / LoveWaveKernel)
// ---------------------------------------------------------------------------
struct LW {
    int mmax;
    double zd[MMAX], zb[MMAX], zrho[MMAX], xmu[MMAX], uu[MMAX], tt[MMAX], exl[MMAX];
    double dcdb[MMAX], dcdr[MMAX];
    double cosq, sinq, yl, zl, mu;
    double sumi0, sumi1, sumi2, ugr;
};

// pi of both Love drivers: a REAL*4 value (slegn96.f90:689, :808)
constexpr double kLovePiF = (double)3.1415926535898f;

// The model (slegn96.f90:697-716, :834-852) with bldsph (:107-167) from the
// per-layer constants; group: iwat from zb > 0, phase: from zb == 0 (the
// same for the models here, which have no water).
__device__ inline void lv_model(LW& W, const float* vs, const float* rho, const LayerConst& L) {
    W.mmax = L.mmax;
    for (int i = 0; i < L.mmax; i++) {
        W.zb[i] = (double)vs[i] * L.rg_vtp[i];
        W.zrho[i] = (double)rho[i] * L.lv_rtp[i];
        W.zd[i] = L.rg_zd[i];
        W.xmu[i] = W.zrho[i] * (W.zb[i] * W.zb[i]);
    }
}

// varl (:248-328)
__device__ inline void lv_varl(LW& W, int m, double& rb, double omega, double wvno, double& xkb,
                               double dpth, double& eexl) {
    xkb = omega / W.zb[m];
    const double wvnop = wvno + xkb;
    const double wvnom = fabs(wvno - xkb);
    rb = sqrt(wvnop * wvnom);
    const double q = rb * dpth;
    W.mu = W.zrho[m] * W.zb[m] * W.zb[m];
    eexl = 0.0;
    if (wvno < xkb) {
        sk_sincos(q, &W.sinq, &W.cosq);
        W.yl = W.sinq / rb;
        W.zl = -(rb * W.sinq);
    } else if (wvno == xkb) {
        W.cosq = 1.0;
        W.yl = dpth;
        W.zl = 0.0;
    } else if (wvno > xkb) {
        eexl = q;
        double fac = 0.0;
        if (q < 18.0) fac = sk_exp(-2.0 * q);
        W.cosq = (1.0 + fac) * 0.5;
        W.sinq = (1.0 - fac) * 0.5;
        W.yl = W.sinq / rb;
        W.zl = rb * W.sinq;
    }
}

// shfunc (:179-246) with up (:372-445) and hskl (:330-351)
static __device__ SK_NOINLINE_EIG void lv_shfunc(LW& W, double omega, double wvno) {
    const int mmax = W.mmax;
    double rb = 0, xkb = 0, eexl = 0;
    if (W.zb[mmax - 1] > (double)0.01f) {
        lv_varl(W, mmax - 1, rb, omega, wvno, xkb, 0.0, eexl);
        W.uu[mmax - 1] = 1.0;
        W.tt[mmax - 1] = -(W.xmu[mmax - 1] * rb);
    } else {
        W.uu[mmax - 1] = 1.0;
        W.tt[mmax - 1] = 0.0;
    }
    W.exl[mmax - 1] = 0.0;
    for (int k = mmax - 2; k >= 0; k--) {
        lv_varl(W, k, rb, omega, wvno, xkb, W.zd[k], eexl);
        const double a11 = W.cosq, a22 = W.cosq, a12 = -(W.yl / W.mu), a21 = -(W.zl * W.mu);
        const double amp0 = a11 * W.uu[k + 1] + a12 * W.tt[k + 1];
        const double str0 = a21 * W.uu[k + 1] + a22 * W.tt[k + 1];
        double rr = fabs(amp0);
        const double ss = fabs(str0);
        if (ss > rr) rr = ss;
        if (rr < 1.e-30) rr = 1.0;
        W.exl[k] = sk_log(rr) + eexl;
        W.uu[k] = amp0 / rr;
        W.tt[k] = str0 / rr;
    }
    double ext = 0.0;
    double umax = W.uu[0];
    W.tt[0] = 0.0;
    for (int k = 1; k < mmax; k++) {
        ext = ext + W.exl[k - 1];
        double fact = 0.0;
        if (ext < 80.0) fact = 1.0 / sk_exp(ext);
        W.uu[k] = W.uu[k] * fact;
        W.tt[k] = W.tt[k] * fact;
        if (fabs(W.uu[k]) > fabs(umax)) umax = W.uu[k];
    }
    if (W.uu[0] != 0.0) umax = W.uu[0];
    if (fabs(umax) > 0.0)
        for (int k = 0; k < mmax; k++) {
            W.uu[k] = W.uu[k] / umax;
            W.tt[k] = W.tt[k] / umax;
        }
}

// energy (:447-629): velocity and density kernels (dc/db, dc/drho) and the
// energy integrals
static __device__ SK_NOINLINE_EIG void lv_energy(LW& W, double omega, double wvno) {
    const int mmax = W.mmax;
    const double c = omega / wvno;
    const double wvno2 = wvno * wvno;
    W.sumi0 = W.sumi1 = W.sumi2 = 0.0;
    for (int k = 0; k < mmax; k++) {
        const double TN = W.zrho[k] * W.zb[k] * W.zb[k];
        const double TL = W.zrho[k] * W.zb[k] * W.zb[k];
        const double VSHH = W.zb[k], VSHV = W.zb[k];
        const double drho = W.zrho[k];
        const double dpth = W.zd[k];
        double rb = 0, xkb = 0, eexl = 0;
        lv_varl(W, k, rb, omega, wvno, xkb, dpth, eexl);
        const double dmu = W.xmu[k];
        if (rb < 1.0e-10) rb = 1.0e-10;
        double upup, dupdup;
        if (k == mmax - 1) {
            upup = (0.5 / rb) * W.uu[mmax - 1] * W.uu[mmax - 1];
            dupdup = (0.5 * rb) * W.uu[mmax - 1] * W.uu[mmax - 1];
        } else {
            cx nub = C(rb, 0.0);
            if (wvno < xkb) nub = C(0.0, rb);
            const cx xnub = dmu * nub;
            // emat (:353-370)
            const cx wx = wvno * xnub;
            const cx ei11 = C(0.5 / wvno), ei12 = C(0.5) / wx, ei21 = C(0.5 / wvno),
                     ei22 = -(C(0.5) / wx);
            const cx el11 = C(wvno), el12 = C(wvno);
            const cx km1dn = ei21 * W.uu[k] + ei22 * W.tt[k];
            const cx kmup = ei11 * W.uu[k + 1] + ei12 * W.tt[k + 1];
            const cx f3 = nub * dpth;
            cx exqq = C(0.0);
            if (f3.re < 40.0) exqq = cexp_(-2.0 * f3);
            const cx f = (1.0 - exqq) / (2.0 * nub);
            exqq = C(0.0);
            if (f3.re < 75.0) exqq = cexp_(-f3);
            const cx g = dpth * exqq;
            const cx f1 = f * (el11 * el11 * kmup * kmup + el12 * el12 * km1dn * km1dn);
            const cx f2 = g * (el11 * el12 + el11 * el12) * kmup * km1dn;
            upup = (f1 + f2).re;
            dupdup = (nub * nub * (f1 - f2)).re;
        }
        W.sumi0 = W.sumi0 + drho * upup;
        W.sumi1 = W.sumi1 + TN * upup;
        W.sumi2 = W.sumi2 + TL * dupdup;
        const double DCDBH = c * drho * VSHH * upup;
        const double DCDBV = c * drho * VSHV * dupdup / wvno2;
        W.dcdb[k] = DCDBH + DCDBV;
        W.dcdr[k] = 0.5 * c * (-(c * c * upup) + VSHH * VSHH * upup + VSHV * VSHV * dupdup / wvno2);
    }
    for (int k = 0; k < mmax; k++) {
        W.dcdb[k] = W.dcdb[k] / W.sumi1;
        W.dcdr[k] = W.dcdr[k] / W.sumi1;
    }
    W.ugr = W.sumi1 / (c * W.sumi0);
}

}  // namespace sk
}  // namespace sa