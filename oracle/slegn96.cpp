// CPU oracle: slegn96 / slegnpu Love-wave eigenfunctions and depth kernels.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Restates src/surfker/slegn96.f90 (modules LoveWaveModel, LoveWaveKernel)
// operation for operation: complex arithmetic as gfortran lowers it
// (ocomplex.h), REAL*4 islands kept -- the model arrives as REAL*4, pi is the
// REAL*4 literal 3.1415926535898 (slegn96) or 4*atan(1.0) in REAL*4
// (slegnpu), both the same float; the threshold 0.01 is REAL*4.  Only the
// velocity and density kernels (and what they depend on) are formed; the
// layer-thickness kernels are not used by the reference's callers.
#include "oracle.h"
#include "omath.h"
#include "ocomplex.h"

#include <cmath>
#include <vector>

namespace {

// module LoveWaveModel (slegn96.f90:55-170), one instance per call
struct LW {
    int mmax = 0;
    std::vector<double> zd, zb, zrho, xmu, uu, tt, dcdb, dcdr, exl, vtp, dtp, rtp;
    std::vector<int> iwat;
    double cosq = 0, sinq = 0, yl = 0, zl = 0, mu = 0;
    double sumi0 = 0, sumi1 = 0, sumi2 = 0, flagr = 0, ale = 0, ugr = 0;
    explicit LW(int n)
        : mmax(n), zd(n), zb(n), zrho(n), xmu(n), uu(n), tt(n), dcdb(n), dcdr(n), exl(n),
          vtp(n), dtp(n), rtp(n), iwat(n) {}
};

// bldsph (:107-167): Love-wave earth flattening; rtp = tmp**(-5) as gfortran
// expands the integer power (x^5 = x^3 * x^2, then the reciprocal)
void bldsph(LW& W) {
    const double ar = 6371.0;
    double dr = 0.0, r0 = ar;
    W.zd[W.mmax - 1] = 1.0;
    for (int i = 0; i < W.mmax; i++) {
        dr = dr + W.zd[i];
        const double r1 = ar - dr;
        const double z0 = ar * std::log(ar / r0);
        const double z1 = ar * std::log(ar / r1);
        W.dtp[i] = ar / r0;
        const double tmp = (2.0 * ar) / (r0 + r1);
        W.vtp[i] = tmp;
        const double x2 = tmp * tmp, x3 = x2 * tmp, x5 = x3 * x2;
        W.rtp[i] = 1.0 / x5;
        W.zb[i] = W.zb[i] * tmp;
        W.zrho[i] = W.zrho[i] * W.rtp[i];
        W.zd[i] = z1 - z0;
        r0 = r1;
    }
    W.zd[W.mmax - 1] = 0.0;
}

// varl (:248-328)
void varl(LW& W, int m, double& rb, double omega, double wvno, double& xkb, double dpth,
          double& eexl) {
    xkb = omega / W.zb[m];
    const double wvnop = wvno + xkb;
    const double wvnom = std::abs(wvno - xkb);
    rb = std::sqrt(wvnop * wvnom);
    const double q = rb * dpth;
    W.mu = W.zrho[m] * W.zb[m] * W.zb[m];
    eexl = 0.0;
    if (wvno < xkb) {
        W.sinq = om::sin(q);
        W.yl = W.sinq / rb;
        W.zl = -(rb * W.sinq);
        W.cosq = om::cos(q);
    } else if (wvno == xkb) {
        W.cosq = 1.0;
        W.yl = dpth;
        W.zl = 0.0;
    } else if (wvno > xkb) {
        eexl = q;
        double fac = 0.0;
        if (q < 18.0) fac = om::exp(-2.0 * q);
        W.cosq = (1.0 + fac) * 0.5;
        W.sinq = (1.0 - fac) * 0.5;
        W.yl = W.sinq / rb;
        W.zl = rb * W.sinq;
    }
}

// up (:372-445), hskl (:330-351) inline: A^-1 of the Haskell matrix
double up(LW& W, double omega, double wvno) {
    const int mmax = W.mmax;
    double rb = 0, xkb = 0, eexl = 0;
    if (W.zb[mmax - 1] > static_cast<double>(0.01f)) {
        varl(W, mmax - 1, rb, omega, wvno, xkb, 0.0, eexl);
        W.uu[mmax - 1] = 1.0;
        W.tt[mmax - 1] = -(W.xmu[mmax - 1] * rb);
    } else {
        W.uu[mmax - 1] = 1.0;
        W.tt[mmax - 1] = 0.0;
    }
    W.exl[mmax - 1] = 0.0;
    double ttlast = 0.0;
    for (int k = mmax - 2; k >= 0; k--) {
        if (W.iwat[k] != 0) continue;
        varl(W, k, rb, omega, wvno, xkb, W.zd[k], eexl);
        const double h11 = W.cosq, h12 = W.yl / W.mu, h21 = W.zl * W.mu, h22 = W.cosq;
        const int k1 = k + 1;
        const double a11 = h11, a22 = h22, a12 = -h12, a21 = -h21;
        const double amp0 = a11 * W.uu[k1] + a12 * W.tt[k1];
        const double str0 = a21 * W.uu[k1] + a22 * W.tt[k1];
        double rr = std::abs(amp0);
        const double ss = std::abs(str0);
        if (ss > rr) rr = ss;
        if (rr < 1.e-30) rr = 1.0;
        W.exl[k] = om::log(rr) + eexl;
        W.uu[k] = amp0 / rr;
        W.tt[k] = str0 / rr;
        ttlast = W.tt[k];
    }
    return ttlast;
}

// shfunc (:179-246)
void shfunc(LW& W, double omega, double wvno) {
    up(W, omega, wvno);
    double ext = 0.0;
    double umax = W.uu[0];
    W.tt[0] = 0.0;
    for (int k = 1; k < W.mmax; k++) {
        if (W.iwat[k] == 0) {
            ext = ext + W.exl[k - 1];
            double fact = 0.0;
            if (ext < 80.0) fact = 1.0 / om::exp(ext);
            W.uu[k] = W.uu[k] * fact;
            W.tt[k] = W.tt[k] * fact;
        } else {
            W.uu[k] = 0.0;
            W.tt[k] = 0.0;
        }
        if (std::abs(W.uu[k]) > std::abs(umax)) umax = W.uu[k];
    }
    if (W.uu[0] != 0.0) umax = W.uu[0];
    if (std::abs(umax) > 0.0)
        for (int k = 0; k < W.mmax; k++)
            if (W.iwat[k] == 0) {
                W.uu[k] = W.uu[k] / umax;
                W.tt[k] = W.tt[k] / umax;
            }
}

// energy (:447-629): the velocity and density kernels and the integrals
void energy(LW& W, double omega, double wvno) {
    const int mmax = W.mmax;
    const double c = omega / wvno;
    const double omega2 = omega * omega;
    const double wvno2 = wvno * wvno;
    W.sumi0 = W.sumi1 = W.sumi2 = 0.0;
    for (int k = 0; k < mmax; k++) {
        if (W.iwat[k] != 0) {
            W.dcdb[k] = 0.0;
            W.dcdr[k] = 0.0;
            continue;
        }
        const double TN = W.zrho[k] * W.zb[k] * W.zb[k];
        const double TL = W.zrho[k] * W.zb[k] * W.zb[k];
        const double VSHH = W.zb[k], VSHV = W.zb[k];
        const int k1 = k + 1;
        const double drho = W.zrho[k];
        const double dpth = W.zd[k];
        double rb = 0, xkb = 0, eexl = 0;
        varl(W, k, rb, omega, wvno, xkb, dpth, eexl);
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
            const cx kmup = ei11 * W.uu[k1] + ei12 * W.tt[k1];
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
        if (W.iwat[k] == 0) {
            W.dcdb[k] = W.dcdb[k] / W.sumi1;
            W.dcdr[k] = W.dcdr[k] / W.sumi1;
        } else {
            W.dcdb[k] = 0.0;
            W.dcdr[k] = 0.0;
        }
    }
    W.flagr = omega2 * W.sumi0 - wvno2 * W.sumi1 - W.sumi2;
    W.ugr = W.sumi1 / (c * W.sumi0);
    W.ale = 0.5 / W.sumi1;
}

// the model of slegn96 / slegnpu (:697-716, :834-852)
void load_model(LW& W, const float* thk, const float* vs, const float* rhom, bool group,
                int iflsph) {
    for (int i = 0; i < W.mmax; i++) {
        W.zb[i] = vs[i];
        W.zrho[i] = rhom[i];
        W.zd[i] = thk[i];
        W.iwat[i] = group ? (W.zb[i] > 0.0 ? 0 : 1) : (W.zb[i] == 0.0 ? 1 : 0);
    }
    if (iflsph > 0) bldsph(W);
    for (int i = 0; i < W.mmax; i++) W.xmu[i] = W.zrho[i] * (W.zb[i] * W.zb[i]);
}

// pi of both drivers: a REAL*4 value (slegn96.f90:689, :808)
const double kPiF = static_cast<double>(3.1415926535898f);

}  // namespace

// slegn96 (:672-783): Love phase kernels dc/db, dc/drho (as dimensionless
// b dc/db, rho dc/drho) at the phase velocity cp, earth-flattening corrected
// (splove, :631-670) when iflsph > 0.
extern "C" void orc_slegn96(const float* thk, const float* vs, const float* rhom, int nlayer,
                            double t, double cp, double* cg, double* dc2db, double* dc2dr,
                            int iflsph) {
    LW W(nlayer);
    load_model(W, thk, vs, rhom, false, iflsph);
    const double twopi = 2.0 * kPiF;
    const double omega = twopi / t;
    const double c = cp;
    const double wvno = omega / c;
    shfunc(W, omega, wvno);
    energy(W, omega, wvno);
    double usph = W.ugr;
    if (iflsph > 0) {
        const double a = 6371.0;
        const double x = (3.0 * c) / ((2.0 * a) * omega);
        const double tm = std::sqrt(1.0 + x * x);
        const double tm3 = tm * tm * tm;
        for (int i = 0; i < W.mmax; i++) {
            W.dcdb[i] = W.dcdb[i] * W.vtp[i] / tm3;
            W.dcdr[i] = W.dcdr[i] * W.rtp[i] / tm3;
        }
        usph = W.ugr * tm;
    }
    for (int i = 0; i < W.mmax; i++) {
        dc2db[i] = W.dcdb[i];
        dc2dr[i] = W.dcdr[i];
    }
    if (cg) *cg = usph;
}

// slegnpu (:785-919): Love group kernels du/db, du/drho from the phase
// kernels at t, t1, t2 (the first term reads the t2 evaluation's kernels, as
// the Fortran's module arrays do), earth-flattening corrected.
extern "C" void orc_slegnpu(const float* thk, const float* vs, const float* rhom, int nlayer,
                            double t, double cp, double t1, double cp1, double t2, double cp2,
                            double* cg_out, double* du2db, double* du2dr, int iflsph) {
    LW W(nlayer);
    load_model(W, thk, vs, rhom, true, iflsph);
    const int mmax = W.mmax;
    const double twopi = 2.0 * kPiF;
    double omega = twopi / t;
    double wvno = omega / cp;
    shfunc(W, omega, wvno);
    energy(W, omega, wvno);
    const double cg = W.ugr;
    const std::vector<double> dc2db = W.dcdb, dc2dr = W.dcdr;
    omega = twopi / t1;
    wvno = omega / cp1;
    shfunc(W, omega, wvno);
    energy(W, omega, wvno);
    const std::vector<double> dc2db1 = W.dcdb, dc2dr1 = W.dcdr;
    omega = twopi / t2;
    wvno = omega / cp2;
    shfunc(W, omega, wvno);
    energy(W, omega, wvno);
    const std::vector<double> dc2db2 = W.dcdb, dc2dr2 = W.dcdr;
    const double uc1 = cg / cp;
    for (int i = 0; i < mmax; i++) {
        du2db[i] = uc1 * (2.0 - uc1) * W.dcdb[i] - uc1 * uc1 * t * (dc2db2[i] - dc2db1[i]) / (t2 - t1);
        du2dr[i] = uc1 * (2.0 - uc1) * W.dcdr[i] - uc1 * uc1 * t * (dc2dr2[i] - dc2dr1[i]) / (t2 - t1);
    }
    double cgs = cg;
    if (iflsph > 0) {
        const double ar = 6371.0;
        omega = twopi / t;
        const double x = (3.0 * cp) / ((2.0 * ar) * omega);
        const double tm = std::sqrt(1.0 + x * x);
        const double y = 1.5 / (ar * omega);
        const double tm1 = (y * y) / tm;
        for (int i = 0; i < mmax; i++) {
            du2db[i] = (tm * du2db[i] + cg * cp * dc2db[i] * tm1) * W.vtp[i];
            du2dr[i] = (tm * du2dr[i] + cg * cp * dc2dr[i] * tm1) * W.rtp[i];
        }
        cgs = cg * tm;
    }
    if (cg_out) *cg_out = cgs;
}
