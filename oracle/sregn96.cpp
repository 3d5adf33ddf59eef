// CPU oracle: sregn96 / sregn96_hti Rayleigh eigenfunctions and depth kernels.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Restates src/surfker/sregn96.f90.  Complex arithmetic follows gfortran's
// lowering: complex*complex is the plain (ac-bd, ad+bc) product, a real operand
// scales both parts, and complex/complex uses the range-reduced (Smith) form
// that gfortran emits by default.  REAL*4 islands (sngl() arguments, default
// literals) are kept.
#include "oracle.h"
#include "omath.h"
#include "ocomplex.h"

#include <cmath>
#include <vector>

namespace {

// module RayleighWaveModel (sregn96.f90:55-185), one instance per call
struct RW {
    int mmax;
    std::vector<double> zd, zrho, za, zb, xmu, xlam;
    std::vector<double> ur, uz, tz, tr, dcda, dcdb, dcdr, dcdh, dcdgc, dcdgs;
    std::vector<int> iwat;
    double sumi0, sumi1, sumi2, sumi3, flagr, are, ugr;
    std::vector<double> vtp, dtp, rtp;
    std::vector<double> exe, exa;
    std::vector<double> cd;   // cd(mmax,5): cd[(i)*5 + j]
    std::vector<double> vv;   // vv(mmax,4): vv[(i)*4 + j]
    bool allfluid;
    cx ra, rb;
    cx e[4][4], einv[4][4];
    double CD(int i, int j) const { return cd[(i - 1) * 5 + (j - 1)]; }
    double& CD(int i, int j) { return cd[(i - 1) * 5 + (j - 1)]; }
    double VV(int i, int j) const { return vv[(i - 1) * 4 + (j - 1)]; }
    double& VV(int i, int j) { return vv[(i - 1) * 4 + (j - 1)]; }
};

// sregn96.f90:129-183
void bldsph(RW& W) {
    const double ar = 6371.0;
    double dr = 0.0;
    double r0 = ar;
    const double expo = static_cast<double>(-2.275f);
    for (int i = 1; i <= W.mmax; i++) {
        if (i == W.mmax) dr = dr + 1.0;
        else dr = dr + W.zd[i - 1];
        const double r1 = ar - dr;
        const double z0 = ar * std::log(ar / r0);
        const double z1 = ar * std::log(ar / r1);
        const double tmp = (2.0 * ar) / (r0 + r1);
        W.vtp[i - 1] = tmp;
        W.rtp[i - 1] = std::pow(tmp, expo);
        W.dtp[i - 1] = ar / r0;
        W.za[i - 1] = W.za[i - 1] * tmp;
        W.zb[i - 1] = W.zb[i - 1] * tmp;
        W.zrho[i - 1] = W.zrho[i - 1] * W.rtp[i - 1];
        W.zd[i - 1] = z1 - z0;
        r0 = r1;
    }
    W.zd[W.mmax - 1] = 0.0;
}

// sregn96.f90:827-911
struct VarSv {
    double cosp, cosq, rsinp, rsinq, sinpr, sinqr, pex, svex;
};
VarSv varsv(cx p, cx q, cx rp, cx rsv, int iwat, double zd) {
    VarSv o;
    const double lim = static_cast<double>(1.0e-5f);
    o.pex = 0.0;
    o.svex = 0.0;
    const double pr = p.re, pi = p.im, qr = q.re, qi = q.im;
    o.pex = pr;
    const cx epp = C(om::cos(pi), om::sin(pi)) / 2.0;
    const cx epm = conj_(epp);
    double pfac;
    if (pr < 30.0) pfac = om::exp(-(2.0 * pr));
    else pfac = 0.0;
    o.cosp = (epp + pfac * epm).re;
    const cx sinp = epp - pfac * epm;
    o.rsinp = (rp * sinp).re;
    if (std::abs(pr) < lim && cabs_(rp) < lim) o.sinpr = zd;
    else o.sinpr = (sinp / rp).re;
    if (iwat == 1) {
        o.cosq = 1.0;
        o.rsinq = 0.0;
        o.sinqr = 0.0;
    } else {
        o.svex = qr;
        const cx eqp = C(om::cos(qi), om::sin(qi)) / 2.0;
        const cx eqm = conj_(eqp);
        double svfac;
        if (qr < 30.0) svfac = om::exp(-(2.0 * qr));
        else svfac = 0.0;
        o.cosq = (eqp + svfac * eqm).re;
        const cx sinq = eqp - svfac * eqm;
        o.rsinq = (rsv * sinq).re;
        if (std::abs(qr) < lim && cabs_(rsv) < lim) o.sinqr = zd;
        else o.sinqr = (sinq / rsv).re;
    }
    return o;
}

// sregn96.f90:491-647; ca[j][i] holds Fortran ca(j+1,i+1)
void dnka(double ca[5][5], double cosp, double rsinp, double sinpr, double cossv, double rsinsv,
          double sinsvr, float rho, float b, int iwat, double ex, double exa, double wvno,
          double wvno2, double om2) {
    if (iwat == 1) {
        for (int j = 0; j < 5; j++)
            for (int i = 0; i < 5; i++) ca[i][j] = 0.0;
        double dfac;
        if (ex > 35.0) dfac = 0.0;
        else dfac = om::exp(-ex);
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
    double a0;
    if (exa < 60.0) a0 = om::exp(-exa);
    else a0 = 0.0;
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
    const double gam = static_cast<double>(2.0f * b * b) * wvno2 / om2;
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
    const double rom2 = static_cast<double>(rho) * om2;
    double temp = a0c * gg1 + g2xz2 + g2wy2;
    ca[2][2] = a0 + temp + temp;
    ca[0][0] = cpcq - temp;
    ca[0][1] = (-cqx + wvno2 * cpy) / rom2;
    temp = 0.5 * a0cgg1 + gxz2 + g1wy2;
    ca[0][2] = wvno * temp / rom2;
    ca[0][3] = (-cqww2 + cpz) / rom2;
    temp = wvno2 * (a0c + wy2) + xz;
    ca[0][4] = -(temp / (static_cast<double>(rho2) * om2 * om2));
    ca[1][0] = (-(gamm2 * cqw) + gam2 * cpz / wvno2) * static_cast<double>(rho) * om2;
    ca[1][1] = cpcq;
    ca[1][2] = (gamm1 * cqww2 - gam * cpz) / wvno;
    ca[1][3] = -wz;
    ca[1][4] = ca[0][3];
    temp = 0.5 * a0cgg1 * gg1 + gam2 * gxz2 + gamm2 * g1wy2;
    ca[2][0] = -(2.0 * temp * static_cast<double>(rho) * om2 / wvno);
    ca[2][1] = -(wvno * (gam * cqxw2 - gamm1 * cpy) * 2.0);
    ca[2][3] = -2.0 * ca[1][2];
    ca[2][4] = -2.0 * ca[0][2];
    ca[3][0] = (-(gam2 * cqxw2) + gamm2 * cpy) * static_cast<double>(rho) * om2;
    ca[3][1] = -xy;
    ca[3][2] = -(ca[2][1] / 2.0);
    ca[3][3] = ca[1][1];
    ca[3][4] = ca[0][1];
    temp = gamm2 * (a0c * gam2 + g2wy2) + gam2 * g2xz2;
    ca[4][0] = -(static_cast<double>(rho2) * om2 * om2 * temp / wvno2);
    ca[4][1] = ca[3][0];
    ca[4][2] = -(ca[2][0] / 2.0);
    ca[4][3] = ca[1][0];
    ca[4][4] = ca[0][0];
}

// sregn96.f90:649-825 with jbdry = 0, inp = 1; gbr is the first row.
void evalg(RW& W, int m, cx gbr[5], double wvno, double om, double om2, double wvno2) {
    const double xka = om / W.za[m - 1];
    double xkb;
    if (W.zb[m - 1] > 0.0) xkb = om / W.zb[m - 1];
    else xkb = 0.0;
    W.ra = csqrt_real(wvno2 - xka * xka);
    W.rb = csqrt_real(wvno2 - xkb * xkb);
    const cx ra = W.ra, rb = W.rb;
    double gam = W.zb[m - 1] * wvno / om;
    gam = 2.0 * (gam * gam);
    const double gamm1 = gam - 1.0;
    const double zr = W.zrho[m - 1];
    auto& E = W.e;
    auto& EI = W.einv;
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

        gbr[0] = ((zr * zr) * om2 * om2) * (-((gam * gam) * ra * rb) + C(wvno2 * gamm1 * gamm1));
        gbr[1] = -((zr * (wvno2 * ra)) * om2);
        gbr[2] = -(((zr * (-((gam * ra) * rb) + C(wvno2 * gamm1))) * om2) * wvno);
        gbr[3] = (zr * (wvno2 * rb)) * om2;
        gbr[4] = wvno2 * (C(wvno2) - ra * rb);
        const cx den = -((((zr * zr) * om2 * om2 * wvno2) * ra) * rb);
        for (int k = 0; k < 5; k++) gbr[k] = (0.25 * gbr[k]) / den;
    } else {
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

// sregn96.f90:1406-1435
void normc(double* ee, double& ex, int nmat) {
    ex = 0.0;
    double t1 = 0.0;
    for (int i = 0; i < nmat; i++)
        if (std::abs(ee[i]) > t1) t1 = std::abs(ee[i]);
    if (t1 < 1.e-40) t1 = 1.0;
    for (int i = 0; i < nmat; i++) {
        double t2 = ee[i];
        t2 = t2 / t1;
        ee[i] = t2;
    }
    ex = om::log(t1);
}

// sregn96.f90:401-489
double up(RW& W, double omega, double wvno) {
    const double wvno2 = wvno * wvno;
    const double om2 = omega * omega;
    cx gbr[5];
    evalg(W, W.mmax, gbr, wvno, omega, om2, wvno2);
    for (int j = 1; j <= 5; j++) W.CD(W.mmax, j) = gbr[j - 1].re;
    W.exe[W.mmax - 1] = 0.0;
    double exsum = 0.0;
    double ca[5][5], ee[5];
    for (int m = W.mmax - 1; m >= 1; m--) {
        const double xka = omega / W.za[m - 1];
        double xkb;
        if (W.zb[m - 1] > 0.0) xkb = omega / W.zb[m - 1];
        else xkb = 0.0;
        const cx rp = csqrt_real(wvno2 - xka * xka);
        const cx rsv = csqrt_real(wvno2 - xkb * xkb);
        const cx p = rp * W.zd[m - 1];
        const cx q = rsv * W.zd[m - 1];
        const VarSv v = varsv(p, q, rp, rsv, W.iwat[m - 1], W.zd[m - 1]);
        dnka(ca, v.cosp, v.rsinp, v.sinpr, v.cosq, v.rsinq, v.sinqr,
             static_cast<float>(W.zrho[m - 1]), static_cast<float>(W.zb[m - 1]), W.iwat[m - 1],
             v.pex, v.pex + v.svex, wvno, wvno2, om2);
        for (int i = 0; i < 5; i++) {
            double cr = 0.0;
            for (int j = 0; j < 5; j++) cr = cr + W.CD(m + 1, j + 1) * ca[j][i];
            ee[i] = cr;
        }
        double exn = 0.0;
        normc(ee, exn, 5);
        exsum = exsum + v.pex + v.svex + exn;
        W.exe[m - 1] = exsum;
        for (int i = 0; i < 5; i++) W.CD(m, i + 1) = ee[i];
    }
    return W.CD(1, 1);
}

// sregn96.f90:913-987; AA[i][j] holds Fortran AA(i+1,j+1)
void hska(double AA[4][4], double cosp, double rsinp, double sinpr, double tcossv,
          double trsinsv, double tsinsvr, float rho, float b, int iwat, double pex, double svex,
          double wvno, double wvno2, double om2) {
    const double rom2 = static_cast<double>(rho) * om2;
    if (iwat == 1) {
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) AA[i][j] = 0.0;
        double dfac;
        if (pex > 35.0) dfac = 0.0;
        else dfac = om::exp(-pex);
        AA[0][0] = dfac;
        AA[3][3] = dfac;
        AA[1][1] = cosp;
        AA[2][2] = cosp;
        AA[1][2] = -(rsinp / rom2);
        AA[2][1] = -(rom2 * sinpr);
        return;
    }
    double dfac;
    if ((pex - svex) > 70.0) dfac = 0.0;
    else dfac = om::exp(svex - pex);
    const double cossv = dfac * tcossv;
    const double rsinsv = dfac * trsinsv;
    const double sinsvr = dfac * tsinsvr;
    const double gam = static_cast<double>(2.0f * b * b) * wvno2 / om2;
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
void down(RW& W, double omega, double wvno) {
    const double om2 = omega * omega;
    const double wvno2 = wvno * wvno;
    for (int i = 1; i <= 4; i++) W.VV(1, i) = (i == 1) ? 1.0 : 0.0;
    W.exa[0] = 0.0;
    double exsum = 0.0;
    double AA[4][4], aa0[4];
    for (int m = 1; m <= W.mmax - 1; m++) {
        const double xka = omega / W.za[m - 1];
        double xkb;
        if (W.zb[m - 1] > 0.0) xkb = omega / W.zb[m - 1];
        else xkb = 0.0;
        const cx rp = csqrt_real(wvno2 - xka * xka);
        const cx rsv = csqrt_real(wvno2 - xkb * xkb);
        const cx p = rp * W.zd[m - 1];
        const cx q = rsv * W.zd[m - 1];
        const VarSv v = varsv(p, q, rp, rsv, W.iwat[m - 1], W.zd[m - 1]);
        hska(AA, v.cosp, v.rsinp, v.sinpr, v.cosq, v.rsinq, v.sinqr,
             static_cast<float>(W.zrho[m - 1]), static_cast<float>(W.zb[m - 1]), W.iwat[m - 1],
             v.pex, v.svex, wvno, wvno2, om2);
        for (int i = 0; i < 4; i++) {
            double cc = 0.0;
            for (int j = 0; j < 4; j++) cc = cc + AA[i][j] * W.VV(m, j + 1);
            aa0[i] = cc;
        }
        double ex2 = 0.0;
        normc(aa0, ex2, 4);
        exsum = exsum + v.pex + ex2;
        W.exa[m] = exsum;
        for (int i = 0; i < 4; i++) W.VV(m + 1, i + 1) = aa0[i];
    }
}

// sregn96.f90:193-399
void svfunc(RW& W, double omega, double wvno) {
    const double fr = up(W, omega, wvno);
    (void)fr;
    down(W, omega, wvno);
    const double f1213 = -W.CD(1, 2);
    W.ur[0] = W.CD(1, 3) / W.CD(1, 2);
    W.uz[0] = 1.0;
    W.tz[0] = 0.0;
    W.tr[0] = 0.0;
    for (int i = 2; i <= W.mmax; i++) {
        const double cd1 = W.CD(i, 1);
        const double cd2 = W.CD(i, 2);
        const double cd3 = W.CD(i, 3);
        const double cd4 = -W.CD(i, 3);
        const double cd5 = W.CD(i, 4);
        const double cd6 = W.CD(i, 5);
        const double tz1 = -W.VV(i, 4);
        const double tz2 = -W.VV(i, 3);
        const double tz3 = W.VV(i, 2);
        const double tz4 = W.VV(i, 1);
        const double uu1 = tz2 * cd6 - tz3 * cd5 + tz4 * cd4;
        const double uu2 = -(tz1 * cd6) + tz3 * cd3 - tz4 * cd2;
        const double uu3 = tz1 * cd5 - tz2 * cd3 + tz4 * cd1;
        const double uu4 = -(tz1 * cd4) + tz2 * cd2 - tz3 * cd1;
        const double ext = W.exa[i - 1] + W.exe[i - 1] - W.exe[0];
        if (ext > -80.0 && ext < 80.0) {
            const double fact = om::exp(ext);
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

// sregn96.f90:1326-1404
cx ffunc(cx nub, double dm) {
    if (cabs_(nub) < 1.0e-08) return C(dm);
    const cx argcd = nub * dm;
    cx exqq;
    if (argcd.re < 40.0) exqq = cexp_(-(2.0 * argcd));
    else exqq = C(0.0);
    return (1.0 - exqq) / (2.0 * nub);
}
cx gfunc(cx nub, double dm) {
    const cx argcd = nub * dm;
    if (argcd.re < 75.0) return cexp_(-argcd) * dm;
    return C(0.0, 0.0);
}
cx h1func(cx nua, cx nub, double dm) {
    if (cabs_(nub + nua) < 1.0e-08) return C(dm);
    const cx argcd = (nua + nub) * dm;
    cx exqq;
    if (argcd.re < 40.0) exqq = cexp_(-argcd);
    else exqq = C(0.0);
    return (1.0 - exqq) / (nub + nua);
}
cx h2func(cx nua, cx nub, double dm) {
    if (cabs_(nub - nua) < 1.0e-08) return C(dm);
    cx argcd = nua * dm;
    cx exqp, exqq;
    if (argcd.re < 40.0) exqp = cexp_(-argcd);
    else exqp = C(0.0);
    argcd = nub * dm;
    if (argcd.re < 40.0) exqq = cexp_(-argcd);
    else exqq = C(0.0);
    return (exqq - exqp) / (nua - nub);
}

// sregn96.f90:1205-1324 (solid layers; fluid branches kept for completeness)
double intijr(RW& W, int i, int j, int m, int typelyr, double om, double om2, double wvno,
              double wvno2) {
    cx gbr[5];
    evalg(W, m, gbr, wvno, om, om2, wvno2);
    auto e = [&](int a, int b) { return W.e[a - 1][b - 1]; };
    auto ei = [&](int a, int b) { return W.einv[a - 1][b - 1]; };
    const cx ra = W.ra, rb = W.rb;
    const double zd = W.zd[m - 1];
    cx c;
    if (W.iwat[m - 1] == 1) {
        if (typelyr < 0) {
            const cx kmpu = ei(1, 1) * W.uz[m] + ei(1, 2) * W.tz[m];
            c = e(i, 1) * e(j, 1) * kmpu * kmpu / (2.0 * ra);
        } else if (typelyr == 0) {
            const cx km1pd = ei(2, 1) * W.uz[m - 1] + ei(2, 2) * W.tz[m - 1];
            const cx kmpu = ei(1, 1) * W.uz[m] + ei(1, 2) * W.tz[m];
            const cx FA = ffunc(ra, zd);
            const cx GA = gfunc(ra, zd);
            c = e(i, 1) * e(j, 1) * kmpu * kmpu * FA
              + (e(i, 1) * e(j, 2) + e(i, 2) * e(j, 1)) * kmpu * km1pd * GA
              + e(i, 2) * e(j, 2) * km1pd * km1pd * FA;
        } else {
            const cx km1pd = ei(2, 1) * W.uz[m - 1] + ei(2, 2) * W.tz[m - 1];
            c = e(i, 2) * e(j, 2) * km1pd * km1pd / (2.0 * ra);
        }
        return c.re;
    }
    const double urm = W.ur[m - 1], uzm = W.uz[m - 1], tzm = W.tz[m - 1], trm = W.tr[m - 1];
    if (typelyr < 0) {
        const cx kmpu = ei(1, 1) * urm + ei(1, 2) * uzm + ei(1, 3) * tzm + ei(1, 4) * trm;
        const cx kmsu = ei(2, 1) * urm + ei(2, 2) * uzm + ei(2, 3) * tzm + ei(2, 4) * trm;
        c = e(i, 1) * e(j, 1) * kmpu * kmpu / (2.0 * ra)
          + (e(i, 1) * e(j, 2) + e(i, 2) * e(j, 1)) * kmpu * kmsu / (ra + rb)
          + e(i, 2) * e(j, 2) * kmsu * kmsu / (2.0 * rb);
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
        c = e(i, 1) * e(j, 1) * kmpu * kmpu * FA
          + e(i, 3) * e(j, 3) * km1pd * km1pd * FA
          + e(i, 2) * e(j, 2) * kmsu * kmsu * FB
          + e(i, 4) * e(j, 4) * km1sd * km1sd * FB
          + H1 * ((e(i, 1) * e(j, 2) + e(i, 2) * e(j, 1)) * kmpu * kmsu
                  + (e(i, 3) * e(j, 4) + e(i, 4) * e(j, 3)) * km1pd * km1sd)
          + H2 * ((e(i, 1) * e(j, 4) + e(i, 4) * e(j, 1)) * kmpu * km1sd
                  + (e(i, 2) * e(j, 3) + e(i, 3) * e(j, 2)) * km1pd * kmsu)
          + GA * (e(i, 1) * e(j, 3) + e(i, 3) * e(j, 1)) * kmpu * km1pd
          + GB * (e(i, 2) * e(j, 4) + e(i, 4) * e(j, 2)) * kmsu * km1sd;
    } else {
        const cx km1pd = ei(3, 1) * urm + ei(3, 2) * uzm + ei(3, 3) * tzm + ei(3, 4) * trm;
        const cx km1sd = ei(4, 1) * urm + ei(4, 2) * uzm + ei(4, 3) * tzm + ei(4, 4) * trm;
        c = e(i, 3) * e(j, 3) * km1pd * km1pd / (2.0 * ra)
          + (e(i, 3) * e(j, 4) + e(i, 4) * e(j, 3)) * km1pd * km1sd / (ra + rb)
          + e(i, 4) * e(j, 4) * km1sd * km1sd / (2.0 * rb);
    }
    return c.re;
}

// sregn96.f90:1437-1536
void getdcdh(RW& W, double om2, double wvno, double wvno2, double fac) {
    for (int m = 1; m <= W.mmax; m++) {
        const double tuz = W.uz[m - 1];
        const double ttz = W.tz[m - 1];
        const double ttr = W.tr[m - 1];
        double tur;
        if (W.iwat[m - 1] == 1) tur = -(wvno * ttz) / (W.zrho[m - 1] * om2);
        else tur = W.ur[m - 1];
        double gfac1, gfac2, gfac3, gfac4, gfac5, gfac6;
        const double xm = W.xmu[m - 1], xl = W.xlam[m - 1];
        if (m == 1) {
            const double drho = W.zrho[0] - 0.0;
            const double dmu = W.xmu[0] - 0.0;
            const double dlm = W.xlam[0] - 0.0;
            const double dl2mu = dlm + dmu + dmu;
            const double xl2mp = xl + xm + xm;
            const double duzdzp = (ttz + wvno * xl * tur) / xl2mp;
            double durdzp;
            if (W.iwat[m - 1] == 1) durdzp = wvno * tuz;
            else durdzp = (ttr / xm) - wvno * tuz;
            const double drur2 = tur * tur * drho;
            const double dlur2 = tur * tur * dl2mu;
            gfac1 = om2 * drho * (tuz * tuz);
            gfac2 = om2 * drur2;
            gfac3 = -(wvno2 * dmu * (tuz * tuz));
            gfac4 = -(wvno2 * dlur2);
            gfac5 = (xl2mp * (duzdzp * duzdzp));
            gfac6 = (xm * (durdzp * durdzp));
        } else {
            const double xmm = W.xmu[m - 2], xlm = W.xlam[m - 2];
            const double drho = W.zrho[m - 1] - W.zrho[m - 2];
            const double dmu = xm - xmm;
            const double dlm = xl - xlm;
            const double dl2mu = dlm + dmu + dmu;
            const double xl2mp = xl + xm + xm;
            const double xl2mm = xlm + xmm + xmm;
            const double duzdzp = (ttz + wvno * xl * tur) / xl2mp;
            double durdzp, durdzm;
            if (xm == 0.0) durdzp = wvno * tuz;
            else durdzp = (ttr / xm) - wvno * tuz;
            if (xmm == 0.0) durdzm = wvno * tuz;
            else durdzm = (ttr / xmm) - wvno * tuz;
            double drur2, dlur2, duzdzm;
            if (W.iwat[m - 2] == 1 && W.iwat[m - 1] == 0) {
                const double URB = -(wvno * W.tz[m - 1]) / (W.zrho[m - 2] * om2);
                drur2 = tur * tur * W.zrho[m - 1] - URB * URB * W.zrho[m - 2];
                dlur2 = tur * tur * xl2mp - URB * URB * xl2mm;
                duzdzm = (ttz + wvno * xlm * URB) / xlm;
            } else if (W.iwat[m - 2] == 1 && W.iwat[m - 1] == 1) {
                const double URB = -(wvno * W.tz[m - 1]) / (W.zrho[m - 2] * om2);
                drur2 = tur * tur * W.zrho[m - 1] - URB * URB * W.zrho[m - 2];
                dlur2 = tur * tur * xl2mp - URB * URB * xl2mm;
                duzdzm = (ttz + wvno * xlm * URB) / xl2mm;
            } else {
                drur2 = tur * tur * drho;
                dlur2 = tur * tur * dl2mu;
                duzdzm = (ttz + wvno * xlm * tur) / xl2mm;
            }
            gfac1 = om2 * drho * (tuz * tuz);
            gfac2 = om2 * drur2;
            gfac3 = -(wvno2 * dmu * (tuz * tuz));
            gfac4 = -(wvno2 * dlur2);
            gfac5 = (xl2mp * (duzdzp * duzdzp) - xl2mm * (duzdzm * duzdzm));
            gfac6 = (xm * (durdzp * durdzp) - xmm * (durdzm * durdzm));
        }
        double dfac = fac * (gfac1 + gfac2 + gfac3 + gfac4 + gfac5 + gfac6);
        if (std::abs(dfac) < 1.0e-38) dfac = 0.0;
        W.dcdh[m - 1] = dfac;
    }
}

// sregn96.f90:1061-1203 (with getmat, :1538-1590)
void energy(RW& W, double om, double wvno) {
    W.sumi0 = 0.0;
    W.sumi1 = 0.0;
    W.sumi2 = 0.0;
    W.sumi3 = 0.0;
    const double c = om / wvno;
    const double om2 = om * om;
    const double wvno2 = wvno * wvno;
    for (int m = 1; m <= W.mmax; m++) {
        double a12 = 0, a14 = 0, a21 = 0, a23 = 0, ah, av, bh, bv, eta, rho, TA, TC, TF, TL, TN;
        if (W.iwat[m - 1] == 1) {
            ah = W.za[m - 1];
            av = W.za[m - 1];
            bh = 0.0;
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
            bh = W.zb[m - 1];
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
        (void)bh;
        const int typelyr = (m == W.mmax) ? 1 : 0;
        const double INT11 = intijr(W, 1, 1, m, typelyr, om, om2, wvno, wvno2);
        const double INT13 = intijr(W, 1, 3, m, typelyr, om, om2, wvno, wvno2);
        const double INT22 = intijr(W, 2, 2, m, typelyr, om, om2, wvno, wvno2);
        const double INT24 = intijr(W, 2, 4, m, typelyr, om, om2, wvno, wvno2);
        const double INT33 = intijr(W, 3, 3, m, typelyr, om, om2, wvno, wvno2);
        const double INT44 = intijr(W, 4, 4, m, typelyr, om, om2, wvno, wvno2);
        if (W.iwat[m - 1] == 1) {
            const double wr = wvno / (rho * om2);
            const double URUR = INT22 * (wr * wr);
            const double UZUZ = INT11;
            const double URDUZ = -(wvno / (rho * om2)) * a12 * INT22;
            const double DUZDUZ = a12 * a12 * INT22;
            W.sumi0 = W.sumi0 + rho * (URUR + UZUZ);
            W.sumi1 = W.sumi1 + TA * URUR;
            W.sumi2 = W.sumi2 - TF * URDUZ;
            W.sumi3 = W.sumi3 + TC * DUZDUZ;
            const double facah = rho * ah * ah * (URUR - 2.0 * eta * URDUZ / wvno);
            const double facav = rho * av * av * DUZDUZ / wvno2;
            W.dcda[m - 1] = facah + facav;
            const double facr = -(0.5 * c * c * (URUR + UZUZ));
            W.dcdr[m - 1] = 0.5 * (av * facav + ah * facah) + facr * rho;
            W.dcdgc[m - 1] = 0.0;
            W.dcdgs[m - 1] = 0.0;
            W.ur[m - 1] = -(wvno * W.tz[m - 1]) / (rho * om2);
        } else {
            const double URUR = INT11;
            const double UZUZ = INT22;
            const double DURDUR = a12 * a12 * INT22 + 2.0 * a12 * a14 * INT24 + a14 * a14 * INT44;
            const double DUZDUZ = a21 * a21 * INT11 + 2.0 * a21 * a23 * INT13 + a23 * a23 * INT33;
            const double URDUZ = a21 * INT11 + a23 * INT13;
            const double UZDUR = a12 * INT22 + a14 * INT24;
            W.sumi0 = W.sumi0 + rho * (URUR + UZUZ);
            W.sumi1 = W.sumi1 + TL * UZUZ + TA * URUR;
            W.sumi2 = W.sumi2 + TL * UZDUR - TF * URDUZ;
            W.sumi3 = W.sumi3 + TL * DURDUR + TC * DUZDUZ;
            const double facah = rho * ah * ah * (URUR - 2.0 * eta * URDUZ / wvno);
            const double facav = rho * av * av * DUZDUZ / wvno2;
            const double facbh = 0.0;
            const double facbv = rho * bv * bv *
                (UZUZ + 2.0 * UZDUR / wvno + DURDUR / wvno2 + 4.0 * eta * URDUZ / wvno);
            W.dcda[m - 1] = facah + facav;
            W.dcdb[m - 1] = facbv + facbh;
            const double facr = -(0.5 * c * c * (URUR + UZUZ));
            W.dcdr[m - 1] = 0.5 * (av * facav + ah * facah + bv * facbv) + facr * rho;
            W.dcdgc[m - 1] = rho * bv * bv * (UZUZ + 2.0 * UZDUR / wvno + DURDUR / wvno2)
                           + rho * bv * bv * (URUR);
            W.dcdgs[m - 1] = W.dcdgc[m - 1];
        }
    }
    W.flagr = om2 * W.sumi0 - wvno2 * W.sumi1 - 2.0 * wvno * W.sumi2 - W.sumi3;
    W.ugr = (wvno * W.sumi1 + W.sumi2) / (om * W.sumi0);
    W.are = wvno / (2.0 * om * W.ugr * W.sumi0);
    const double fac = W.are * c / wvno2;
    for (int m = 0; m < W.mmax; m++) {
        W.dcda[m] = W.dcda[m] / (W.ugr * W.sumi0);
        W.dcdb[m] = W.dcdb[m] / (W.ugr * W.sumi0);
        W.dcdr[m] = W.dcdr[m] / (W.ugr * W.sumi0);
        W.dcdgs[m] = W.dcdgs[m] / (W.ugr * W.sumi0);
        W.dcdgc[m] = W.dcdgc[m] / (W.ugr * W.sumi0);
    }
    getdcdh(W, om2, wvno, wvno2, fac);
}

// sregn96.f90:1592-1638
void sprayl(RW& W, double om, double c, double& csph, double& usph) {
    const double ar = 6371.0;
    const double r = c / (2.0 * ar * om);
    const double tm = std::sqrt(1.0 + r * r);
    const double tm3 = (tm * tm) * tm;
    for (int i = 0; i < W.mmax; i++) {
        W.dcda[i] = W.dcda[i] * W.vtp[i] / tm3;
        W.dcdb[i] = W.dcdb[i] * W.vtp[i] / tm3;
        W.dcdh[i] = W.dcdh[i] * W.dtp[i] / tm3;
        W.dcdr[i] = W.dcdr[i] * W.rtp[i] / tm3;
        W.dcdgc[i] = W.dcdgc[i] * W.vtp[i] / tm3;
        W.dcdgs[i] = W.dcdgs[i] * W.vtp[i] / tm3;
    }
    usph = W.ugr * tm;
    csph = c / tm;
}

void run_sregn(const float* thk, const float* vp, const float* vs, const float* rhom,
               int nlayer, double* t, double* cp, double* cg, double* dispu, double* dispw,
               double* stressu, double* stressw, double* dc2da, double* dc2db, double* dc2dh,
               double* dc2dr, double* dc2dgc, double* dc2dgs, int iflsph) {
    RW W;
    const int mmax = nlayer;
    W.mmax = mmax;
    W.zd.resize(mmax);
    W.zrho.resize(mmax);
    W.za.resize(mmax);
    W.zb.resize(mmax);
    W.xmu.resize(mmax);
    W.xlam.resize(mmax);
    for (auto* v : {&W.ur, &W.uz, &W.tz, &W.tr, &W.dcda, &W.dcdb, &W.dcdr, &W.dcdh, &W.dcdgc,
                    &W.dcdgs, &W.exe, &W.exa})
        v->assign(mmax, 0.0);
    W.iwat.assign(mmax, 0);
    W.cd.assign(static_cast<size_t>(mmax) * 5, 0.0);
    W.vv.assign(static_cast<size_t>(mmax) * 4, 0.0);
    for (int i = 0; i < mmax; i++) {
        W.zb[i] = vs[i];
        W.za[i] = vp[i];
        W.zrho[i] = rhom[i];
        W.zd[i] = thk[i];
    }
    W.allfluid = true;
    for (int i = 0; i < mmax; i++) {
        if (W.zb[i] > 0.0) {
            W.allfluid = false;
            W.iwat[i] = 0;
        } else {
            W.iwat[i] = 1;
        }
    }
    const int nsph = iflsph;
    if (nsph > 0) {
        W.vtp.assign(mmax, 0.0);
        W.dtp.assign(mmax, 0.0);
        W.rtp.assign(mmax, 0.0);
        bldsph(W);
    }
    for (int i = 0; i < mmax; i++) {
        W.xmu[i] = W.zrho[i] * (W.zb[i] * W.zb[i]);
        W.xlam[i] = W.zrho[i] * (W.za[i] * W.za[i]) - 2.0 * W.xmu[i];
    }
    const double pi = 3.1415926535897932384626433832795;
    const double twopi = 2.0 * pi;
    const double omega = twopi / *t;
    double c = *cp;
    W.ugr = c;
    double wvno = omega / c;
    svfunc(W, omega, wvno);
    energy(W, omega, wvno);
    if (std::abs(c) < 1.0e-36) c = 0.0;
    if (std::abs(W.ugr) < 1.0e-36) W.ugr = 0.0;
    double csph, usph;
    if (nsph > 0) {
        sprayl(W, omega, c, csph, usph);
        wvno = omega / csph;
    } else {
        csph = c;
        usph = W.ugr;
    }
    for (int i = 0; i < mmax - 1; i++) {
        double sums = 0.0;
        for (int k = i + 1; k < mmax; k++) sums = sums + W.dcdh[k];
        W.dcdh[i] = sums;
    }
    W.dcdh[mmax - 1] = 0.0;
    for (int i = 0; i < mmax; i++) {
        dc2da[i] = W.dcda[i];
        dc2db[i] = W.dcdb[i];
        if (dc2dgc) dc2dgc[i] = W.dcdgc[i];
        if (dc2dgs) dc2dgs[i] = W.dcdgs[i];
        dc2dr[i] = W.dcdr[i];
        dc2dh[i] = W.dcdh[i];
        dispu[i] = W.ur[i];
        dispw[i] = W.uz[i];
        stressu[i] = W.tr[i];
        stressw[i] = W.tz[i];
    }
    *cp = csph;
    *cg = usph;
}


// sregnpu (sregn96.f90:1851-1992): Rayleigh group-velocity kernels from the
// phase kernels at t, t1 and t2 (finite difference in period).
void run_sregnpu(const float* thk, const float* vp, const float* vs, const float* rhom,
                 int nlayer, double t, double cp, double t1, double cp1, double t2, double cp2,
                 double* cg_out, double* du2da, double* du2db, double* du2dh, double* du2dr,
                 double* dc2da, double* dc2db, double* dc2dh, double* dc2dr, int iflsph) {
    RW W;
    const int mmax = nlayer;
    W.mmax = mmax;
    for (auto* v : {&W.zd, &W.zrho, &W.za, &W.zb, &W.xmu, &W.xlam}) v->assign(mmax, 0.0);
    for (auto* v : {&W.ur, &W.uz, &W.tz, &W.tr, &W.dcda, &W.dcdb, &W.dcdr, &W.dcdh, &W.dcdgc,
                    &W.dcdgs, &W.exe, &W.exa})
        v->assign(mmax, 0.0);
    W.iwat.assign(mmax, 0);
    W.cd.assign(static_cast<size_t>(mmax) * 5, 0.0);
    W.vv.assign(static_cast<size_t>(mmax) * 4, 0.0);
    for (int i = 0; i < mmax; i++) {
        W.zb[i] = vs[i];
        W.za[i] = vp[i];
        W.zrho[i] = rhom[i];
        W.zd[i] = thk[i];
    }
    W.allfluid = true;
    for (int i = 0; i < mmax; i++) {
        if (W.zb[i] > 0.0) {
            W.allfluid = false;
            W.iwat[i] = 0;
        } else {
            W.iwat[i] = 1;
        }
    }
    const int nsph = iflsph;
    if (nsph > 0) {
        W.vtp.assign(mmax, 0.0);
        W.dtp.assign(mmax, 0.0);
        W.rtp.assign(mmax, 0.0);
        bldsph(W);
    }
    for (int i = 0; i < mmax; i++) {
        W.xmu[i] = W.zrho[i] * (W.zb[i] * W.zb[i]);
        W.xlam[i] = W.zrho[i] * (W.za[i] * W.za[i]) - 2.0 * W.xmu[i];
    }
    const double pi = 3.1415926535897932384626433832795;
    const double twopi = 2.0 * pi;
    std::vector<double> da1(mmax), db1(mmax), dr1(mmax), dh1(mmax), da2(mmax), db2(mmax),
        dr2(mmax), dh2(mmax);
    // period t (:1908-1918)
    double omega = twopi / t;
    double wvno = omega / cp;
    svfunc(W, omega, wvno);
    energy(W, omega, wvno);
    double cg = W.ugr;
    for (int i = 0; i < mmax; i++) {
        dc2da[i] = W.dcda[i];
        dc2db[i] = W.dcdb[i];
        dc2dr[i] = W.dcdr[i];
        dc2dh[i] = W.dcdh[i];
    }
    // period t1 (:1921-1930)
    omega = twopi / t1;
    wvno = omega / cp1;
    svfunc(W, omega, wvno);
    energy(W, omega, wvno);
    for (int i = 0; i < mmax; i++) {
        da1[i] = W.dcda[i];
        db1[i] = W.dcdb[i];
        dr1[i] = W.dcdr[i];
        dh1[i] = W.dcdh[i];
    }
    // period t2 (:1933-1942)
    omega = twopi / t2;
    wvno = omega / cp2;
    svfunc(W, omega, wvno);
    energy(W, omega, wvno);
    for (int i = 0; i < mmax; i++) {
        da2[i] = W.dcda[i];
        db2[i] = W.dcdb[i];
        dr2[i] = W.dcdr[i];
        dh2[i] = W.dcdh[i];
    }
    // :1945-1949.  The first term reads the module arrays dcda.. , which hold
    // the t2 evaluation at this point.
    const double uc1 = cg / cp;
    for (int i = 0; i < mmax; i++) {
        du2da[i] = uc1 * (2.0 - uc1) * W.dcda[i] - uc1 * uc1 * t * (da2[i] - da1[i]) / (t2 - t1);
        du2db[i] = uc1 * (2.0 - uc1) * W.dcdb[i] - uc1 * uc1 * t * (db2[i] - db1[i]) / (t2 - t1);
        du2dr[i] = uc1 * (2.0 - uc1) * W.dcdr[i] - uc1 * uc1 * t * (dr2[i] - dr1[i]) / (t2 - t1);
        du2dh[i] = uc1 * (2.0 - uc1) * W.dcdh[i] - uc1 * uc1 * t * (dh2[i] - dh1[i]) / (t2 - t1);
    }
    if (nsph > 0) {   // :1952-1971
        const double ar = 6371.0;
        omega = twopi / t;
        const double r = cp / (2.0 * ar * omega);
        const double tm = std::sqrt(1.0 + r * r);
        const double q = 0.5 / (ar * omega);
        const double tm1 = (q * q) / tm;
        const double tm3 = (tm * tm) * tm;
        for (int i = 0; i < mmax; i++) {
            du2da[i] = (tm * du2da[i] + cg * cp * dc2da[i] * tm1) * W.vtp[i];
            du2db[i] = (tm * du2db[i] + cg * cp * dc2db[i] * tm1) * W.vtp[i];
            du2dr[i] = (tm * du2dr[i] + cg * cp * dc2dr[i] * tm1) * W.rtp[i];
            du2dh[i] = (tm * du2dh[i] + cg * cp * dc2dh[i] * tm1) * W.dtp[i];
            dc2da[i] = dc2da[i] / tm3 * W.vtp[i];
            dc2db[i] = dc2db[i] / tm3 * W.vtp[i];
            dc2dr[i] = dc2dr[i] / tm3 * W.rtp[i];
            dc2dh[i] = dc2dh[i] / tm3 * W.dtp[i];
        }
        cg = cg * tm;
    }
    for (int i = 0; i < mmax - 1; i++) {   // :1974-1981
        double sums = 0.0;
        for (int k = i + 1; k < mmax; k++) sums = sums + dc2dh[k];
        dc2dh[i] = sums;
        sums = 0.0;
        for (int k = i + 1; k < mmax; k++) sums = sums + du2dh[k];
        du2dh[i] = sums;
    }
    dc2dh[mmax - 1] = 0.0;
    du2dh[mmax - 1] = 0.0;
    *cg_out = cg;
}
}  // namespace

extern "C" void orc_sregn96_hti(const float* thk, const float* vp, const float* vs,
                                const float* rhom, int nlayer, double* t, double* cp,
                                double* cg, double* dispu, double* dispw, double* stressu,
                                double* stressw, double* dc2da, double* dc2db, double* dc2dh,
                                double* dc2dr, double* dc2dgc, double* dc2dgs, int iflsph) {
    run_sregn(thk, vp, vs, rhom, nlayer, t, cp, cg, dispu, dispw, stressu, stressw, dc2da,
              dc2db, dc2dh, dc2dr, dc2dgc, dc2dgs, iflsph);
}

extern "C" void orc_sregn96(const float* thk, const float* vp, const float* vs,
                            const float* rhom, int nlayer, double* t, double* cp, double* cg,
                            double* dispu, double* dispw, double* stressu, double* stressw,
                            double* dc2da, double* dc2db, double* dc2dh, double* dc2dr,
                            int iflsph) {
    run_sregn(thk, vp, vs, rhom, nlayer, t, cp, cg, dispu, dispw, stressu, stressw, dc2da,
              dc2db, dc2dh, dc2dr, nullptr, nullptr, iflsph);
}

extern "C" void orc_sregnpu(const float* thk, const float* vp, const float* vs, const float* rhom,
                            int nlayer, double t, double cp, double t1, double cp1, double t2,
                            double cp2, double* cg, double* du2da, double* du2db, double* du2dh,
                            double* du2dr, double* dc2da, double* dc2db, double* dc2dh,
                            double* dc2dr, int iflsph) {
    run_sregnpu(thk, vp, vs, rhom, nlayer, t, cp, t1, cp1, t2, cp2, cg, du2da, du2db, du2dh,
                du2dr, dc2da, dc2db, dc2dh, dc2dr, iflsph);
}
