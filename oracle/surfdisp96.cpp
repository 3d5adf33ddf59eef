// CPU oracle: surfdisp96 phase/group velocity root search.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Restates src/surfker/surfdisp96.f operation for operation.  Fortran implicit
// typing is kept: names starting i-n are integers, all other undeclared names
// are REAL*4 (float here), unless the routine says `implicit double precision`.
// Default-kind literals such as 0.01 or .95 are REAL*4 constants.
#include "oracle.h"
#include "omath.h"

#include <cmath>
#include <vector>

namespace {

struct Model {           // the REAL*4 layer arrays d, a, b, rho, rtp, dtp, btp
    int mmax, llw;
    std::vector<float> d, a, b, rho, rtp, dtp, btp;
    float dhalf;         // common/sphere_module/ (surfdisp96.f:534-536)
    double del1st;       // common/getsol_module/ (surfdisp96.f:429-430)
};

inline double dsign1(double x) { return std::copysign(1.0, x); }

// surfdisp96.f:502-574
void sphere(Model& M, int ifunc, int iflag) {
    const int mmax = M.mmax;
    const double ar = 6370.0;
    double dr = 0.0;
    double r0 = ar;
    M.d[mmax - 1] = 1.0f;
    if (iflag == 0) {
        for (int i = 0; i < mmax; i++) {
            M.dtp[i] = M.d[i];
            M.rtp[i] = M.rho[i];
        }
        for (int i = 0; i < mmax; i++) {
            dr = dr + static_cast<double>(M.d[i]);
            const double r1 = ar - dr;
            const double z0 = ar * std::log(ar / r0);
            const double z1 = ar * std::log(ar / r1);
            M.d[i] = static_cast<float>(z1 - z0);
            const double tmp = (ar + ar) / (r0 + r1);
            M.a[i] = static_cast<float>(M.a[i] * tmp);
            M.b[i] = static_cast<float>(M.b[i] * tmp);
            M.btp[i] = static_cast<float>(tmp);
            r0 = r1;
        }
        M.dhalf = M.d[mmax - 1];
    } else {
        M.d[mmax - 1] = M.dhalf;
        for (int i = 0; i < mmax; i++) {
            if (ifunc == 1) {
                // btp**(-5): gfortran expands the integer power as
                // x2 = x*x, x3 = x2*x, x5 = x3*x2, then 1/x5.
                const float x = M.btp[i];
                const float x2 = x * x;
                const float x3 = x2 * x;
                const float x5 = x3 * x2;
                M.rho[i] = M.rtp[i] * (1.0f / x5);
            } else if (ifunc == 2) {
                M.rho[i] = M.rtp[i] * std::pow(M.btp[i], -2.275f);
            }
        }
    }
    M.d[mmax - 1] = 0.0f;
}

// surfdisp96.f:380-401 (all REAL*4)
float gtsolh(float a, float b) {
    float c = 0.95f * b;
    for (int i = 0; i < 5; i++) {
        const float gamma = b / a;
        const float kappa = c / b;
        const float k2 = kappa * kappa;
        const float gk2 = (gamma * kappa) * (gamma * kappa);
        const float fac1 = std::sqrt(1.0f - gk2);
        const float fac2 = std::sqrt(1.0f - k2);
        const float t = 2.0f - k2;
        const float fr = t * t - 4.0f * fac1 * fac2;
        float frp = -(4.0f * (2.0f - k2) * kappa)
                  + 4.0f * fac2 * gamma * gamma * kappa / fac1
                  + 4.0f * fac1 * kappa / fac2;
        frp = frp / b;
        c = c - fr / frp;
    }
    return c;
}

// surfdisp96.f:904-1021 (outputs that are used by the callers only)
struct VarOut {
    double w, cosp, exa, a0, cpcq, cpy, cpz, cqw, cqx, xy, xz, wy, wz;
};

VarOut var(double p, double q, double ra, double rb, double wvno, double xka, double xkb,
           double dpth) {
    VarOut o;
    double pex = 0.0, sex = 0.0;
    double sinp = 0.0, w = 0.0, x = 0.0, cosp = 0.0;
    double sinq = 0.0, y = 0.0, z = 0.0, cosq = 0.0;
    if (wvno < xka) {
        sinp = om::sin(p);
        w = sinp / ra;
        x = -(ra * sinp);
        cosp = om::cos(p);
    } else if (wvno == xka) {
        cosp = 1.0;
        w = dpth;
        x = 0.0;
    } else if (wvno > xka) {
        pex = p;
        double fac = 0.0;
        if (p < 16) fac = om::exp(-2.0 * p);
        cosp = (1.0 + fac) * 0.5;
        sinp = (1.0 - fac) * 0.5;
        w = sinp / ra;
        x = ra * sinp;
    }
    if (wvno < xkb) {
        sinq = om::sin(q);
        y = sinq / rb;
        z = -(rb * sinq);
        cosq = om::cos(q);
    } else if (wvno == xkb) {
        cosq = 1.0;
        y = dpth;
        z = 0.0;
    } else if (wvno > xkb) {
        sex = q;
        double fac = 0.0;
        if (q < 16) fac = om::exp(-2.0 * q);
        cosq = (1.0 + fac) * 0.5;
        sinq = (1.0 - fac) * 0.5;
        y = sinq / rb;
        z = rb * sinq;
    }
    o.exa = pex + sex;
    o.a0 = 0.0;
    if (o.exa < 60.0) o.a0 = om::exp(-o.exa);
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
    // The trailing rescaling of cosq, y, z (surfdisp96.f:1014-1019) only
    // touches locals and has no effect on the outputs.
    return o;
}

// surfdisp96.f:1054-1098; ca[j][i] holds Fortran ca(j+1, i+1)
void dnka(double ca[5][5], double wvno2, double gam, double gammk, double rho, const VarOut& v) {
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

// surfdisp96.f:1025-1050
void normc(double* ee, int n, double& ex) {
    double t1 = 0.0;
    for (int i = 0; i < n; i++)
        if (std::abs(ee[i]) > t1) t1 = std::abs(ee[i]);
    if (t1 < 1.e-40) t1 = 1.0;
    for (int i = 0; i < n; i++) {
        double t2 = ee[i];
        t2 = t2 / t1;
        ee[i] = t2;
    }
    ex = om::log(t1);
}

// surfdisp96.f:801-901
double dltar4(const Model& M, double wvno, double omga) {
    const int mmax = M.mmax;
    double omega = omga;
    if (omega < 1.0e-4) omega = 1.0e-4;
    const double wvno2 = wvno * wvno;
    double xka = omega / static_cast<double>(M.a[mmax - 1]);
    double xkb = omega / static_cast<double>(M.b[mmax - 1]);
    double wvnop = wvno + xka;
    double wvnom = std::abs(wvno - xka);
    double ra = std::sqrt(wvnop * wvnom);
    wvnop = wvno + xkb;
    wvnom = std::abs(wvno - xkb);
    double rb = std::sqrt(wvnop * wvnom);
    double t = static_cast<double>(M.b[mmax - 1]) / omega;
    double gammk = 2.0 * t * t;
    double gam = gammk * wvno2;
    const double gamm1 = gam - 1.0;
    double rho1 = static_cast<double>(M.rho[mmax - 1]);
    double e[5], ee[5], ca[5][5];
    e[0] = rho1 * rho1 * (gamm1 * gamm1 - gam * gammk * ra * rb);
    e[1] = -(rho1 * ra);
    e[2] = rho1 * (gamm1 - gammk * ra * rb);
    e[3] = rho1 * rb;
    e[4] = wvno2 - ra * rb;
    for (int m = mmax - 2; m >= M.llw - 1; m--) {
        xka = omega / static_cast<double>(M.a[m]);
        xkb = omega / static_cast<double>(M.b[m]);
        t = static_cast<double>(M.b[m]) / omega;
        gammk = 2.0 * t * t;
        gam = gammk * wvno2;
        wvnop = wvno + xka;
        wvnom = std::abs(wvno - xka);
        ra = std::sqrt(wvnop * wvnom);
        wvnop = wvno + xkb;
        wvnom = std::abs(wvno - xkb);
        rb = std::sqrt(wvnop * wvnom);
        const double dpth = static_cast<double>(M.d[m]);
        rho1 = static_cast<double>(M.rho[m]);
        const double p = ra * dpth;
        const double q = rb * dpth;
        const VarOut v = var(p, q, ra, rb, wvno, xka, xkb, dpth);
        dnka(ca, wvno2, gam, gammk, rho1, v);
        for (int i = 0; i < 5; i++) {
            double cr = 0.0;
            for (int j = 0; j < 5; j++) cr = cr + e[j] * ca[j][i];
            ee[i] = cr;
        }
        double exa;
        normc(ee, 5, exa);
        for (int i = 0; i < 5; i++) e[i] = ee[i];
    }
    if (M.llw != 1) {
        xka = omega / static_cast<double>(M.a[0]);
        wvnop = wvno + xka;
        wvnom = std::abs(wvno - xka);
        ra = std::sqrt(wvnop * wvnom);
        const double dpth = static_cast<double>(M.d[0]);
        rho1 = static_cast<double>(M.rho[0]);
        const double p = ra * dpth;
        const double znul = 1.0e-05;
        const VarOut v = var(p, znul, ra, znul, wvno, xka, znul, dpth);
        const double w0 = -(rho1 * v.w);
        return v.cosp * e[0] + w0 * e[1];
    }
    return e[0];
}

// surfdisp96.f:737-797
double dltar1(const Model& M, double wvno, double omega) {
    const int mmax = M.mmax;
    double beta1 = static_cast<double>(M.b[mmax - 1]);
    double rho1 = static_cast<double>(M.rho[mmax - 1]);
    double xkb = omega / beta1;
    double wvnop = wvno + xkb;
    double wvnom = std::abs(wvno - xkb);
    double rb = std::sqrt(wvnop * wvnom);
    double e1 = rho1 * rb;
    double e2 = 1.0 / (beta1 * beta1);
    for (int m = mmax - 2; m >= M.llw - 1; m--) {
        beta1 = static_cast<double>(M.b[m]);
        rho1 = static_cast<double>(M.rho[m]);
        const double xmu = rho1 * beta1 * beta1;
        xkb = omega / beta1;
        wvnop = wvno + xkb;
        wvnom = std::abs(wvno - xkb);
        rb = std::sqrt(wvnop * wvnom);
        const double q = static_cast<double>(M.d[m]) * rb;
        double sinq, y, z, cosq;
        if (wvno < xkb) {
            sinq = om::sin(q);
            y = sinq / rb;
            z = -(rb * sinq);
            cosq = om::cos(q);
        } else if (wvno == xkb) {
            cosq = 1.0;
            y = static_cast<double>(M.d[m]);
            z = 0.0;
        } else {
            double fac = 0.0;
            if (q < 16) fac = om::exp(-2.0 * q);
            cosq = (1.0 + fac) * 0.5;
            sinq = (1.0 - fac) * 0.5;
            y = sinq / rb;
            z = rb * sinq;
        }
        const double e10 = e1 * cosq + e2 * xmu * z;
        const double e20 = e1 * y / xmu + e2 * cosq;
        double xnor = std::abs(e10);
        const double ynor = std::abs(e20);
        if (ynor > xnor) xnor = ynor;
        if (xnor < 1.e-40) xnor = 1.0;
        e1 = e10 / xnor;
        e2 = e20 / xnor;
    }
    return e1;
}

double dltar(const Model& M, double wvno, double omega, int kk) {
    if (kk == 1) return dltar1(M, wvno, omega);
    return dltar4(M, wvno, omega);
}

// surfdisp96.f:699-711
void half(const Model& M, double c1, double c2, double& c3, double& del3, double omega, int ifunc) {
    c3 = 0.5 * (c1 + c2);
    const double wvno = omega / c3;
    del3 = dltar(M, wvno, omega, ifunc);
}

// surfdisp96.f:578-697
double nevill(const Model& M, double t, double c1, double c2, double del1, double del2,
              int ifunc, double twopi) {
    double x[20], y[20];
    const double omega = twopi / t;
    double c3, del3;
    half(M, c1, c2, c3, del3, omega, ifunc);
    int nev = 1;
    int nctrl = 1;
    int m = 1;
    const double p01 = static_cast<double>(0.01f);   // REAL*4 literal 0.01
    for (;;) {
        nctrl = nctrl + 1;
        if (nctrl >= 100) break;
        if (c3 < std::fmin(c1, c2) || c3 > std::fmax(c1, c2)) {
            nev = 0;
            half(M, c1, c2, c3, del3, omega, ifunc);
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
        if (std::abs(c1 - c2) <= 1.e-6 * c1) break;
        if (dsign1(s13) != dsign1(s32)) nev = 0;
        const double ss1 = std::abs(del1);
        const double s1 = p01 * ss1;
        const double ss2 = std::abs(del2);
        const double s2 = p01 * ss2;
        if (s1 > ss2 || s2 > ss1 || nev == 0) {
            half(M, c1, c2, c3, del3, omega, ifunc);
            nev = 1;
            m = 1;
        } else {
            if (nev == 2) {
                x[m] = c3;        // x(m+1)
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
                const int j = m - kk + 1;                  // Fortran index
                const double denom = y[m] - y[j - 1];      // y(m+1) - y(j)
                if (std::abs(denom) < 1.0e-10 * std::abs(y[m])) {
                    bad = true;
                    break;
                }
                x[j - 1] = (-(y[j - 1] * x[j]) + y[m] * x[j - 1]) / denom;
            }
            if (!bad) {
                c3 = x[0];
                const double wvno = omega / c3;
                del3 = dltar(M, wvno, omega, ifunc);
                nev = 2;
                m = m + 1;
                if (m > 10) m = 10;
            } else {
                half(M, c1, c2, c3, del3, omega, ifunc);
                nev = 1;
                m = 1;
            }
        }
    }
    return c3;
}

// surfdisp96.f:403-498.  Returns iret (1 found, -1 not found); c1 in/out.
int getsol(Model& M, double t1, double& c1, double clow, double dc, double cm, float betmx,
           int ifunc, int ifirst) {
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
    double c2;
    for (;;) {
        if (idir > 0) c2 = c1 + dc;
        else c2 = c1 - dc;
        if (c2 <= clow) {
            idir = +1;
            c1 = clow;
        }
        if (c2 <= clow) continue;
        omega = twopi / t1;
        wvno = omega / c2;
        const double del2 = dltar(M, wvno, omega, ifunc);
        if (dsign1(del1) != dsign1(del2)) {
            const double cn = nevill(M, t1, c1, c2, del1, del2, ifunc, twopi);
            c1 = cn;
            if (c1 > static_cast<double>(betmx)) return -1;
            return 1;
        }
        c1 = c2;
        del1 = del2;
        if (c1 < cm) return -1;
        if (c1 >= (static_cast<double>(betmx) + dc)) return -1;
    }
}

}  // namespace

// surfdisp96.f:57-373
// ---------------------------------------------------------------------------
// Derivatives of the phase-velocity root (no reference counterpart: the
// reference's kernels come from sregn96's energy integrals, which agree
// with differences of surfdisp96's phase velocities only to about 1e-3).
// The Rayleigh secular function of dltar4 is F = e_hs CA_{n} ... CA_0 u / N,
// e_hs the half-space row vector, CA_m the 5x5 compound layer matrix
// (dnka), u the first unit vector, N the product of the normc scalings.  At
// the root F = 0, so with B_m = CA_{m-1} ... CA_0 u and e_{m+1} the
// normalised row vector entering layer m,
//   dF/dp_m = e_{m+1} (dCA_m/dp_m) B_m / (n_m ... n_0),
//   dc/dp = -(dF/dp) / (dF/dc),
// dCA_m/dp_m and de_hs/dp by central differences of the single layer's
// matrix (relative step 1e-6), dF/dc by central differences of dltar4.
// ---------------------------------------------------------------------------
namespace {

// the layer matrix of dltar4's loop (surfdisp96.f:840-889) from double
// parameters
void layer_ca(double a, double b, double rho, double d, double wvno, double omega,
              double ca[5][5]) {
    const double wvno2 = wvno * wvno;
    const double xka = omega / a, xkb = omega / b;
    const double t = b / omega;
    const double gammk = 2.0 * t * t;
    const double gam = gammk * wvno2;
    const double ra = std::sqrt((wvno + xka) * std::abs(wvno - xka));
    const double rb = std::sqrt((wvno + xkb) * std::abs(wvno - xkb));
    const VarOut v = var(ra * d, rb * d, ra, rb, wvno, xka, xkb, d);
    dnka(ca, wvno2, gam, gammk, rho, v);
}

// the half-space vector of dltar4 (surfdisp96.f:811-830)
void halfspace_e(double a, double b, double rho, double wvno, double omega, double e[5]) {
    const double wvno2 = wvno * wvno;
    const double xka = omega / a, xkb = omega / b;
    const double ra = std::sqrt((wvno + xka) * std::abs(wvno - xka));
    const double rb = std::sqrt((wvno + xkb) * std::abs(wvno - xkb));
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

}  // namespace

// Rayleigh phase velocities c[kmax] (surfdisp96's roots for the unflattened
// float layer model, iflsph 1) -> dc/d(vs, vp, rho) of every layer,
// [k * nlayer + layer].  Returns 0, or 1 for a model with a water layer.
extern "C" int orc_dispersion_dcdm(const float* thkm, const float* vpm, const float* vsm,
                                   const float* rhom, int nlayer, int kmax, const double* t,
                                   const double* c, double* dcdb, double* dcda, double* dcdr) {
    Model M;
    const int mmax = nlayer;
    M.mmax = mmax;
    M.d.assign(thkm, thkm + mmax);
    M.a.assign(vpm, vpm + mmax);
    M.b.assign(vsm, vsm + mmax);
    M.rho.assign(rhom, rhom + mmax);
    M.rtp.assign(mmax, 0.0f);
    M.dtp.assign(mmax, 0.0f);
    M.btp.assign(mmax, 0.0f);
    M.dhalf = 0.0f;
    M.llw = (M.b[0] <= 0.0f) ? 2 : 1;
    if (M.llw != 1) return 1;
    sphere(M, 0, 0);
    sphere(M, 2, 1);
    const double twopi = 2.0 * 3.141592653589793;
    std::vector<double> ein(5 * static_cast<size_t>(mmax)), logn(mmax, 0.0);
    for (int k = 0; k < kmax; k++) {
        const double omega = std::max(twopi / t[k], 1.0e-4);
        const double wvno = omega / c[k];
        // forward pass of dltar4 keeping each layer's input vector and scale
        double e[5], ee[5], ca[5][5];
        halfspace_e(M.a[mmax - 1], M.b[mmax - 1], M.rho[mmax - 1], wvno, omega, e);
        for (int m = mmax - 2; m >= 0; m--) {
            for (int i = 0; i < 5; i++) ein[5 * m + i] = e[i];
            layer_ca(M.a[m], M.b[m], M.rho[m], M.d[m], wvno, omega, ca);
            double t1 = 0.0;
            for (int i = 0; i < 5; i++) {
                double cr = 0.0;
                for (int j = 0; j < 5; j++) cr += e[j] * ca[j][i];
                ee[i] = cr;
                t1 = std::max(t1, std::abs(cr));
            }
            if (t1 < 1.e-40) t1 = 1.0;
            for (int i = 0; i < 5; i++) e[i] = ee[i] / t1;
            logn[m] = std::log(t1);
        }
        // dF/dc by central differences of the secular function
        const double hc = 1e-7 * c[k];
        const double Fc = (dltar4(M, omega / (c[k] + hc), omega)
                           - dltar4(M, omega / (c[k] - hc), omega)) / (2.0 * hc);
        // top-down vectors B_m (normalised, log scale LB) and the layer terms
        double B[5] = {1.0, 0.0, 0.0, 0.0, 0.0};
        double LB = 0.0, LN = 0.0;   // log |B| scale, log (n_m ... n_0)
        auto dF = [&](const double* row, const double dca[5][5]) {
            double s = 0.0;
            for (int i = 0; i < 5; i++) {
                double r = 0.0;
                for (int j = 0; j < 5; j++) r += dca[i][j] * B[j];
                s += row[i] * r;
            }
            return s;
        };
        for (int m = 0; m <= mmax - 2; m++) {
            LN += logn[m];
            const double scale = std::exp(LB - LN);
            const double p0[3] = {M.b[m], M.a[m], M.rho[m]};
            double out[3];
            for (int q = 0; q < 3; q++) {
                double pp[3] = {p0[0], p0[1], p0[2]}, pm[3] = {p0[0], p0[1], p0[2]};
                const double h = 1e-6 * p0[q];
                pp[q] += h;
                pm[q] -= h;
                double cp[5][5], cm[5][5], dca[5][5];
                layer_ca(pp[1], pp[0], pp[2], M.d[m], wvno, omega, cp);
                layer_ca(pm[1], pm[0], pm[2], M.d[m], wvno, omega, cm);
                for (int i = 0; i < 5; i++)
                    for (int j = 0; j < 5; j++) dca[i][j] = (cp[i][j] - cm[i][j]) / (2.0 * h);
                out[q] = -(dF(&ein[5 * m], dca) * scale) / Fc;
            }
            // unflattened parameters: b_f = b tmp, a_f = a tmp, rho_f = rho btp^-2.275
            const double tmp = M.btp[m];
            const size_t o = static_cast<size_t>(k) * mmax + m;
            dcdb[o] = out[0] * tmp;
            dcda[o] = out[1] * tmp;
            dcdr[o] = out[2] * std::pow(M.btp[m], -2.275f);
            // B_{m+1} = CA_m B_m
            layer_ca(M.a[m], M.b[m], M.rho[m], M.d[m], wvno, omega, ca);
            double nb[5], bm = 0.0;
            for (int i = 0; i < 5; i++) {
                double r = 0.0;
                for (int j = 0; j < 5; j++) r += ca[i][j] * B[j];
                nb[i] = r;
                bm = std::max(bm, std::abs(r));
            }
            if (bm < 1e-300) bm = 1.0;
            for (int i = 0; i < 5; i++) B[i] = nb[i] / bm;
            LB += std::log(bm);
        }
        // the half-space layer
        {
            const int m = mmax - 1;
            const double scale = std::exp(LB - LN);
            const double p0[3] = {M.b[m], M.a[m], M.rho[m]};
            double out[3];
            for (int q = 0; q < 3; q++) {
                double pp[3] = {p0[0], p0[1], p0[2]}, pm[3] = {p0[0], p0[1], p0[2]};
                const double h = 1e-6 * p0[q];
                pp[q] += h;
                pm[q] -= h;
                double ep[5], em[5];
                halfspace_e(pp[1], pp[0], pp[2], wvno, omega, ep);
                halfspace_e(pm[1], pm[0], pm[2], wvno, omega, em);
                double s = 0.0;
                for (int i = 0; i < 5; i++) s += (ep[i] - em[i]) / (2.0 * h) * B[i];
                out[q] = -(s * scale) / Fc;
            }
            const double tmp = M.btp[m];
            const size_t o = static_cast<size_t>(k) * mmax + m;
            dcdb[o] = out[0] * tmp;
            dcda[o] = out[1] * tmp;
            dcdr[o] = out[2] * std::pow(M.btp[m], -2.275f);
        }
    }
    return 0;
}

extern "C" int orc_surfdisp96(const float* thkm, const float* vpm, const float* vsm,
                              const float* rhom, int nlayer, int iflsph, int iwave, int mode,
                              int igr, int kmax, const double* t, double* cg) {
    Model M;
    const int mmax = nlayer;
    M.mmax = mmax;
    M.d.assign(thkm, thkm + mmax);
    M.a.assign(vpm, vpm + mmax);
    M.b.assign(vsm, vsm + mmax);
    M.rho.assign(rhom, rhom + mmax);
    M.rtp.assign(mmax, 0.0f);
    M.dtp.assign(mmax, 0.0f);
    M.btp.assign(mmax, 0.0f);
    M.dhalf = 0.0f;
    M.del1st = 0.0;
    const int nsph = iflsph;
    int idispl = 0, idispr = 0;
    if (iwave == 1) {
        idispl = kmax;
        idispr = 0;
    } else if (iwave == 2) {
        idispl = 0;
        idispr = kmax;
    }
    const float sone0 = 1.500f;
    float vmin = vsm[0];
    for (int i = 1; i < mmax; i++) vmin = std::fmin(vmin, vsm[i]);
    float ddc0;
    if (vmin < 1.0f) ddc0 = 0.001f;
    else if (vmin < 2.0f) ddc0 = 0.002f;
    else ddc0 = 0.005f;
    const float h0 = 0.005f;
    M.llw = 1;
    if (M.b[0] <= 0.0f) M.llw = 2;
    const double twopi = 2.0 * 3.141592653589793;
    (void)twopi;
    const double one = 1.0e-2;
    if (nsph == 1) sphere(M, 0, 0);
    int jmn = 1;
    int jsol = 1;
    float betmx = -1.e20f;
    float betmn = 1.e20f;
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
    std::vector<double> c(kmax, 0.0), cb(kmax, 0.0);
    int status = 0;
    for (int ifunc = 1; ifunc <= 2; ifunc++) {
        if (ifunc == 1 && idispl <= 0) continue;
        if (ifunc == 2 && idispr <= 0) continue;
        if (nsph == 1) sphere(M, ifunc, 1);
        const float ddc = ddc0;
        float sone = sone0;
        const float h = h0;
        if (sone < 0.01f) sone = 2.0f;
        const double onea = static_cast<double>(sone);
        float cc1;
        if (jsol == 0) cc1 = betmn;
        else cc1 = gtsolh(M.a[jmn - 1], M.b[jmn - 1]);
        cc1 = 0.95f * cc1;
        cc1 = 0.90f * cc1;
        const double cc = static_cast<double>(cc1);
        double dc = static_cast<double>(ddc);
        dc = std::abs(dc);
        double c1 = cc;
        const double cm = cc;
        double clow = cc;
        for (int i = 0; i < kmax; i++) {
            cb[i] = 0.0;
            c[i] = 0.0;
        }
        int ift = 999;
        for (int iq = 1; iq <= mode; iq++) {
            const int is = 1;
            const int ie = kmax;
            int kfail = -1;
            for (int k = is; k <= ie; k++) {
                if (k >= ift) {
                    kfail = k;
                    break;
                }
                double t1 = t[k - 1];
                float t1a = 0.0f, t1b = 0.0f;
                if (igr > 0) {
                    t1a = static_cast<float>(t1 / static_cast<double>(1.0f + h));
                    t1b = static_cast<float>(t1 / static_cast<double>(1.0f - h));
                    t1 = static_cast<double>(t1a);
                } else {
                    t1a = static_cast<float>(t1);
                }
                int ifirst;
                if (k == is && iq == 1) {
                    c1 = cc;
                    clow = cc;
                    ifirst = 1;
                } else if (k == is && iq > 1) {
                    c1 = c[is - 1] + one * dc;
                    clow = c1;
                    ifirst = 1;
                } else if (k > is && iq > 1) {
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
                    t1 = static_cast<double>(t1b);
                    ifirst = 0;
                    clow = cb[k - 1] + one * dc;
                    c1 = c1 - onea * dc;
                    iret = getsol(M, t1, c1, clow, dc, cm, betmx, ifunc, ifirst);
                    if (iret == -1) c1 = c[k - 1];
                    cb[k - 1] = c1;
                } else {
                    c1 = 0.0;
                }
                const float cc0 = static_cast<float>(c[k - 1]);
                const float ccg = static_cast<float>(c1);
                if (igr == 0) {
                    cg[k - 1] = cc0;
                } else {
                    const float gvel = (1.0f / t1a - 1.0f / t1b) / (1.0f / (t1a * cc0) - 1.0f / (t1b * ccg));
                    cg[k - 1] = gvel;
                }
            }
            if (kfail < 0) continue;
            if (iq <= 1) {
                // surfdisp96.f:325-357: the Fortran prints diagnostics and stops.
                status = 1;
                for (int i = kfail; i <= ie; i++) cg[i - 1] = 0.0;
                return status;
            }
            ift = kfail;
            for (int i = kfail; i <= ie; i++) cg[i - 1] = 0.0;
        }
    }
    return status;
}
