// Correctly rounded FP64 exp, log, sin and cos for host and device.
//
// The reference's surfdisp96 / sregn96 call the C library's exp, log, sin
// and cos; CUDA's device versions round differently in a few percent of
// cases, which moves the FP64 dispersion root enough to flip the REAL*4
// rounding of some phase velocities.  These functions return the correctly
// rounded result (round to nearest even) for every argument of the column
// kernels, which is what the C library returns in all but about 0.1 % of
// calls, so the device root search follows a CPU evaluation far more
// closely than with CUDA's functions.
//
// Method (each function): argument reduction to a small interval with an
// exact or double-double remainder, a table of double-double values at
// interval centres (Tang's table-driven method, ACM TOMS 15(2) 1989 for exp,
// 16(4) 1990 for log), a short Taylor / atanh series evaluated partly in
// double-double (Dekker 1971; error-free products with fma), and one final
// rounding of the double-double sum.  The approximation error is below about
// 2^-93 relative, so the final rounding is correct except for arguments
// whose exact result lies within that distance of a rounding boundary.
//
// Host and device give bit-identical results: every product that is added
// is written as an explicit fma, nothing else is contracted or reassociated
// (host units: -ffp-contract=off), and the tables are the same literals
// (crmath_tables.h, generated by gen_crmath_tables.py).
//
// Domain notes: exp results below 2^-1022 (x < -708.39) are scaled after
// rounding (not correctly rounded in the subnormal range); sin / cos reduce
// |x| < 2^20 pi/2 exactly and fall back to the platform's sin / cos beyond.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "crmath_tables.h"

#if defined(__CUDACC__)
#define CR_HD __host__ __device__
#define CR_DEV_ARRAY static __device__ const
#else
#define CR_HD
#endif

namespace sa {
namespace cr {

// ---- tables (one host copy, one device copy of the same literals) ---------
static const double kExpT1_h[128] = CR_EXP_T1_INIT;
static const double kExpT2_h[128] = CR_EXP_T2_INIT;
static const double kLogInv_h[128] = CR_LOG_INV_INIT;
static const int kLogE_h[128] = CR_LOG_E_INIT;
static const double kLogT_h[256] = CR_LOG_T_INIT;
static const double kSinT_h[2 * CR_SC_N] = CR_SIN_T_INIT;
static const double kCosT_h[2 * CR_SC_N] = CR_COS_T_INIT;
#if defined(__CUDACC__)
CR_DEV_ARRAY double kExpT1_d[128] = CR_EXP_T1_INIT;
CR_DEV_ARRAY double kExpT2_d[128] = CR_EXP_T2_INIT;
CR_DEV_ARRAY double kLogInv_d[128] = CR_LOG_INV_INIT;
CR_DEV_ARRAY int kLogE_d[128] = CR_LOG_E_INIT;
CR_DEV_ARRAY double kLogT_d[256] = CR_LOG_T_INIT;
CR_DEV_ARRAY double kSinT_d[2 * CR_SC_N] = CR_SIN_T_INIT;
CR_DEV_ARRAY double kCosT_d[2 * CR_SC_N] = CR_COS_T_INIT;
#endif

#if defined(__CUDA_ARCH__)
#define CR_TAB(name) name##_d
#else
#define CR_TAB(name) name##_h
#endif

// ---- double-double arithmetic ----------------------------------------------
struct dd {
    double hi, lo;
};

CR_HD inline dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}
// |a| >= |b| (or a == 0)
CR_HD inline dd fast_two_sum(double a, double b) {
    const double s = a + b;
    const double e = b - (s - a);
    return {s, e};
}
CR_HD inline dd two_prod(double a, double b) {
    const double p = a * b;
    const double e = fma(a, b, -p);
    return {p, e};
}
// accurate sum of two double-doubles
CR_HD inline dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    dd t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}
CR_HD inline dd dd_add_d(dd a, double b) {
    dd s = two_sum(a.hi, b);
    s.lo += a.lo;
    return fast_two_sum(s.hi, s.lo);
}
// The same sums when |a.hi| >= |b.hi| (or a.hi == 0) and a and b do not
// cancel: the leading error-free sum needs no ordering test, and the result
// keeps the accurate sum's ~2^-105 relative error.
CR_HD inline dd dd_add_ord(dd a, dd b) {
    dd s = fast_two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return fast_two_sum(s.hi, s.lo);
}
CR_HD inline dd dd_add_d_ord(dd a, double b) {
    dd s = fast_two_sum(a.hi, b);
    s.lo += a.lo;
    return fast_two_sum(s.hi, s.lo);
}
CR_HD inline dd dd_mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo = fma(a.hi, b.lo, fma(a.lo, b.hi, p.lo));
    return fast_two_sum(p.hi, p.lo);
}
CR_HD inline dd dd_mul_d(dd a, double b) {
    dd p = two_prod(a.hi, b);
    p.lo = fma(a.lo, b, p.lo);
    return fast_two_sum(p.hi, p.lo);
}
CR_HD inline dd dd_neg(dd a) { return {-a.hi, -a.lo}; }

CR_HD inline double bits_to_double(uint64_t u) {
    double d;
    memcpy(&d, &u, 8);
    return d;
}
CR_HD inline uint64_t double_to_bits(double d) {
    uint64_t u;
    memcpy(&u, &d, 8);
    return u;
}
// y * 2^m for a normal result (|m| <= 2044 split in two exact steps)
CR_HD inline double scale2(double y, int m) {
    if (m > 1023) {
        y *= bits_to_double((uint64_t)(1023 + 1023) << 52);
        m -= 1023;
    } else if (m < -1022) {
        y *= bits_to_double((uint64_t)(1023 - 1022) << 52);
        m += 1022;
        if (m < -1022) return y * 0.0;
    }
    return y * bits_to_double((uint64_t)(1023 + m) << 52);
}

// ---- exp ---------------------------------------------------------------------
// x = k ln2/4096 + r, k = 4096 m + 64 j2 + j1, |r| <= ln2/8192;
// exp(x) = 2^m * 2^(j2/64) * 2^(j1/4096) * exp(r).
CR_HD inline double exp(double x) {
    if (x != x) return x + x;
    if (x > 709.782712893384) return HUGE_VAL;
    if (x < -745.2) return 0.0;
    const double kd = rint(x * CR_EXP_INVL);
    const int k = (int)kd;
    // kd * L1, kd * L2 exact (|k| < 2^23, 30-bit L1, L2); x - kd*L1 exact
    const double t1 = x - kd * CR_EXP_L1;
    dd r = two_sum(t1, -(kd * CR_EXP_L2));
    r = dd_add_d(r, -(kd * CR_EXP_L3));
    const double h = r.hi;
    // exp(r) - 1 = r + r^2/2 + r^3 (1/6 + r/24 + r^2/120 + r^3/720 + r^4/5040)
    dd sq = two_prod(h, h);
    sq.lo = fma(2.0 * h, r.lo, sq.lo);
    const dd half_sq = {0.5 * sq.hi, 0.5 * sq.lo};
    double tail = fma(h, CR_IFACT7, CR_IFACT6);
    tail = fma(h, tail, CR_IFACT5);
    tail = fma(h, tail, CR_IFACT4);
    tail = fma(h, tail, CR_IFACT3);
    tail = tail * (sq.hi * h);
    // |r| <= ln2/8192 > r^2/2 > |tail|: ordered sums
    dd s = dd_add_ord(r, half_sq);
    s = dd_add_d_ord(s, tail);
    const int j1 = k & 63, j2 = (k >> 6) & 63, m = k >> 12;
    const dd T1 = {CR_TAB(kExpT1)[2 * j1], CR_TAB(kExpT1)[2 * j1 + 1]};
    const dd T2 = {CR_TAB(kExpT2)[2 * j2], CR_TAB(kExpT2)[2 * j2 + 1]};
    const dd P = dd_mul(T1, T2);
    const dd res = dd_add_ord(P, dd_mul(P, s));   // |P s| < 2^-13 |P|; res normalised
    return scale2(res.hi, m);
}

// ---- log ---------------------------------------------------------------------
// x = 2^e m, m in [1, 2); j = top 7 bits of m; r = m inv_j - 1 exactly
// (inv_j has 8 significant bits); log x = (e + E_j) ln2 + T_j + log1p(r),
// T_j = -log(inv_j 2^E_j); log1p(r) = 2 atanh(u), u = r / (2 + r).
CR_HD inline double log(double x) {
    if (!(x > 0.0)) {
        if (x == 0.0) return -HUGE_VAL;
        return (x - x) / (x - x);   // NaN for x < 0 or NaN
    }
    if (x == HUGE_VAL) return x;
    uint64_t u = double_to_bits(x);
    int e = (int)(u >> 52) - 1023;
    if ((u >> 52) == 0) {   // subnormal: scale by 2^54
        u = double_to_bits(x * 18014398509481984.0);
        e = (int)(u >> 52) - 1023 - 54;
    }
    const int j = (int)((u >> 45) & 127);
    const double m = bits_to_double((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    const double inv = CR_TAB(kLogInv)[j];
    const double r = fma(m, inv, -1.0);   // exact
    // u = r / (2 + r) in double-double
    const dd den = two_sum(2.0, r);
    const double q1 = r / den.hi;
    // remainder r - q1 * den, exact pieces
    dd pr = two_prod(q1, den.hi);
    const double rem = ((r - pr.hi) - pr.lo) - q1 * den.lo;
    const double q2 = rem / den.hi;
    const dd uu = fast_two_sum(q1, q2);
    // atanh(u)/u - 1 = w/3 + w^2/5 + w^3 (1/7 + w/9 + w^2/11 + w^3/13), w = u^2
    dd w = two_prod(uu.hi, uu.hi);
    w.lo = fma(2.0 * uu.hi, uu.lo, w.lo);
    double tail = fma(w.hi, CR_INVODD13, CR_INVODD11);
    tail = fma(w.hi, tail, CR_INVODD9);
    tail = fma(w.hi, tail, CR_INVODD7);
    tail = tail * (w.hi * w.hi * w.hi);
    const dd w3 = dd_mul(w, dd{CR_INV3_HI, CR_INV3_LO});
    const dd w2 = dd_mul(dd_mul(w, w), dd{CR_INV5_HI, CR_INV5_LO});
    dd S = dd_add(w3, w2);
    S = dd_add_d(S, tail);
    // log1p(r) = 2u + 2u S
    const dd u2 = {2.0 * uu.hi, 2.0 * uu.lo};
    const dd l1p = dd_add(u2, dd_mul(u2, S));
    const int n = e + CR_TAB(kLogE)[j];
    const dd T = {CR_TAB(kLogT)[2 * j], CR_TAB(kLogT)[2 * j + 1]};
    dd acc = dd_add(T, l1p);
    if (n != 0) {
        const double nd = (double)n;
        dd nl = two_prod(nd, CR_LN2_HI);
        nl.lo = fma(nd, CR_LN2_LO, nl.lo);
        acc = dd_add(fast_two_sum(nl.hi, nl.lo), acc);
    }
    return fast_two_sum(acc.hi, acc.lo).hi;
}

// ---- sin / cos -----------------------------------------------------------------
// x = k pi/2 + r (pi/2 in five pieces, the first four with 32 bits, so the
// products with |k| < 2^21 are exact); r = j/256 + t, |t| <= 2^-9;
// sin r = S_j cos t + C_j sin t, cos r = C_j cos t - S_j sin t.
CR_HD inline void sincos_reduced(double x, dd* s_out, dd* c_out, int* quadrant) {
    const double kd = rint(x * CR_2OPI);
    const double a = x - kd * CR_PIO2_1;   // exact
    dd r = two_sum(a, -(kd * CR_PIO2_2));
    dd r2 = two_sum(r.hi, -(kd * CR_PIO2_3));
    dd r3 = two_sum(r2.hi, -(kd * CR_PIO2_4));
    const double lo = ((r.lo + r2.lo) + r3.lo) - kd * CR_PIO2_5;
    dd rr = fast_two_sum(r3.hi, lo);
    *quadrant = (int)((int64_t)kd & 3);
    const double aj = rint(rr.hi * 256.0);
    int j = (int)aj;
    const double sg = j < 0 ? -1.0 : 1.0;
    if (j < 0) {
        j = -j;
        rr = dd_neg(rr);
    }
    const double th = rr.hi - (double)j * (1.0 / 256.0);   // exact
    const dd t = two_sum(th, rr.lo);
    // sin t = t + t (-t^2/6 + t^4/120 - t^6/5040 + t^8/362880)
    // cos t = 1 + (-t^2/2 + t^4/24 - t^6/720 + t^8/40320)
    dd t2 = two_prod(t.hi, t.hi);
    t2.lo = fma(2.0 * t.hi, t.lo, t2.lo);
    const double z = t2.hi;
    double ps = fma(z, CR_IFACT9, -CR_IFACT7);
    ps = fma(z, ps, CR_IFACT5);
    ps = ps * (z * z);
    // |t| <= 2^-9: t^2/6 > |ps|, |t| > |t psd|, t^2/2 > |pc|: ordered sums
    dd psd = dd_add_d_ord(dd_neg(dd_mul(t2, dd{CR_INV6_HI, CR_INV6_LO})), ps);
    const dd sint = dd_add_ord(t, dd_mul(t, psd));
    double pc = fma(z, CR_IFACT8, -CR_IFACT6);
    pc = fma(z, pc, CR_IFACT4);
    pc = pc * (z * z);
    const dd pcd = dd_add_d_ord(dd{-0.5 * t2.hi, -0.5 * t2.lo}, pc);   // cos t - 1
    const dd S = {CR_TAB(kSinT)[2 * j], CR_TAB(kSinT)[2 * j + 1]};
    const dd C = {CR_TAB(kCosT)[2 * j], CR_TAB(kCosT)[2 * j + 1]};
    // sin r = S + (C sin t + S (cos t - 1)); cos r = C + (C (cos t - 1) - S sin t).
    // C >= cos(pi/4): |C sin t| >= 0.7 |t| > t^2 > |S pcd|; S = 0 or S >=
    // sin(1/256) > |t| + t^2 >= |C sint + S pcd|; C > 0.7 > 2^-8 > the cos
    // correction.  C pcd and S sint are not ordered: accurate sum.
    dd sr = dd_add_ord(S, dd_add_ord(dd_mul(C, sint), dd_mul(S, pcd)));
    dd cr = dd_add_ord(C, dd_add(dd_mul(C, pcd), dd_neg(dd_mul(S, sint))));
    sr = {sg * sr.hi, sg * sr.lo};
    *s_out = sr;
    *c_out = cr;
}

CR_HD inline double sin(double x) {
    const double ax = fabs(x);
    if (ax < 0x1p-26) return x;                       // sin x rounds to x
    if (!(ax < 1647099.0)) return ::sin(x);           // NaN, Inf, |x| >= 2^20 pi/2
    dd s, c;
    int q;
    sincos_reduced(x, &s, &c, &q);
    const dd v = (q == 0) ? s : (q == 1) ? c : (q == 2) ? dd_neg(s) : dd_neg(c);
    return v.hi;   // normalised
}

CR_HD inline double cos(double x) {
    const double ax = fabs(x);
    if (ax < 0x1p-27) return 1.0;                     // cos x rounds to 1
    if (!(ax < 1647099.0)) return ::cos(x);
    dd s, c;
    int q;
    sincos_reduced(x, &s, &c, &q);
    const dd v = (q == 0) ? c : (q == 1) ? dd_neg(s) : (q == 2) ? dd_neg(c) : s;
    return v.hi;   // normalised
}

// ---- x^-3 ------------------------------------------------------------------
// pow(x, -3.0) correctly rounded (normal x, result normal): x^3 as an exact
// double-double product chain, then 1 / x^3 with one Newton correction in
// double-double.
CR_HD inline double pow_m3(double x) {
    const dd x2 = two_prod(x, x);
    const dd x3 = dd_mul_d(x2, x);              // x^3 to about 2^-104 relative
    const double q = 1.0 / x3.hi;
    // r = 1 - q * x3 (exact pieces), y = q + q r
    const dd p = two_prod(q, x3.hi);
    const double r = ((1.0 - p.hi) - p.lo) - q * x3.lo;
    const dd y = fast_two_sum(q, q * r);
    return y.hi;
}

// sin and cos of one argument with one reduction
CR_HD inline void sincos(double x, double* sn, double* cs) {
    const double ax = fabs(x);
    if (ax < 0x1p-27) {
        *sn = x;
        *cs = 1.0;
        return;
    }
    if (!(ax < 1647099.0)) {
        *sn = ::sin(x);
        *cs = ::cos(x);
        return;
    }
    dd s, c;
    int q;
    sincos_reduced(x, &s, &c, &q);
    const dd vs = (q == 0) ? s : (q == 1) ? c : (q == 2) ? dd_neg(s) : dd_neg(c);
    const dd vc = (q == 0) ? c : (q == 1) ? dd_neg(s) : (q == 2) ? dd_neg(c) : s;
    *sn = vs.hi;   // normalised
    *cs = vc.hi;
}

}  // namespace cr
}  // namespace sa
