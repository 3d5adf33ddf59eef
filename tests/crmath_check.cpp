// Host build of the product's correctly rounded exp/log/sin/cos
// (surfattpp_b200/csrc/crmath.cuh) for the tests: cr_eval evaluates them on
// host arrays; cr_check compares them with quad-precision values rounded to
// double (libquadmath, 113-bit) and with the C library on seeded random
// arguments.  Built by tests/test_crmath.py with -ffp-contract=off.
#include <cmath>
#include <cstdint>
#include <random>
#include <quadmath.h>

#include "crmath.cuh"

extern "C" void cr_eval(int f, const double* x, double* y, long n) {
    for (long i = 0; i < n; i++) {
        switch (f) {
            case 0: y[i] = sa::cr::exp(x[i]); break;
            case 1: y[i] = sa::cr::log(x[i]); break;
            case 2: y[i] = sa::cr::sin(x[i]); break;
            case 3: y[i] = sa::cr::cos(x[i]); break;
            case 5: y[i] = sa::cr::pow_m3(x[i]); break;
            default: {
                double s, c;
                sa::cr::sincos(x[i], &s, &c);
                y[2 * i] = s;
                y[2 * i + 1] = c;
            }
        }
    }
}

// Arguments uniform on [lo, hi] (log-uniform if logu); counts of results
// differing from the rounded quad value and from the C library.
extern "C" void cr_check(int f, double lo, double hi, int logu, long n, unsigned long seed,
                         long* n_not_cr, long* n_ne_libc, long* n_libc_not_cr) {
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    long a = 0, b = 0, c = 0;
    for (long i = 0; i < n; i++) {
        const double t = U(g);
        const double x = logu ? std::exp(std::log(lo) + (std::log(hi) - std::log(lo)) * t)
                              : lo + (hi - lo) * t;
        double y, q, l;
        switch (f) {
            case 0: y = sa::cr::exp(x); q = (double)expq((__float128)x); l = std::exp(x); break;
            case 1: y = sa::cr::log(x); q = (double)logq((__float128)x); l = std::log(x); break;
            case 2: y = sa::cr::sin(x); q = (double)sinq((__float128)x); l = std::sin(x); break;
            case 3: y = sa::cr::cos(x); q = (double)cosq((__float128)x); l = std::cos(x); break;
            default:
                y = sa::cr::pow_m3(x);
                q = (double)powq((__float128)x, -3);
                l = std::pow(x, -3.0);
                break;
        }
        if (y != q) a++;
        if (y != l) b++;
        if (l != q) c++;
    }
    *n_not_cr = a;
    *n_ne_libc = b;
    *n_libc_not_cr = c;
}
