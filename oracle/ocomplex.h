// gfortran's complex(8) arithmetic, as the oracle's sregn96 / slegn96
// restatements need it: complex*complex is the plain (ac-bd, ad+bc) product,
// a real operand scales both parts, complex/complex uses the range-reduced
// (Smith) form gfortran emits by default, and the complex exponential is
// exp(re) * (cos im, sin im).  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cmath>

#include "omath.h"

namespace {

struct cx {
    double re, im;
};
inline cx C(double r, double i = 0.0) { return {r, i}; }
inline cx operator+(cx a, cx b) { return {a.re + b.re, a.im + b.im}; }
inline cx operator-(cx a, cx b) { return {a.re - b.re, a.im - b.im}; }
inline cx operator-(cx a) { return {-a.re, -a.im}; }
inline cx operator*(cx a, cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cx operator*(double s, cx a) { return {s * a.re, s * a.im}; }
inline cx operator*(cx a, double s) { return {a.re * s, a.im * s}; }
inline cx operator+(double s, cx a) { return {s + a.re, a.im}; }
inline cx operator-(double s, cx a) { return {s - a.re, -a.im}; }
inline cx operator/(cx a, double s) { return {a.re / s, a.im / s}; }
inline cx operator/(cx a, cx b) {
    const double ar = a.re, ai = a.im, br = b.re, bi = b.im;
    if (std::abs(br) < std::abs(bi)) {
        const double ratio = br / bi;
        const double div = (br * ratio) + bi;
        return {((ar * ratio) + ai) / div, ((ai * ratio) - ar) / div};
    }
    const double ratio = bi / br;
    const double div = (bi * ratio) + br;
    return {((ai * ratio) + ar) / div, (ai - (ar * ratio)) / div};
}
inline cx operator/(double s, cx b) { return C(s) / b; }
inline double cabs_(cx a) { return std::hypot(a.re, a.im); }
inline cx csqrt_real(double x) {   // cdsqrt(dcmplx(x, 0d0)) for real x
    if (x < 0.0) return {0.0, std::sqrt(-x)};
    return {std::sqrt(x), 0.0};
}
inline cx cexp_(cx a) {
    const double e = om::exp(a.re);
    return {e * om::cos(a.im), e * om::sin(a.im)};
}
inline cx conj_(cx a) { return {a.re, -a.im}; }

}  // namespace
