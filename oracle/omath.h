// Transcendentals of the oracle's surfdisp96 / sregn96 restatement and of
// the kernel accumulation's svel^-3 (preproc.cpp).
//
// Default build (liboracle.so): the C library's exp, log, sin, cos -- what
// the reference's gfortran-compiled Fortran calls.  With -DORACLE_CR_MATH
// (liboracle_cr.so): the correctly rounded functions of the product's
// crmath.cuh, which the device column kernels use; comparing the device
// against that build checks the transliteration bit for bit, independently
// of the about 0.1 % of arguments where the C library itself misrounds.
// The earth-flattening logarithms (sphere / bldsph) stay the C library's in
// both builds: the device precomputes them on the host.
#pragma once
#include <cmath>

#ifdef ORACLE_CR_MATH
#include "crmath.cuh"
namespace om {
inline double exp(double x) { return sa::cr::exp(x); }
inline double log(double x) { return sa::cr::log(x); }
inline double sin(double x) { return sa::cr::sin(x); }
inline double cos(double x) { return sa::cr::cos(x); }
inline double pow_m3(double x) { return sa::cr::pow_m3(x); }
}  // namespace om
#else
namespace om {
inline double exp(double x) { return std::exp(x); }
inline double log(double x) { return std::log(x); }
inline double sin(double x) { return std::sin(x); }
inline double cos(double x) { return std::cos(x); }
inline double pow_m3(double x) { return std::pow(x, -3.0); }
}  // namespace om
#endif
