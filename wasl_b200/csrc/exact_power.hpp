// Integer powers x^2 and x^3 rounded to the nearest double, with a flag for
// the values whose rounding is not settled by the C library's pow.
//
// The Dubiner basis takes ((1 - eta) / 2)^i with the C library's pow
// (cpp/include/wasl/basis/dubiner_triangle.hpp:59).  That pow is accurate to
// about half an ulp but not correctly rounded: where the exact power lies
// very close to the midpoint between two doubles it may return either one.
// Here the exact power is carried as an unevaluated sum of doubles (products
// split with fma, which is exact), rounded once, and its distance from the
// nearest midpoint measured in ulps.  For a value further than kPowerMargin
// ulp from every midpoint only one double, the correctly rounded one, lies
// within the library's error bound (0.52 ulp < 1/2 + kPowerMargin), so pow
// returns exactly it; values nearer a midpoint, at a power of two (where the
// ulp changes), or outside the normal range are flagged, and their powers are
// taken from the host's pow instead.
//
// The same code compiles for the host (tests check it against the library's
// pow) and the device.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define WASL_HD __host__ __device__ __forceinline__
#else
#define WASL_HD inline
#endif

namespace wasl_b200 {

// Ulps from the midpoint below which a power is left to the library's pow:
// its documented error bound is 0.52 ulp (0.02 beyond the rounding), and the
// largest error measured over 10^8 random cubes is 0.5076 ulp.
constexpr double kPowerMargin = 1.0 / 32.0;

WASL_HD std::uint64_t power_bits(double x) {
#if defined(__CUDA_ARCH__)
  return static_cast<std::uint64_t>(__double_as_longlong(x));
#else
  std::uint64_t b;
  std::memcpy(&b, &x, sizeof b);
  return b;
#endif
}

WASL_HD double power_from_bits(std::uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(static_cast<long long>(b));
#else
  double x;
  std::memcpy(&x, &b, sizeof x);
  return x;
#endif
}

WASL_HD double power_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

// The rounded value r of an exact sum r + tail (|tail| <= ulp(r) / 2 + tiny),
// flagged when r is not safely the correctly rounded result.
WASL_HD bool power_unsettled(double r, double tail) {
  const std::uint64_t b = power_bits(r) & 0x7fffffffffffffffULL;
  const int biased = static_cast<int>(b >> 52);
  if (biased < 64 || biased > 2000) // zero, subnormal or near the range ends
    return true;
  if ((b & 0x000fffffffffffffULL) == 0) // a power of two: the ulp changes here
    return true;
  const double ulp = power_from_bits(static_cast<std::uint64_t>(biased - 52) << 52);
  const double t = tail / ulp; // exact: ulp is a power of two
  return std::fabs(t) > 0.5 - kPowerMargin;
}

// x^2 rounded to nearest; *unsettled when the library's pow may differ.
WASL_HD double power2(double x, bool *unsettled) {
  if (x == 0.0) {
    *unsettled = false;
    return 0.0;
  }
  const double s = x * x;
  const double e = power_fma(x, x, -s);
  *unsettled = power_unsettled(s, e);
  return s;
}

// x^3 rounded to nearest; *unsettled when the library's pow may differ.
WASL_HD double power3(double x, bool *unsettled) {
  if (x == 0.0) {
    *unsettled = false;
    return x;
  }
  const double a = std::fabs(x);
  const double s = a * a, e1 = power_fma(a, a, -s);  // a^2 = s + e1
  const double p = s * a, e2 = power_fma(s, a, -p);  // s a = p + e2
  const double q = e1 * a, e3 = power_fma(e1, a, -q); // e1 a = q + e3
  const double c = e2 + q + e3;                       // a^3 = p + c, |c| ~ ulp(p) / 2
  const double r = p + c;
  const double tail = (p - r) + c; // p - r is exact: they are within an ulp
  *unsettled = power_unsettled(r, tail);
  return x < 0.0 ? -r : r;
}

} // namespace wasl_b200
