// Pointwise ideal-gas Euler physics for the kernels, templated on the real type.
//
// Operation order follows the reference expressions so that, compiled without
// FMA contraction (--fmad=false), the FP64 instantiation rounds exactly as the
// reference CPU code:
//   primitive        cpp/include/wasl/equations/euler/primitive.hpp:19-31
//   physical fluxes  cpp/include/wasl/equations/euler/flux.hpp:11-33
//   HLLC             cpp/include/wasl/flux/hllc.hpp:12-74
// Conserved variables are (density, x-momentum, y-momentum, total energy).
#pragma once

#include <cstdint>

namespace wasl_b200 {

// std::min / std::max semantics (the second argument wins only if strictly less / greater).
template <typename T> __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }

template <typename T> struct Prim {
  T rho, vx, vy, p;
};

template <typename T> __device__ __forceinline__ Prim<T> primitive(T gamma, const T *s) {
  const T inv = T(1) / s[0];
  const T vx = s[1] * inv;
  const T vy = s[2] * inv;
  const T ke = T(0.5) * (s[1] * vx + s[2] * vy);
  return {s[0], vx, vy, (gamma - T(1)) * (s[3] - ke)};
}

template <typename T> __device__ __forceinline__ T sound_speed(T gamma, const Prim<T> &v) {
  return sqrt(gamma * v.p / v.rho);
}

// The CFL wave speed |u| + c (hypot(u, v) + c in 2D) of a cell average s
// (cpp/src/time/cfl_timestep.cpp:33-47), with the operations of primitive()
// and sound_speed() written as explicitly rounded steps, so kernels compiled
// with and without multiply-add contraction compute the same bits.  physical
// is false for a non-positive density or pressure.
__device__ __forceinline__ double cfl_speed(double gamma, const double *s, int dimensions,
                                            bool &physical) {
  const double inv = 1.0 / s[0];
  const double vx = __dmul_rn(s[1], inv);
  const double vy = __dmul_rn(s[2], inv);
  const double ke = __dmul_rn(0.5, __dadd_rn(__dmul_rn(s[1], vx), __dmul_rn(s[2], vy)));
  const double p = __dmul_rn(gamma - 1.0, __dsub_rn(s[3], ke));
  physical = s[0] > 0.0 && p > 0.0;
  const double velocity = dimensions == 1 ? fabs(vx) : hypot(vx, vy);
  return __dadd_rn(velocity, sqrt(__dmul_rn(gamma, p) / s[0]));
}

// Both physical flux components from one primitive evaluation.
template <typename T>
__device__ __forceinline__ void flux_xy(T gamma, const T *s, T *fx, T *fy) {
  const Prim<T> v = primitive(gamma, s);
  fx[0] = s[1];
  fx[1] = s[1] * v.vx + v.p;
  fx[2] = s[2] * v.vx;
  fx[3] = (s[3] + v.p) * v.vx;
  fy[0] = s[2];
  fy[1] = s[1] * v.vy;
  fy[2] = s[2] * v.vy + v.p;
  fy[3] = (s[3] + v.p) * v.vy;
}

template <typename T>
__device__ __forceinline__ void normal_flux(T gamma, const T *s, T nx, T ny, T *f) {
  T fx[4], fy[4];
  flux_xy(gamma, s, fx, fy);
#pragma unroll
  for (int v = 0; v < 4; ++v)
    f[v] = nx * fx[v] + ny * fy[v];
}

template <typename T>
__device__ __forceinline__ void hllc_star(const T *s, const Prim<T> &v, T nx, T ny, T wave,
                                          T contact, T *star) {
  const T un = v.vx * nx + v.vy * ny;
  const T rho_star = s[0] * (wave - un) / (wave - contact);
  const T shift = contact - un;
  const T e_star = s[3] / s[0] + shift * (contact + v.p / (s[0] * (wave - un)));
  star[0] = rho_star;
  star[1] = rho_star * (v.vx + shift * nx);
  star[2] = rho_star * (v.vy + shift * ny);
  star[3] = rho_star * e_star;
}

// HLLC flux through a face with unit normal (nx, ny) from the left to the right state.
template <typename T>
__device__ __forceinline__ void hllc(T gamma, const T *l, const T *r, T nx, T ny, T *f) {
  const Prim<T> lv = primitive(gamma, l);
  const Prim<T> rv = primitive(gamma, r);
  const T lu = lv.vx * nx + lv.vy * ny;
  const T ru = rv.vx * nx + rv.vy * ny;
  const T lc = sound_speed(gamma, lv);
  const T rc = sound_speed(gamma, rv);
  const T sl = smin(lu - lc, ru - rc);
  const T sr = smax(lu + lc, ru + rc);
  T lf[4];
  normal_flux(gamma, l, nx, ny, lf);
  if (sl >= T(0)) {
#pragma unroll
    for (int v = 0; v < 4; ++v)
      f[v] = lf[v];
    return;
  }
  T rf[4];
  normal_flux(gamma, r, nx, ny, rf);
  if (sr <= T(0)) {
#pragma unroll
    for (int v = 0; v < 4; ++v)
      f[v] = rf[v];
    return;
  }
  const T contact = (rv.p - lv.p + l[0] * lu * (sl - lu) - r[0] * ru * (sr - ru)) /
                    (l[0] * (sl - lu) - r[0] * (sr - ru));
  T star[4];
  if (contact >= T(0)) {
    hllc_star(l, lv, nx, ny, sl, contact, star);
#pragma unroll
    for (int v = 0; v < 4; ++v)
      f[v] = lf[v] + sl * (star[v] - l[v]);
    return;
  }
  hllc_star(r, rv, nx, ny, sr, contact, star);
#pragma unroll
  for (int v = 0; v < 4; ++v)
    f[v] = rf[v] + sr * (star[v] - r[v]);
}

// Device error word: the first failure of a step, read by the host after the step.
enum ErrorCode : int {
  kOk = 0,
  kNonPhysicalAverage = 1,
  kBelowFloor = 2,
  kNonFinite = 3,
  kIndexCheck = 4 // a device index check of the checked build failed
};

__device__ __forceinline__ void raise_error(unsigned long long *word, int code, long long element) {
  const unsigned long long value =
      (static_cast<unsigned long long>(code) << 56) | (static_cast<unsigned long long>(element) & 0xffffffffffffffULL);
  atomicCAS(word, 0ULL, value);
}

// An element index read from mesh data, checked in the checked build
// (compiled with WASL_DEVICE_CHECKS, python -m wasl_b200.build --checked): an
// index outside [0, n) is recorded in the error word (code kIndexCheck, with
// the index) and replaced by 0, so the kernel neither faults nor leaves a
// barrier its block waits at; the host raises the error when the step ends.
// In the ordinary build this is the index itself.
__device__ __forceinline__ long long checked_index(long long i, long long n,
                                                   unsigned long long *word) {
#ifdef WASL_DEVICE_CHECKS
  if (i < 0 || i >= n) {
    raise_error(word, kIndexCheck, i < 0 ? -i : i);
    return 0;
  }
#else
  (void)n;
  (void)word;
#endif
  return i;
}

} // namespace wasl_b200
