// Plain FP64 kernels of the 2D Euler SSP-RK3 stage, bit-consistent with the
// reference CPU solver.
//
// This translation unit is compiled with --fmad=false: every product and sum
// rounds separately, in the order of the reference expressions, so given the
// same inputs and tables each element's result is the double the reference
// computes.  Summation orders reproduced:
//   * modal sums over modes 0..M-1 from 0.0   (dg/modal_layout.hpp:26-36)
//   * the volume term accumulated over the points of the order-(p+2) rule,
//     rhs += w (Fx gx + Fy gy)                 (dg/euler/triangle_residual.hpp:38-57)
//   * face terms added in ascending global face index, points in order,
//     rhs -= value * basis (left) / += (right) (triangle_residual.hpp:59-102)
//   * rhs *= 1/det(J), then the Shu-Osher combination (time/ssp_rk3.hpp:44-60).
// One thread owns one element, so no atomics touch the residual.
#include <climits>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "euler_device.cuh"
#include "kernels.hpp"
#include "tri_tables.hpp"

namespace wasl_b200 {

__constant__ VolumeTable<0, double> c_vol0;
__constant__ VolumeTable<1, double> c_vol1;
__constant__ VolumeTable<2, double> c_vol2;
__constant__ VolumeTable<3, double> c_vol3;

template <int P> __device__ __forceinline__ const VolumeTable<P, double> &volume_table();
template <> __device__ __forceinline__ const VolumeTable<0, double> &volume_table<0>() { return c_vol0; }
template <> __device__ __forceinline__ const VolumeTable<1, double> &volume_table<1>() { return c_vol1; }
template <> __device__ __forceinline__ const VolumeTable<2, double> &volume_table<2>() { return c_vol2; }
template <> __device__ __forceinline__ const VolumeTable<3, double> &volume_table<3>() { return c_vol3; }

// Euler state of element `e` of a global SoA array at a point with basis `b`.
template <int M>
__device__ __forceinline__ void eval_global(const double *__restrict__ u, std::int64_t ne,
                                            std::int64_t e, const double *b, double *s) {
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m)
      acc += __ldg(u + (static_cast<std::int64_t>(v) * M + m) * ne + e) * b[m];
    s[v] = acc;
  }
}

template <int M>
__device__ __forceinline__ void eval_local(const double (&c)[4][M], const double *b, double *s) {
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m)
      acc += c[v][m] * b[m];
    s[v] = acc;
  }
}

template <int P>
__global__ void __launch_bounds__(128) euler_tri_stage_f64(const StageArgs a) {
  using S = TriShape<P>;
  constexpr int M = S::M, QV = S::QV, QF = S::QF;
  const std::int64_t ne = a.mesh.ne;
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= ne)
    return;
  const double *__restrict__ in = a.in;
  const VolumeTable<P, double> &T = volume_table<P>();
  const FaceTable<P, double> *__restrict__ F = static_cast<const FaceTable<P, double> *>(a.face_table);
  const double gamma = a.gamma;

  double c[4][M], r[4][M];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      c[v][m] = in[(static_cast<std::int64_t>(v) * M + m) * ne + e];
      r[v][m] = 0.0;
    }
  const double *__restrict__ geo = a.mesh.geo;
  const double ax = geo[e], ay = geo[ne + e], bx = geo[2 * ne + e], by = geo[3 * ne + e];

  // Volume term: sum_q w_q (F_x . d(phi)/dx + F_y . d(phi)/dy) det(J).
#pragma unroll 1
  for (int q = 0; q < QV; ++q) {
    double s[4], fx[4], fy[4];
    eval_local<M>(c, T.phi[q], s);
    flux_xy(gamma, s, fx, fy);
    const double w = T.w[q];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const double gxi = T.dxi[q][m], geta = T.deta[q][m];
      const double gx = 0.5 * (by * gxi - ay * geta);
      const double gy = 0.5 * (-bx * gxi + ax * geta);
#pragma unroll
      for (int v = 0; v < 4; ++v)
        r[v][m] += w * (fx[v] * gx + fy[v] * gy);
    }
  }

  // Face terms in ascending global face index.  A neighbour's trace at the
  // face's points is gathered once per face: each of its coefficients is
  // loaded once and added into every point's sum (each sum still runs over
  // the modes 0..M-1 from 0.0), and the sums wait in this thread's column of
  // shared memory for the point loop.
  __shared__ double outside[QF * 4][128];
  const int t = threadIdx.x;
  // u^n (read by the combination at the end of stages 2 and 3) into L1 while
  // the faces run; no registers wait on it.
  if (a.stage > 0) {
#pragma unroll
    for (int row = 0; row < 4 * M; ++row)
      asm volatile("prefetch.global.L1 [%0];\n" ::"l"(a.u0 + static_cast<std::int64_t>(row) * ne + e));
  }
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const std::int32_t raw = a.mesh.slot_nbr[k * ne + e];
    const std::int32_t nb =
        raw >= 0 ? static_cast<std::int32_t>(checked_index(raw, ne, a.error)) : raw;
    const unsigned code = a.mesh.slot_code[k * ne + e];
    const double nx = a.mesh.slot_geo[(3 * k) * ne + e];
    const double ny = a.mesh.slot_geo[(3 * k + 1) * ne + e];
    const double scale = a.mesh.slot_geo[(3 * k + 2) * ne + e];
    const bool self_left = code & 1u;
    const int le = (code >> 1) & 3u, re = (code >> 3) & 3u, flip = (code >> 5) & 1u;
    const double(*lb)[M] = F->lb[le];
    const double(*rb)[M] = F->rb[(le * 3 + re) * 2 + flip];
    if (nb >= 0) {
      const double(*ob)[M] = self_left ? rb : lb;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        double acc[QF];
#pragma unroll
        for (int q = 0; q < QF; ++q)
          acc[q] = 0.0;
#pragma unroll
        for (int m = 0; m < M; ++m) {
          const double x = __ldg(in + (static_cast<std::int64_t>(v) * M + m) * ne + nb);
#pragma unroll
          for (int q = 0; q < QF; ++q)
            acc[q] += x * ob[q][m];
        }
#pragma unroll
        for (int q = 0; q < QF; ++q)
          outside[q * 4 + v][t] = acc[q];
      }
    }
#pragma unroll 1
    for (int q = 0; q < QF; ++q) {
      double ls[4], rs[4], f[4];
      if (self_left) {
        eval_local<M>(c, lb[q], ls);
        if (nb >= 0) {
#pragma unroll
          for (int v = 0; v < 4; ++v)
            rs[v] = outside[q * 4 + v][t];
        } else if (a.mesh.boundary == 3) {
#pragma unroll
          for (int v = 0; v < 4; ++v)
            rs[v] = ls[v];
        } else {
          const std::int64_t point = static_cast<std::int64_t>(-nb - 1) * QF + q;
          eval_global<M>(in, ne, checked_index(a.mesh.donor[point], ne, a.error),
                         a.mesh.donor_basis + point * M, rs);
        }
      } else {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          ls[v] = outside[q * 4 + v][t];
        eval_local<M>(c, rb[q], rs);
      }
      hllc(gamma, ls, rs, nx, ny, f);
      const double weight = F->ew[le][q] * scale;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const double value = f[v] * weight;
        if (self_left) {
#pragma unroll
          for (int m = 0; m < M; ++m)
            r[v][m] -= value * lb[q][m];
        } else {
#pragma unroll
          for (int m = 0; m < M; ++m)
            r[v][m] += value * rb[q][m];
        }
      }
    }
  }

  // Mass inverse and the Shu-Osher combination.
  const double inv = geo[4 * ne + e];
  const double dt = a.dt ? *a.dt : a.dt_value;
  double rho[M];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const std::int64_t idx = (static_cast<std::int64_t>(v) * M + m) * ne + e;
      const double rr = r[v][m] * inv;
      double o;
      if (a.stage == 0)
        o = c[v][m] + dt * rr;
      else if (a.stage == 1)
        o = 0.75 * a.u0[idx] + 0.25 * (c[v][m] + dt * rr);
      else
        o = (1.0 / 3.0) * a.u0[idx] + (2.0 / 3.0) * (c[v][m] + dt * rr);
      a.out[idx] = o;
      if (v == 0)
        rho[m] = o;
    }

  // Modal-decay sensor on the density modes of the new stage
  // (limiting/troubled_cell/modal_decay.hpp:23-33, euler_modal_limiter.cpp:18-24).
  if (a.sense) {
    double total = 0.0, high = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      total += rho[m] * rho[m];
      if (m >= a.highest_degree_begin)
        high += rho[m] * rho[m];
    }
    const bool troubled = !(total == 0.0 || high / total <= a.threshold);
    a.flags[e] = troubled ? 1 : 0;
    const unsigned active = __activemask();
    const unsigned ballot = __ballot_sync(active, troubled);
    if (ballot) {
      const int lane = threadIdx.x & 31;
      const int leader = __ffs(ballot) - 1;
      int base = 0;
      if (lane == leader)
        base = atomicAdd(a.troubled_count, __popc(ballot));
      base = __shfl_sync(active, base, leader);
      if (troubled)
        a.troubled[base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<std::int32_t>(e);
    }
  }
}

// ---- limiter ------------------------------------------------------------------

// euler_characteristic.hpp:19-42
__device__ __forceinline__ void to_characteristic(double gamma, const double *avg,
                                                  const double *d, double nx, double ny,
                                                  double *out) {
  const Prim<double> mean = primitive(gamma, avg);
  const double un = mean.vx * nx + mean.vy * ny;
  const double ut = -mean.vx * ny + mean.vy * nx;
  const double nm = d[1] * nx + d[2] * ny;
  const double tm = -d[1] * ny + d[2] * nx;
  const double c2 = gamma * mean.p / mean.rho;
  const double c = sqrt(c2);
  const double ke = 0.5 * (un * un + ut * ut);
  const double factor = (gamma - 1.0) / c2;
  const double common = factor * (ke * d[0] - un * nm - ut * tm + d[3]);
  const double diff = (un * d[0] - nm) / c;
  out[0] = 0.5 * (common + diff);
  out[1] = d[0] - common;
  out[2] = tm - ut * d[0];
  out[3] = 0.5 * (common - diff);
}

// euler_characteristic.hpp:44-67
__device__ __forceinline__ void from_characteristic(double gamma, const double *avg,
                                                    const double *w, double nx, double ny,
                                                    double *out) {
  const Prim<double> mean = primitive(gamma, avg);
  const double un = mean.vx * nx + mean.vy * ny;
  const double ut = -mean.vx * ny + mean.vy * nx;
  const double c = sound_speed(gamma, mean);
  const double h = (avg[3] + mean.p) / avg[0];
  const double ke = 0.5 * (un * un + ut * ut);
  const double rho = w[0] + w[1] + w[3];
  const double nm = (un - c) * w[0] + un * w[1] + (un + c) * w[3];
  const double tm = ut * rho + w[2];
  const double energy = (h - un * c) * w[0] + ke * w[1] + ut * w[2] + (h + un * c) * w[3];
  out[0] = rho;
  out[1] = nx * nm - ny * tm;
  out[2] = ny * nm + nx * tm;
  out[3] = energy;
}

template <int M> __device__ __forceinline__ double smoothness(const double *c) {
  double value = 0.0;
#pragma unroll
  for (int m = 1; m < M; ++m)
    value += c[m] * c[m];
  return value;
}

// The positivity limiter on one element's modes lim[4 M]
// (cpp/include/wasl/limiting/positivity/euler_positivity.hpp:44-102): density
// scaled toward the mean to keep rho >= floor at every check point, then the
// pressure factor found by 64 bisection steps per violating point; a mean
// below a floor sets the error word instead.
template <int M>
__device__ __forceinline__ void positivity_limit(const LimitArgs &a, double *lim, std::int64_t e) {
  const double inv_root2 = 1.0 / sqrt(2.0);
  const double pavg[4] = {lim[0] * inv_root2, lim[M] * inv_root2, lim[2 * M] * inv_root2,
                          lim[3 * M] * inv_root2};
  if (!(pavg[0] > a.density_floor && primitive(a.gamma, pavg).p > a.pressure_floor)) {
    // (a NaN mean fails too) - recorded against its case when cases are tracked
    if (a.case_status)
      atomicCAS(a.case_status + a.element_case[e], 0, static_cast<int>(kBelowFloor));
    else
      raise_error(a.error, kBelowFloor, e);
    return;
  }
  // Check-point floors: the absolute floors, raised to a fraction of the mean
  // density and energy when relative_floor > 0 (forms whose fluxes evaluate
  // point states in FP32, which resolves them only to ~1e-7 of the mean).
  const double rf = a.relative_floor > 0.0 ? fmax(a.density_floor, a.relative_floor * pavg[0])
                                           : a.density_floor;
  const double pf = a.relative_floor > 0.0 ? fmax(a.pressure_floor, a.relative_floor * pavg[3])
                                           : a.pressure_floor;
  double dscale = 1.0;
  for (int pt = 0; pt < a.check_points; ++pt) {
    const double *b = a.check_basis + pt * M;
    double rho = 0.0;
    for (int m = 0; m < M; ++m)
      rho += lim[m] * b[m];
    if (rho < rf)
      dscale = smin(dscale, (pavg[0] - rf) / (pavg[0] - rho));
  }
  for (int v = 0; v < 4; ++v)
    for (int m = 1; m < M; ++m)
      lim[v * M + m] *= dscale;
  double pscale = 1.0;
  for (int pt = 0; pt < a.check_points; ++pt) {
    const double *b = a.check_basis + pt * M;
    double s[4];
    for (int v = 0; v < 4; ++v) {
      double acc = 0.0;
      for (int m = 0; m < M; ++m)
        acc += lim[v * M + m] * b[m];
      s[v] = acc;
    }
    if (primitive(a.gamma, s).p >= pf)
      continue;
    double lower = 0.0, upper = 1.0;
    for (int it = 0; it < 64; ++it) {
      const double middle = 0.5 * (lower + upper);
      double x[4];
      for (int v = 0; v < 4; ++v)
        x[v] = pavg[v] + middle * (s[v] - pavg[v]);
      if (primitive(a.gamma, x).p >= pf)
        lower = middle;
      else
        upper = middle;
    }
    pscale = smin(pscale, lower);
  }
  for (int v = 0; v < 4; ++v)
    for (int m = 1; m < M; ++m)
      lim[v * M + m] *= pscale;
}

// Whether an element provably keeps density and pressure at or above the
// check-point floors of positivity_limit at every check point, from bounds
// on the point values: |sum_{m>=1} c_m phi_m| <= sum_{m>=1} |c_m| max|phi_m|
// (max over the check points, check_bound), then the pressure's lower bound
// from the bounds on density, momentum and energy.  Where it holds the limiter
// would scale by exactly 1, so skipping it gives the same bits.  Small
// margins cover the rounding of the point sums.
template <int M> __device__ __forceinline__ bool positivity_clear(const LimitArgs &a,
                                                                  const double *lim) {
  const double inv_root2 = 1.0 / sqrt(2.0);
  const double avg[4] = {lim[0] * inv_root2, lim[M] * inv_root2, lim[2 * M] * inv_root2,
                         lim[3 * M] * inv_root2};
  if (!(avg[0] > a.density_floor && primitive(a.gamma, avg).p > a.pressure_floor))
    return false; // positivity_limit reports it
  const double rf = a.relative_floor > 0.0 ? fmax(a.density_floor, a.relative_floor * avg[0])
                                           : a.density_floor;
  const double pf = a.relative_floor > 0.0 ? fmax(a.pressure_floor, a.relative_floor * avg[3])
                                           : a.pressure_floor;
  double b[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double sum = 0.0;
#pragma unroll
    for (int m = 1; m < M; ++m)
      sum += fabs(lim[v * M + m]) * a.check_bound[m];
    b[v] = sum;
  }
  const double rho_lo = avg[0] - b[0] - 1e-12 * (avg[0] + b[0]);
  if (!(rho_lo >= rf))
    return false;
  const double mx = fabs(avg[1]) + b[1], my = fabs(avg[2]) + b[2];
  const double energy_lo = avg[3] - b[3];
  const double p_lo = (a.gamma - 1.0) * (energy_lo - 0.5 * (mx * mx + my * my) / rho_lo) -
                      1e-12 * (a.gamma - 1.0) * (fabs(avg[3]) + b[3] + 0.5 * (mx * mx + my * my) / rho_lo);
  return p_lo >= pf;
}

// The positivity limiter on every element the sensor did not flag (flags[e]
// == 0), in place: the always-on positivity of the non-reference forms (the
// reference limits positivity in troubled cells only,
// cpp/src/limiting/euler_modal_limiter.cpp:81-96).  Elements that provably
// need no scaling (positivity_clear) are skipped.
template <int M> __global__ void positivity_rest(const LimitArgs a) {
  for (std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < a.ne;
       e += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    if (a.flags && a.flags[e])
      continue;
    double lim[4 * M];
#pragma unroll
    for (int i = 0; i < 4 * M; ++i)
      lim[i] = a.state[i * a.ne + e];
    if (a.check_bound && positivity_clear<M>(a, lim))
      continue;
    positivity_limit<M>(a, lim, e);
#pragma unroll
    for (int i = 0; i < 4 * M; ++i)
      a.state[i * a.ne + e] = lim[i];
  }
}

// The warp's minimum under smin (the reference's running std::min; the
// minimum of a set does not depend on the order it is taken in).
__device__ __forceinline__ double warp_min(double x) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    x = smin(x, __shfl_xor_sync(0xffffffffu, x, off));
  return x;
}

// The stage limiter (cpp/src/limiting/euler_modal_limiter.cpp:70-98) with one
// warp per troubled element of the compacted list: the lanes share out the
// candidates (one output mode each), the characteristic projections (one mode
// of one candidate each), the WENO smoothness sums and weights (one wave each),
// the recombination, and the positivity limiter's check points, whose
// 64-step pressure bisections then run side by side instead of one after
// another.  Every value is still one lane's serial sum in the reference's
// order, so the result is the reference's bit for bit.  Limited modes go to
// scratch by list position; scatter_limited writes them back.
template <int M, int NB>
__global__ void __launch_bounds__(128) limit_f64(const LimitArgs a) {
  constexpr int W = 4 * M;  // one element's values
  constexpr int WARPS = 128 / 32;
  struct Cell {
    double target[W], cand[NB * W], tc[W], cc[NB * W], lim[W];
    double smooth[4][NB + 1], weights[4][NB + 1], sum[4];
    int slot[NB];
  };
  __shared__ Cell cells[WARPS];
  Cell &cell = cells[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int count = *a.troubled_count;
  const std::int64_t ne = a.ne;
  const double *u = a.state;
  const int warps = gridDim.x * WARPS;
  for (int k = blockIdx.x * WARPS + (threadIdx.x >> 5); k < count; k += warps) {
    const std::int64_t e = a.troubled[k];
    for (int i = lane; i < W; i += 32)
      cell.target[i] = u[i * ne + e];
    // Candidate slots in neighbour order (absent neighbours leave none).
    int n = 0;
    std::int32_t nbs[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      nbs[j] = a.neighbors[e * NB + j];
      if (nbs[j] >= 0)
        nbs[j] = static_cast<std::int32_t>(checked_index(nbs[j], ne, a.error));
      if (lane == 0)
        cell.slot[j] = nbs[j] >= 0 ? n : -1;
      n += nbs[j] >= 0 ? 1 : 0;
    }
    __syncwarp();
    // Candidates: T_{e,j} c_nbr per variable and target mode, then this
    // element's own mean as mode 0 (euler_modal_limiter.cpp:43-66).
    for (int i = lane; i < NB * W; i += 32) {
      const int j = i / W, v = (i % W) / M, t = i % M;
      if (nbs[j] < 0)
        continue;
      const double *T = a.transforms + (e * NB + j) * M * M;
      double acc = 0.0;
      for (int q = 0; q < M; ++q)
        acc += T[t * M + q] * u[(static_cast<std::int64_t>(v) * M + q) * ne + nbs[j]];
      cell.cand[(cell.slot[j] * 4 + v) * M + t] = t == 0 ? cell.target[v * M] : acc;
    }
    __syncwarp();
    const double root2 = sqrt(2.0);
    const double avg[4] = {cell.target[0] / root2, cell.target[M] / root2,
                           cell.target[2 * M] / root2, cell.target[3 * M] / root2};
    const double nx = a.normal_x[e], ny = a.normal_y[e];
    // Characteristic projection of the target (item 0) and the candidates
    // (euler_characteristic_weno.hpp:31-44), one mode of one item per lane.
    for (int i = lane; i < (n + 1) * M; i += 32) {
      const int item = i / M, m = i % M;
      const double *src = item == 0 ? cell.target : cell.cand + (item - 1) * W;
      const double d[4] = {src[m], src[M + m], src[2 * M + m], src[3 * M + m]};
      double w[4];
      to_characteristic(a.gamma, avg, d, nx, ny, w);
      double *dst = item == 0 ? cell.tc : cell.cc + (item - 1) * W;
      for (int wv = 0; wv < 4; ++wv)
        dst[wv * M + m] = w[wv];
    }
    __syncwarp();
    // Simple WENO per wave (simple_weno.hpp:21-48): smoothness per item,
    // then each wave's weights and their sum in the reference's order.
    for (int i = lane; i < 4 * (n + 1); i += 32) {
      const int wv = i / (n + 1), item = i % (n + 1);
      cell.smooth[wv][item] =
          smoothness<M>(item == 0 ? cell.tc + wv * M : cell.cc + ((item - 1) * 4 + wv) * M);
    }
    __syncwarp();
    if (lane < 4 && n > 0) {
      const int wv = lane;
      const double td = 1e-12 + cell.smooth[wv][0];
      cell.weights[wv][0] = 0.5 / (td * td);
      double sum = cell.weights[wv][0];
      const double ideal = 0.5 / static_cast<double>(n);
      for (int i = 0; i < n; ++i) {
        const double dd = 1e-12 + cell.smooth[wv][i + 1];
        cell.weights[wv][i + 1] = ideal / (dd * dd);
        sum += cell.weights[wv][i + 1];
      }
      cell.sum[wv] = sum;
    }
    __syncwarp();
    // Recombined characteristic modes (mode 0 kept), into lim as scratch.
    for (int i = lane; i < W; i += 32) {
      const int wv = i / M, m = i % M;
      const double *tw = cell.tc + wv * M;
      double out = tw[m];
      if (n > 0 && m > 0) {
        double value = cell.weights[wv][0] * tw[m];
        for (int c = 0; c < n; ++c)
          value += cell.weights[wv][c + 1] * cell.cc[(c * 4 + wv) * M + m];
        out = value / cell.sum[wv];
      }
      cell.lim[i] = out;
    }
    __syncwarp();
    // Back to conserved variables, one mode per lane; mode 0 is the target's.
    double back[W > 32 ? (W + 31) / 32 * 4 : 4];
    {
      int r = 0;
      for (int m = lane; m < M; m += 32, ++r) {
        const double w[4] = {cell.lim[m], cell.lim[M + m], cell.lim[2 * M + m],
                             cell.lim[3 * M + m]};
        from_characteristic(a.gamma, avg, w, nx, ny, back + 4 * r);
      }
    }
    __syncwarp();
    {
      int r = 0;
      for (int m = lane; m < M; m += 32, ++r)
        for (int v = 0; v < 4; ++v)
          cell.lim[v * M + m] = m == 0 ? cell.target[v * M] : back[4 * r + v];
    }
    __syncwarp();
    // Positivity (euler_positivity.hpp:63-102), one check point per lane.
    const double inv_root2 = 1.0 / sqrt(2.0);
    const double pavg[4] = {cell.lim[0] * inv_root2, cell.lim[M] * inv_root2,
                            cell.lim[2 * M] * inv_root2, cell.lim[3 * M] * inv_root2};
    if (!(pavg[0] > a.density_floor && primitive(a.gamma, pavg).p > a.pressure_floor)) {
      if (lane == 0) {
        if (a.case_status)
          atomicCAS(a.case_status + a.element_case[e], 0, static_cast<int>(kBelowFloor));
        else
          raise_error(a.error, kBelowFloor, e);
      }
    } else {
      const double rf = a.relative_floor > 0.0
                            ? fmax(a.density_floor, a.relative_floor * pavg[0])
                            : a.density_floor;
      const double pf = a.relative_floor > 0.0
                            ? fmax(a.pressure_floor, a.relative_floor * pavg[3])
                            : a.pressure_floor;
      double dscale = 1.0;
      for (int pt = lane; pt < a.check_points; pt += 32) {
        const double *b = a.check_basis + pt * M;
        double rho = 0.0;
        for (int m = 0; m < M; ++m)
          rho += cell.lim[m] * b[m];
        if (rho < rf)
          dscale = smin(dscale, (pavg[0] - rf) / (pavg[0] - rho));
      }
      dscale = warp_min(dscale);
      __syncwarp();
      for (int i = lane; i < W; i += 32)
        if (i % M != 0)
          cell.lim[i] *= dscale;
      __syncwarp();
      double pscale = 1.0;
      for (int pt = lane; pt < a.check_points; pt += 32) {
        const double *b = a.check_basis + pt * M;
        double st[4];
        for (int v = 0; v < 4; ++v) {
          double acc = 0.0;
          for (int m = 0; m < M; ++m)
            acc += cell.lim[v * M + m] * b[m];
          st[v] = acc;
        }
        if (primitive(a.gamma, st).p >= pf)
          continue;
        double lower = 0.0, upper = 1.0;
        for (int it = 0; it < 64; ++it) {
          const double middle = 0.5 * (lower + upper);
          double x[4];
          for (int v = 0; v < 4; ++v)
            x[v] = pavg[v] + middle * (st[v] - pavg[v]);
          if (primitive(a.gamma, x).p >= pf)
            lower = middle;
          else
            upper = middle;
        }
        pscale = smin(pscale, lower);
      }
      pscale = warp_min(pscale);
      __syncwarp();
      for (int i = lane; i < W; i += 32)
        if (i % M != 0)
          cell.lim[i] *= pscale;
    }
    __syncwarp();
    double *dst = a.limited + static_cast<std::int64_t>(k) * W;
    for (int i = lane; i < W; i += 32)
      dst[i] = cell.lim[i];
    __syncwarp();
  }
}

template <int M>
__global__ void scatter_limited(double *state, std::int64_t ne, const std::int32_t *troubled,
                                const std::int32_t *count, const double *limited) {
  const int n = *count;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const std::int64_t e = troubled[k];
#pragma unroll
    for (int i = 0; i < 4 * M; ++i)
      state[i * ne + e] = limited[static_cast<std::int64_t>(k) * 4 * M + i];
  }
}

// Modal-decay sensor over a whole state (the stage kernels fuse it instead).
template <int M>
__global__ void sense_f64(SenseArgs a) {
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= a.ne)
    return;
  double total = 0.0, high = 0.0;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const double value = a.state[static_cast<std::int64_t>(m) * a.ne + e];
    total += value * value;
    if (m >= a.highest_degree_begin)
      high += value * value;
  }
  const bool troubled = !(total == 0.0 || high / total <= a.threshold);
  a.flags[e] = troubled ? 1 : 0;
  if (troubled)
    a.troubled[atomicAdd(a.troubled_count, 1)] = static_cast<std::int32_t>(e);
}

// ---- CFL ------------------------------------------------------------------------

__device__ __forceinline__ double cell_speed(const CflArgs &a, std::int64_t e, bool &physical) {
  const double scale = 1.0 / sqrt(2.0);
  const std::int64_t plane = static_cast<std::int64_t>(a.M) * a.ne;
  const double s[4] = {scale * a.state[e], scale * a.state[plane + e],
                       scale * a.state[2 * plane + e], scale * a.state[3 * plane + e]};
  return cfl_speed(a.gamma, s, a.dimensions, physical);
}

__global__ void cfl_max(const CflArgs a) {
  __shared__ unsigned long long block_max[32];
  unsigned long long best = 0;
  for (std::int64_t e = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; e < a.ne;
       e += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    bool physical = true;
    const double speed = cell_speed(a, e, physical);
    if (!physical) {
      raise_error(a.error, kNonPhysicalAverage, e);
      continue;
    }
    const unsigned long long bits = __double_as_longlong(speed);
    best = bits > best ? bits : best;
  }
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_down_sync(0xffffffffu, best, off);
    best = o > best ? o : best;
  }
  if ((threadIdx.x & 31) == 0)
    block_max[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    best = threadIdx.x < (blockDim.x >> 5) ? block_max[threadIdx.x] : 0ULL;
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long o = __shfl_down_sync(0xffffffffu, best, off);
      best = o > best ? o : best;
    }
    if (threadIdx.x == 0)
      atomicMax(a.result, best);
  }
}

// The larger of two (speed bits, element) pairs; on equal speeds the smaller
// element, as the reference's first strict maximum in element order.
__device__ __forceinline__ void better_pair(unsigned long long &best, long long &arg,
                                            unsigned long long other, long long other_arg) {
  if (other > best || (other == best && other_arg < arg)) {
    best = other;
    arg = other_arg;
  }
}

// Block-wide pair reduction; thread 0 returns the block's pair.
__device__ __forceinline__ void block_pair(unsigned long long &best, long long &arg) {
  __shared__ unsigned long long speeds[32];
  __shared__ long long args[32];
  for (int off = 16; off > 0; off >>= 1)
    better_pair(best, arg, __shfl_down_sync(0xffffffffu, best, off),
                __shfl_down_sync(0xffffffffu, arg, off));
  if ((threadIdx.x & 31) == 0) {
    speeds[threadIdx.x >> 5] = best;
    args[threadIdx.x >> 5] = arg;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool live = threadIdx.x < (blockDim.x >> 5);
    best = live ? speeds[threadIdx.x] : 0ULL;
    arg = live ? args[threadIdx.x] : LLONG_MAX;
    for (int off = 16; off > 0; off >>= 1)
      better_pair(best, arg, __shfl_down_sync(0xffffffffu, best, off),
                  __shfl_down_sync(0xffffffffu, arg, off));
  }
  __syncthreads();
}

// The whole CFL reduction in one pass over the cell averages: each block
// reduces its elements to (largest speed, smallest element reaching it) and
// stores the pair; the last block to finish reduces the pairs, records the
// winner's mode-0 coefficients and forms dt (cfl_timestep.cpp:70-84), then
// re-arms the block counter.
__global__ void __launch_bounds__(256) cfl_reduce(const CflArgs a) {
  unsigned long long best = 0;
  long long arg = LLONG_MAX;
  for (std::int64_t e = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; e < a.ne;
       e += static_cast<std::int64_t>(gridDim.x) * blockDim.x) {
    bool physical = true;
    const double speed = cell_speed(a, e, physical);
    if (!physical) {
      raise_error(a.error, kNonPhysicalAverage, e);
      continue;
    }
    // The tie key is the caller's element index (high word); the storage
    // column rides in the low word.
    const long long key = a.order ? a.order[e] : e;
    better_pair(best, arg, static_cast<unsigned long long>(__double_as_longlong(speed)),
                (key << 32) | e);
  }
  block_pair(best, arg);
  __shared__ bool last;
  unsigned long long *pairs = a.result + 16;
  if (threadIdx.x == 0) {
    pairs[2 * blockIdx.x] = best;
    pairs[2 * blockIdx.x + 1] = static_cast<unsigned long long>(arg);
    __threadfence();
    last = atomicAdd(a.result + 8, 1ULL) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  best = 0;
  arg = LLONG_MAX;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
    better_pair(best, arg, __ldcg(pairs + 2 * b), static_cast<long long>(__ldcg(pairs + 2 * b + 1)));
  block_pair(best, arg);
  if (threadIdx.x == 0) {
    const std::int64_t e = arg == LLONG_MAX ? 0 : (arg & 0xffffffffLL);
    const double speed = __longlong_as_double(static_cast<long long>(best));
    const std::int64_t plane = static_cast<std::int64_t>(a.M) * a.ne;
    a.result[0] = best;
    a.result[1] = ~static_cast<unsigned long long>(arg == LLONG_MAX ? 0 : arg >> 32);
    for (int v = 0; v < 4; ++v)
      a.result[2 + v] = static_cast<unsigned long long>(__double_as_longlong(a.state[v * plane + e]));
    const double dt = speed > 0.0 ? a.cfl * a.length / (speed * (2 * a.p + 1)) : 0.0;
    a.result[6] = static_cast<unsigned long long>(__double_as_longlong(dt));
    if (a.dt)
      *a.dt = dt;
    a.result[8] = 0;
  }
}

// dt from a reduced speed word per case (the finish step of the CFL kernels),
// then the word is zeroed for the next reduction.
__global__ void dt_from_speed(std::int64_t cases, unsigned long long *speed, double cfl,
                              const double *length, const int *p, double length_all, int p_all,
                              double *dt, double *elapsed, const int *status) {
  // As a programmatic dependent launch: the next launch (the step's first
  // stage) may start its CTAs now, and this kernel waits for the launch
  // before it (the last stage, which max-reduced the speed) to complete.
  // Launched plainly, both are no-ops.
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  const std::int64_t c = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= cases)
    return;
  const double v = __longlong_as_double(static_cast<long long>(speed[c]));
  const double h = length ? length[c] : length_all;
  const int order = p ? p[c] : p_all;
  // A failed case is frozen: dt 0.
  const double step = v > 0.0 && !(status && status[c]) ? cfl * h / (v * (2 * order + 1)) : 0.0;
  dt[c] = step;
  if (elapsed)
    elapsed[c] += step;
  speed[c] = 0ULL;
}

// ---- host launchers -------------------------------------------------------------

namespace {

void check(cudaError_t rc, const char *what) {
  if (rc != cudaSuccess)
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(rc));
}

template <int P> void upload_volume(const void *symbol) {
  static VolumeTable<P, double> table;
  fill_volume_table<P, double>(table);
  check(cudaMemcpyToSymbol(symbol, &table, sizeof(table)), "upload volume table");
}

template <int P> void stage(const StageArgs &a, cudaStream_t s) {
  const unsigned blocks = static_cast<unsigned>((a.mesh.ne + 127) / 128);
  euler_tri_stage_f64<P><<<blocks, 128, 0, s>>>(a);
}

} // namespace

bool euler_tri_order_supported(int p) { return p >= 0 && p <= 3; }

void upload_euler_tri_tables_f64(int p) {
  switch (p) {
  case 0: upload_volume<0>(reinterpret_cast<const void *>(&c_vol0)); break;
  case 1: upload_volume<1>(reinterpret_cast<const void *>(&c_vol1)); break;
  case 2: upload_volume<2>(reinterpret_cast<const void *>(&c_vol2)); break;
  case 3: upload_volume<3>(reinterpret_cast<const void *>(&c_vol3)); break;
  default: throw std::invalid_argument("triangle polynomial order must be 0..3");
  }
}

void launch_euler_tri_stage_f64(int p, const StageArgs &a, cudaStream_t s) {
  switch (p) {
  case 0: stage<0>(a, s); break;
  case 1: stage<1>(a, s); break;
  case 2: stage<2>(a, s); break;
  case 3: stage<3>(a, s); break;
  default: throw std::invalid_argument("triangle polynomial order must be 0..3");
  }
}

void launch_limit_f64(int M, int NB, const LimitArgs &a, cudaStream_t s) {
  // Four warps (troubled elements) per block.
  const unsigned blocks = static_cast<unsigned>(std::min<std::int64_t>((a.ne + 3) / 4, 148 * 16));
  const unsigned sblocks = static_cast<unsigned>(std::min<std::int64_t>((a.ne + 255) / 256, 148 * 8));
  const unsigned pblocks = static_cast<unsigned>(std::min<std::int64_t>((a.ne + 127) / 128, 148 * 16));
#define WASL_LIMIT(MM, NN)                                                                     \
  if (M == MM && NB == NN) {                                                                   \
    limit_f64<MM, NN><<<blocks, 128, 0, s>>>(a);                                               \
    scatter_limited<MM><<<sblocks, 256, 0, s>>>(a.state, a.ne, a.troubled, a.troubled_count,   \
                                                 a.limited);                                   \
    if (a.positivity_all)                                                                      \
      positivity_rest<MM><<<pblocks, 128, 0, s>>>(a);                                          \
    return;                                                                                    \
  }
  WASL_LIMIT(3, 3)
  WASL_LIMIT(6, 3)
  WASL_LIMIT(10, 3)
  WASL_LIMIT(2, 2)
  WASL_LIMIT(3, 2)
  WASL_LIMIT(4, 2)
  WASL_LIMIT(5, 2)
  WASL_LIMIT(6, 2)
  WASL_LIMIT(7, 2)
#undef WASL_LIMIT
  throw std::invalid_argument("limiter: unsupported mode count");
}

void launch_sense_f64(int M, const SenseArgs &a, cudaStream_t s) {
  const unsigned blocks = static_cast<unsigned>((a.ne + 255) / 256);
  switch (M) {
  case 1: sense_f64<1><<<blocks, 256, 0, s>>>(a); break;
  case 2: sense_f64<2><<<blocks, 256, 0, s>>>(a); break;
  case 3: sense_f64<3><<<blocks, 256, 0, s>>>(a); break;
  case 4: sense_f64<4><<<blocks, 256, 0, s>>>(a); break;
  case 5: sense_f64<5><<<blocks, 256, 0, s>>>(a); break;
  case 6: sense_f64<6><<<blocks, 256, 0, s>>>(a); break;
  case 7: sense_f64<7><<<blocks, 256, 0, s>>>(a); break;
  case 10: sense_f64<10><<<blocks, 256, 0, s>>>(a); break;
  default: throw std::invalid_argument("sensor: unsupported mode count");
  }
}

std::vector<double> positivity_check_bound(const std::vector<double> &check_basis, int M) {
  std::vector<double> bound(M, 0.0);
  for (std::size_t i = 0; i < check_basis.size(); ++i)
    bound[i % M] = std::max(bound[i % M], std::fabs(check_basis[i]));
  return bound;
}

void launch_dt_from_speed(std::int64_t cases, unsigned long long *speed, double cfl,
                          const double *length, const int *p, double length_all, int p_all,
                          double *dt, double *elapsed, const int *status, cudaStream_t s,
                          bool dependent) {
  if (!dependent) {
    dt_from_speed<<<static_cast<unsigned>((cases + 255) / 256), 256, 0, s>>>(
        cases, speed, cfl, length, p, length_all, p_all, dt, elapsed, status);
    return;
  }
  cudaLaunchConfig_t config = {};
  config.gridDim = dim3(static_cast<unsigned>((cases + 255) / 256));
  config.blockDim = dim3(256);
  config.stream = s;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attribute[0].val.programmaticStreamSerializationAllowed = 1;
  config.attrs = attribute;
  config.numAttrs = 1;
  check(cudaLaunchKernelEx(&config, dt_from_speed, cases, speed, cfl, length, p, length_all, p_all,
                           dt, elapsed, status),
        "dt launch");
}

void launch_cfl_speed(const CflArgs &a, cudaStream_t s) {
  check(cudaMemsetAsync(a.result, 0, sizeof(unsigned long long), s), "cfl reset");
  const unsigned blocks = static_cast<unsigned>(std::min<std::int64_t>((a.ne + 255) / 256, 148 * 4));
  cfl_max<<<blocks, 256, 0, s>>>(a);
}

void launch_cfl(const CflArgs &a, cudaStream_t s) {
  check(cudaMemsetAsync(a.result, 0, 16 * sizeof(unsigned long long), s), "cfl reset");
  const unsigned blocks =
      static_cast<unsigned>(std::min<std::int64_t>((a.ne + 255) / 256, kCflBlocks));
  cfl_reduce<<<blocks, 256, 0, s>>>(a);
}

} // namespace wasl_b200
