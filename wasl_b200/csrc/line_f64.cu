// Plain FP64 kernels of the 1D SSP-RK3 stage on line meshes, bit-consistent
// with the reference CPU solver:
//   compressible Euler  cpp/include/wasl/dg/euler/line_residual.hpp:24-86
//   scalar advection    cpp/include/wasl/dg/scalar_advection/line_residual.hpp:48-111
// with the boundary exteriors evaluated inline:
//   Euler ends          cpp/src/boundaries/line_euler_exterior.cpp:13-43
//   scalar ends         cpp/include/wasl/boundaries/line_boundary_conditions.hpp:36-57
//
// Compiled with --fmad=false.  One thread owns one element; the reference's
// face loop runs in ascending face index and element e owns faces e (left)
// and e+1 (right), so the thread adds the volume term, then its left face,
// then its right face.  Each face's flux is computed by both of its elements
// from the same traces in the same order, so both use the same double.  Then
// rhs *= 1/J and the Shu-Osher combination (time/ssp_rk3.hpp:44-60).
#include <stdexcept>
#include <string>

#include "basis.hpp"
#include "euler_device.cuh"
#include "kernels.hpp"

namespace wasl_b200 {
namespace {

// Trace of a thread-local element at an endpoint (modes summed from 0.0).
template <int V, int M>
__device__ __forceinline__ void trace_local(const double (&c)[V][M], const double *b, double *s) {
#pragma unroll
  for (int v = 0; v < V; ++v) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m)
      acc += c[v][m] * b[m];
    s[v] = acc;
  }
}

template <int V, int M>
__device__ __forceinline__ void trace_global(const double *__restrict__ u, std::int64_t ne,
                                             std::int64_t e, const double *b, double *s) {
#pragma unroll
  for (int v = 0; v < V; ++v) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m)
      acc += u[(static_cast<std::int64_t>(v) * M + m) * ne + e] * b[m];
    s[v] = acc;
  }
}

// scalar_advection.hpp:36-42
__device__ __forceinline__ double upwind(double a, double l, double r) {
  return a >= 0.0 ? a * l : a * r;
}

template <int V, int P>
__global__ void __launch_bounds__(128) line_stage_f64(const LineStageArgs a) {
  constexpr int M = P + 1;
  constexpr int NQ = V == 4 ? P + 1 : (P > 0 ? P : 1);
  const std::int64_t ne = a.ne;
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= ne)
    return;
  const double *__restrict__ in = a.in;
  const LineTable &T = a.table;
  const double *lb = T.lb, *rb = T.rb;

  double c[V][M], r[V][M];
#pragma unroll
  for (int v = 0; v < V; ++v)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      c[v][m] = in[(static_cast<std::int64_t>(v) * M + m) * ne + e];
      r[v][m] = 0.0;
    }

  if constexpr (V == 4) {
    const double gamma = a.gamma;
    // Volume term: sum_q w_q F(u_q) dphi/dxi (line_residual.hpp:34-45).
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double s[4], fx[4], fy[4];
      trace_local<4, M>(c, T.phi[q], s);
      flux_xy(gamma, s, fx, fy);
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int m = 0; m < M; ++m)
          r[v][m] += T.w[q] * fx[v] * T.dphi[q][m];
    }
    // Left face (face e): the flux runs from the left state to this element's
    // left trace; at the left end the exterior is the periodic image (the last
    // element's right trace) or this element's own trace (outflow).
    {
      double own[4], other[4], f[4];
      trace_local<4, M>(c, lb, own);
      if (e > 0)
        trace_global<4, M>(in, ne, e - 1, rb, other);
      else if (a.left_kind == 0)
        trace_global<4, M>(in, ne, ne - 1, rb, other);
      else
        trace_local<4, M>(c, lb, other);
      hllc(gamma, other, own, 1.0, 0.0, f);
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int m = 0; m < M; ++m)
          r[v][m] += lb[m] * f[v];
    }
    // Right face (face e+1).
    {
      double own[4], other[4], f[4];
      trace_local<4, M>(c, rb, own);
      if (e + 1 < ne)
        trace_global<4, M>(in, ne, e + 1, lb, other);
      else if (a.right_kind == 0)
        trace_global<4, M>(in, ne, 0, lb, other);
      else
        trace_local<4, M>(c, rb, other);
      hllc(gamma, own, other, 1.0, 0.0, f);
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int m = 0; m < M; ++m)
          r[v][m] += -rb[m] * f[v];
    }
  } else {
    const double speed = a.speed;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double s;
      trace_local<1, M>(c, T.phi[q], &s);
      const double flux = speed * s;
#pragma unroll
      for (int m = 0; m < M; ++m)
        r[0][m] += T.w[q] * flux * T.dphi[q][m];
    }
    {
      double own, other;
      trace_local<1, M>(c, lb, &own);
      double flux;
      if (e > 0) {
        trace_global<1, M>(in, ne, e - 1, rb, &other);
        flux = upwind(speed, other, own);
      } else {
        if (a.left_kind == 1)
          other = a.left_value;
        else if (a.left_kind == 2)
          trace_local<1, M>(c, lb, &other);
        else
          trace_global<1, M>(in, ne, ne - 1, rb, &other);
        flux = upwind(speed, other, own);
      }
#pragma unroll
      for (int m = 0; m < M; ++m)
        r[0][m] += lb[m] * flux;
    }
    {
      double own, other;
      trace_local<1, M>(c, rb, &own);
      if (e + 1 < ne)
        trace_global<1, M>(in, ne, e + 1, lb, &other);
      else if (a.right_kind == 1)
        other = a.right_value;
      else if (a.right_kind == 2)
        trace_local<1, M>(c, rb, &other);
      else
        trace_global<1, M>(in, ne, 0, lb, &other);
      const double flux = upwind(speed, own, other);
#pragma unroll
      for (int m = 0; m < M; ++m)
        r[0][m] -= rb[m] * flux;
    }
  }

  const double inv = a.inv_jacobian[e];
  const double dt = a.dt ? *a.dt : a.dt_value;
  double rho[M];
#pragma unroll
  for (int v = 0; v < V; ++v)
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

  // Modal-decay sensor on the density modes (modal_decay.hpp:23-33).
  if (V == 4 && a.sense) {
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

template <int V, int P> void launch(const LineStageArgs &a, cudaStream_t s) {
  const unsigned blocks = static_cast<unsigned>((a.ne + 127) / 128);
  line_stage_f64<V, P><<<blocks, 128, 0, s>>>(a);
}

template <int V> void launch_order(int p, const LineStageArgs &a, cudaStream_t s) {
  switch (p) {
  case 0: launch<V, 0>(a, s); break;
  case 1: launch<V, 1>(a, s); break;
  case 2: launch<V, 2>(a, s); break;
  case 3: launch<V, 3>(a, s); break;
  case 4: launch<V, 4>(a, s); break;
  case 5: launch<V, 5>(a, s); break;
  case 6: launch<V, 6>(a, s); break;
  default: throw std::invalid_argument("line polynomial order must be 0..6");
  }
}

} // namespace

bool line_order_supported(int p) { return p >= 0 && p <= 6; }

void fill_line_table(int p, int points, LineTable &t) {
  if (!line_order_supported(p) || points < 1 || points > 7)
    throw std::invalid_argument("line table: unsupported order or point count");
  t = LineTable{};
  const Rule1D rule = gauss_legendre(points);
  for (int q = 0; q < points; ++q) {
    const auto b = legendre(rule.x[q], p);
    const auto g = legendre_gradient(rule.x[q], p);
    for (int m = 0; m <= p; ++m) {
      t.phi[q][m] = b[m];
      t.dphi[q][m] = g[m];
    }
    t.w[q] = rule.w[q];
  }
  const auto l = legendre(-1.0, p), r = legendre(1.0, p);
  for (int m = 0; m <= p; ++m) {
    t.lb[m] = l[m];
    t.rb[m] = r[m];
  }
}

void launch_line_stage_f64(int variables, int p, const LineStageArgs &a, cudaStream_t s) {
  if (variables == 4)
    launch_order<4>(p, a, s);
  else if (variables == 1)
    launch_order<1>(p, a, s);
  else
    throw std::invalid_argument("line stage: 1 or 4 variables");
}

} // namespace wasl_b200
