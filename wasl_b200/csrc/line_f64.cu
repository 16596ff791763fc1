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
#include <algorithm>
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
__device__ __forceinline__ void trace_global(const double *u, std::int64_t ne,
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

// One element's stage: residual of `in`, scaled by 1/J, and the Shu-Osher
// combination into `out`; rho receives the new density (or scalar) modes.
// The pointers carry no __restrict__: the whole-run kernel reads buffers that
// other threads of its block wrote earlier in the same launch.
template <int V, int P>
__device__ __forceinline__ void line_element_stage(const LineStageArgs &a, std::int64_t e,
                                                   const double *in, const double *u0,
                                                   double *out, int stage, double dt,
                                                   double (&rho)[P + 1]) {
  constexpr int M = P + 1;
  constexpr int NQ = V == 4 ? P + 1 : (P > 0 ? P : 1);
  const std::int64_t ne = a.ne;
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
#pragma unroll
  for (int v = 0; v < V; ++v)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const std::int64_t idx = (static_cast<std::int64_t>(v) * M + m) * ne + e;
      const double rr = r[v][m] * inv;
      double o;
      if (stage == 0)
        o = c[v][m] + dt * rr;
      else if (stage == 1)
        o = 0.75 * u0[idx] + 0.25 * (c[v][m] + dt * rr);
      else
        o = (1.0 / 3.0) * u0[idx] + (2.0 / 3.0) * (c[v][m] + dt * rr);
      out[idx] = o;
      if (v == 0)
        rho[m] = o;
    }
}

template <int V, int P>
__global__ void __launch_bounds__(128) line_stage_f64(const LineStageArgs a) {
  constexpr int M = P + 1;
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= a.ne)
    return;
  double rho[M];
  line_element_stage<V, P>(a, e, a.in, a.u0, a.out, a.stage, a.dt ? *a.dt : a.dt_value, rho);

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

// A whole run in one launch of one CTA (meshes whose three state buffers fit
// in its shared memory): the serial run loop of cpp/src/case/serial_case_runner.cpp:107-142
// (dt clipped to land on end_time; "timestep cannot advance time" ends the
// run) around the SSP-RK3 stages of line_stage_f64, with a block barrier
// between stages instead of a kernel boundary.  The CFL step is fixed
// (fixed_dt > 0: scalar advection, cfl_timestep.cpp:55-60) or taken from the
// state each step (Euler: the largest |u| + c of the cell averages,
// cfl_timestep.cpp:33-47 and 70-76, the arithmetic of the CFL kernels).
template <int V, int P> __global__ void __launch_bounds__(512) line_run_f64(LineRunArgs r) {
  constexpr int M = P + 1;
  extern __shared__ double buffers[]; // u, stage 1, stage 2: V M ne each
  const std::int64_t ne = r.stage.ne, n = static_cast<std::int64_t>(V) * M * ne;
  double *u = buffers, *s1 = buffers + n, *s2 = buffers + 2 * n;
  for (std::int64_t i = threadIdx.x; i < n; i += blockDim.x)
    u[i] = r.state[i];
  __shared__ unsigned long long speed_bits[32];
  __shared__ int status;
  if (threadIdx.x == 0)
    status = 0;
  __syncthreads();
  double time = r.start_time;
  unsigned long long steps = 0;
  while (time < r.end_time && steps < r.max_steps) {
    double stable = r.fixed_dt;
    if (V == 4) {
      // Largest cell-average speed, with the CFL kernels' physical-state check.
      unsigned long long best = 0;
      for (std::int64_t e = threadIdx.x; e < ne; e += blockDim.x) {
        const double scale = 1.0 / sqrt(2.0);
        const double sa[4] = {scale * u[e], scale * u[M * ne + e], scale * u[2 * M * ne + e],
                              scale * u[3 * M * ne + e]};
        bool physical = true;
        const double speed = cfl_speed(r.stage.gamma, sa, 1, physical);
        if (!physical) {
          raise_error(r.error, kNonPhysicalAverage, e);
          status = 2;
        } else {
          const unsigned long long bits = __double_as_longlong(speed);
          best = bits > best ? bits : best;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_down_sync(0xffffffffu, best, off);
        best = o > best ? o : best;
      }
      if ((threadIdx.x & 31) == 0)
        speed_bits[threadIdx.x >> 5] = best;
      __syncthreads();
      best = 0;
      for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
        best = speed_bits[w] > best ? speed_bits[w] : best;
      __syncthreads();
      if (status)
        break;
      const double speed = __longlong_as_double(static_cast<long long>(best));
      stable = speed > 0.0 ? r.cfl * r.length / (speed * (2 * P + 1)) : 0.0;
    }
    const double remaining = r.end_time - time;
    const double dt = stable > 0.0 ? (remaining < stable ? remaining : stable) : remaining;
    if (dt <= 0.0 || time + dt == time) {
      status = 1; // every thread finds the same dt: the same value, one break
      break;
    }
    double *ins[3] = {u, s1, s2}, *outs[3] = {s1, s2, u};
    for (int k = 0; k < 3; ++k) {
      double rho[M];
      for (std::int64_t e = threadIdx.x; e < ne; e += blockDim.x)
        line_element_stage<V, P>(r.stage, e, ins[k], u, outs[k], k, dt, rho);
      __syncthreads();
    }
    time += dt;
    ++steps;
  }
  __syncthreads();
  for (std::int64_t i = threadIdx.x; i < n; i += blockDim.x)
    r.state[i] = u[i];
  if (threadIdx.x == 0) {
    r.result[0] = steps;
    r.result[1] = static_cast<unsigned long long>(__double_as_longlong(time));
    r.result[2] = static_cast<unsigned long long>(status);
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

template <int V, int P> void launch_run(const LineRunArgs &r, cudaStream_t s) {
  const std::size_t bytes = line_run_bytes(V, P, r.stage.ne);
  static bool opted_in[64] = {};
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64)
    throw std::runtime_error("resident run: no usable CUDA device");
  if (!opted_in[device]) {
    if (cudaFuncSetAttribute(line_run_f64<V, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kLineRunMaxBytes)) != cudaSuccess)
      throw std::runtime_error("resident run: shared memory opt-in failed");
    opted_in[device] = true;
  }
  const std::int64_t threads = std::min<std::int64_t>(512, (r.stage.ne + 31) / 32 * 32);
  line_run_f64<V, P><<<1, static_cast<unsigned>(threads), bytes, s>>>(r);
}

template <int V> void launch_run_order(int p, const LineRunArgs &r, cudaStream_t s) {
  switch (p) {
  case 0: launch_run<V, 0>(r, s); break;
  case 1: launch_run<V, 1>(r, s); break;
  case 2: launch_run<V, 2>(r, s); break;
  case 3: launch_run<V, 3>(r, s); break;
  case 4: launch_run<V, 4>(r, s); break;
  case 5: launch_run<V, 5>(r, s); break;
  case 6: launch_run<V, 6>(r, s); break;
  default: throw std::invalid_argument("line polynomial order must be 0..6");
  }
}

} // namespace

std::size_t line_run_bytes(int variables, int p, std::int64_t ne) {
  return 3 * sizeof(double) * static_cast<std::size_t>(variables) * (p + 1) *
         static_cast<std::size_t>(ne);
}

void launch_line_run_f64(int variables, int p, const LineRunArgs &r, cudaStream_t s) {
  if (line_run_bytes(variables, p, r.stage.ne) > kLineRunMaxBytes || r.stage.ne < 1)
    throw std::invalid_argument("resident run: the state does not fit in one CTA's shared memory");
  if (variables == 4)
    launch_run_order<4>(p, r, s);
  else if (variables == 1)
    launch_run_order<1>(p, r, s);
  else
    throw std::invalid_argument("resident run: 1 or 4 variables");
}

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
