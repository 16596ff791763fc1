// Plain FP64 kernel of the 2D scalar-advection SSP-RK3 stage on triangles
// (cpp/include/wasl/dg/scalar_advection/triangle_residual.hpp:25-104, constant
// velocity), bit-consistent with the reference CPU solver.
//
// Compiled with --fmad=false.  The layout and face slots are the 2D Euler
// kernels' (one thread per element, faces in ascending global face index);
// differences from the Euler residual, all as the reference writes them:
//   * the volume rule has order p ((p+1)^2 points), not p+2;
//   * volume: rhs += w_q u_q (v . grad phi) with the scaled gradient;
//   * faces: upwind flux (v.n) u_upwind, rhs -= (weight phi) flux on the left
//     side and += on the right, weight = edge weight x the left edge's scale;
//   * periodic exterior: the donor's modes against the stored donor basis
//     (periodic_triangle_trace.cpp:69-82).
// State [mode][element].
#include <stdexcept>

#include "kernels.hpp"
#include "tri_tables.hpp"

namespace wasl_b200 {

template <int P> struct ScalarTriVolume {
  static constexpr int M = TriShape<P>::M, QV = (P + 1) * (P + 1);
  double phi[QV][M];
  double dxi[QV][M];
  double deta[QV][M];
  double w[QV];
};

__constant__ ScalarTriVolume<0> c_svol0;
__constant__ ScalarTriVolume<1> c_svol1;
__constant__ ScalarTriVolume<2> c_svol2;
__constant__ ScalarTriVolume<3> c_svol3;

namespace {

template <int P> __device__ __forceinline__ const ScalarTriVolume<P> &svol();
template <> __device__ __forceinline__ const ScalarTriVolume<0> &svol<0>() { return c_svol0; }
template <> __device__ __forceinline__ const ScalarTriVolume<1> &svol<1>() { return c_svol1; }
template <> __device__ __forceinline__ const ScalarTriVolume<2> &svol<2>() { return c_svol2; }
template <> __device__ __forceinline__ const ScalarTriVolume<3> &svol<3>() { return c_svol3; }

template <int M>
__device__ __forceinline__ double modal_sum(const double (&c)[M], const double *b) {
  double value = 0.0;
#pragma unroll
  for (int m = 0; m < M; ++m)
    value += c[m] * b[m];
  return value;
}

template <int M>
__device__ __forceinline__ double modal_sum_global(const double *__restrict__ u, std::int64_t ne,
                                                   std::int64_t e, const double *b) {
  double value = 0.0;
#pragma unroll
  for (int m = 0; m < M; ++m)
    value += u[static_cast<std::int64_t>(m) * ne + e] * b[m];
  return value;
}

template <int P>
__global__ void __launch_bounds__(128) scalar_tri_stage_f64(const StageArgs a) {
  using S = TriShape<P>;
  constexpr int M = S::M, QF = S::QF, QV = ScalarTriVolume<P>::QV;
  const std::int64_t ne = a.mesh.ne;
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= ne)
    return;
  const double *__restrict__ in = a.in;
  const ScalarTriVolume<P> &T = svol<P>();
  const FaceTable<P, double> *__restrict__ F = static_cast<const FaceTable<P, double> *>(a.face_table);
  const double vx = a.velocity_x, vy = a.velocity_y;

  double c[M], r[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    c[m] = in[static_cast<std::int64_t>(m) * ne + e];
    r[m] = 0.0;
  }
  const double *__restrict__ geo = a.mesh.geo;
  const double ax = geo[e], ay = geo[ne + e], bx = geo[2 * ne + e], by = geo[3 * ne + e];

#pragma unroll 1
  for (int q = 0; q < QV; ++q) {
    const double state = modal_sum<M>(c, T.phi[q]);
    const double ws = T.w[q] * state;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const double gx = 0.5 * (by * T.dxi[q][m] - ay * T.deta[q][m]);
      const double gy = 0.5 * (-bx * T.dxi[q][m] + ax * T.deta[q][m]);
      r[m] += ws * (vx * gx + vy * gy);
    }
  }

  // u^n (read by the combination at the end of stages 2 and 3) into L1 while
  // the faces run.
  if (a.stage > 0) {
#pragma unroll
    for (int m = 0; m < M; ++m)
      asm volatile("prefetch.global.L1 [%0];\n" ::"l"(a.u0 + static_cast<std::int64_t>(m) * ne + e));
  }

#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const std::int32_t nb = a.mesh.slot_nbr[k * ne + e];
    const unsigned code = a.mesh.slot_code[k * ne + e];
    const double nx = a.mesh.slot_geo[(3 * k) * ne + e];
    const double ny = a.mesh.slot_geo[(3 * k + 1) * ne + e];
    const double scale = a.mesh.slot_geo[(3 * k + 2) * ne + e];
    const bool self_left = code & 1u;
    const int le = (code >> 1) & 3u, re = (code >> 3) & 3u, flip = (code >> 5) & 1u;
    const double(*lb)[M] = F->lb[le];
    const double(*rb)[M] = F->rb[(le * 3 + re) * 2 + flip];
    const double normal_speed = vx * nx + vy * ny;
    // The neighbour's trace at every point of the face from one load of each
    // of its coefficients (each sum over the modes 0..M-1 from 0.0, as
    // modal_sum_global).
    double outside[QF];
    if (nb >= 0) {
      const double(*ob)[M] = self_left ? rb : lb;
#pragma unroll
      for (int q = 0; q < QF; ++q)
        outside[q] = 0.0;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const double x = in[static_cast<std::int64_t>(m) * ne + nb];
#pragma unroll
        for (int q = 0; q < QF; ++q)
          outside[q] += x * ob[q][m];
      }
    }
#pragma unroll
    for (int q = 0; q < QF; ++q) {
      double ls, rs;
      if (self_left) {
        ls = modal_sum<M>(c, lb[q]);
        if (nb >= 0) {
          rs = outside[q];
        } else {
          const std::int64_t point = static_cast<std::int64_t>(-nb - 1) * QF + q;
          rs = modal_sum_global<M>(in, ne, a.mesh.donor[point], a.mesh.donor_basis + point * M);
        }
      } else {
        ls = outside[q];
        rs = modal_sum<M>(c, rb[q]);
      }
      const double flux = normal_speed * (normal_speed >= 0.0 ? ls : rs);
      const double weight = F->ew[le][q] * scale;
      if (self_left) {
#pragma unroll
        for (int m = 0; m < M; ++m)
          r[m] -= weight * lb[q][m] * flux;
      } else {
#pragma unroll
        for (int m = 0; m < M; ++m)
          r[m] += weight * rb[q][m] * flux;
      }
    }
  }

  const double inv = geo[4 * ne + e];
  const double dt = a.dt ? *a.dt : a.dt_value;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const std::int64_t idx = static_cast<std::int64_t>(m) * ne + e;
    const double rr = r[m] * inv;
    double o;
    if (a.stage == 0)
      o = c[m] + dt * rr;
    else if (a.stage == 1)
      o = 0.75 * a.u0[idx] + 0.25 * (c[m] + dt * rr);
    else
      o = (1.0 / 3.0) * a.u0[idx] + (2.0 / 3.0) * (c[m] + dt * rr);
    a.out[idx] = o;
  }
}

template <int P> void upload(const void *symbol) {
  constexpr int M = TriShape<P>::M, QV = ScalarTriVolume<P>::QV;
  static ScalarTriVolume<P> t;
  const Rule2D rule = triangle_rule(P);
  std::vector<double> gx, ge;
  for (int q = 0; q < QV; ++q) {
    const auto b = dubiner(rule.xi[q], rule.eta[q], P);
    dubiner_gradient(rule.xi[q], rule.eta[q], P, gx, ge);
    for (int m = 0; m < M; ++m) {
      t.phi[q][m] = b[m];
      t.dxi[q][m] = gx[m];
      t.deta[q][m] = ge[m];
    }
    t.w[q] = rule.w[q];
  }
  const cudaError_t rc = cudaMemcpyToSymbol(symbol, &t, sizeof(t));
  if (rc != cudaSuccess)
    throw std::runtime_error(std::string("upload scalar volume table: ") + cudaGetErrorString(rc));
}

template <int P> void stage(const StageArgs &a, cudaStream_t s) {
  const unsigned blocks = static_cast<unsigned>((a.mesh.ne + 127) / 128);
  scalar_tri_stage_f64<P><<<blocks, 128, 0, s>>>(a);
}

} // namespace

void upload_scalar_tri_tables(int p) {
  switch (p) {
  case 0: upload<0>(reinterpret_cast<const void *>(&c_svol0)); break;
  case 1: upload<1>(reinterpret_cast<const void *>(&c_svol1)); break;
  case 2: upload<2>(reinterpret_cast<const void *>(&c_svol2)); break;
  case 3: upload<3>(reinterpret_cast<const void *>(&c_svol3)); break;
  default: throw std::invalid_argument("triangle polynomial order must be 0..3");
  }
}

void launch_scalar_tri_stage_f64(int p, const StageArgs &a, cudaStream_t s) {
  switch (p) {
  case 0: stage<0>(a, s); break;
  case 1: stage<1>(a, s); break;
  case 2: stage<2>(a, s); break;
  case 3: stage<3>(a, s); break;
  default: throw std::invalid_argument("triangle polynomial order must be 0..3");
  }
}

} // namespace wasl_b200
