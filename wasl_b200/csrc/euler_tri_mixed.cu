// Mixed-precision 2D Euler SSP-RK3 stage (the fast form).
//
// Same discretization as the plain path (order-(p+2) volume rule, HLLC faces,
// SSP-RK3), arranged so that FP32 only ever carries small quantities:
//   * each element's state is split into its cell average U_bar = c0 phi0
//     (FP64) and the high-mode part dU(x) = sum_{m>=1} c_m phi_m(x) (FP32);
//   * for the high modes the element's own mean flux F(U_bar) drops out: its
//     volume term F(U_bar) . sum_q w grad(phi_m) equals its face term
//     F(U_bar) . sum_faces w phi_m n (divergence theorem; both rules are exact
//     for these degrees), so only perturbations remain:
//       volume  dF = F(U_bar + dU) - F(U_bar), evaluated in perturbation form
//               (every term proportional to dU) and projected through the
//               contravariant fluxes G_xi = w (b_y dF_x - b_x dF_y),
//               G_eta = w (a_x dF_y - a_y dF_x);
//       faces   HLLC(U_L, U_R).n - F(U_bar).n, from an HLLC written in
//               perturbation form around the face's left mean;
//     all in FP32 with FMA;
//   * mode 0 (the cell averages) takes the full face value, the left mean's
//     normal flux in FP64 plus the FP32 perturbation, computed identically by
//     both sides of a face, so mass, momentum and energy are conserved to FP64
//     round-off and a uniform state stays exactly uniform;
//   * the residual scaling and the Shu-Osher combination are FP64.
// The plain kernels (euler_tri_f64.cu) remain the bit-consistent drop-in.
#include <stdexcept>
#include <type_traits>

#include "euler_device.cuh"
#include "kernels.hpp"
#include "tri_tables.hpp"

namespace wasl_b200 {

// FP32 volume tables for modes 1..M-1 on the collapsed rule of order R
// ((R+1)^2 points, exact to degree 2R; the reference residual uses R = p+2).
// Volume rule R: the collapsed rule of order R ((R+1)^2 points, exact to
// degree 2R), or, for R = 0, the fully symmetric rule of degree 2P (3, 6 and
// 12 points at P1, P2, P3: the collapsed order-P rule's exactness with fewer
// points).
template <int P, int R> struct VolumeRuleSize {
  static constexpr int value = (R + 1) * (R + 1);
};
template <int P> struct VolumeRuleSize<P, 0> {
  static constexpr int value = P == 1 ? 3 : (P == 2 ? 6 : 12);
};

template <int P, int R> struct MixedVolume {
  static constexpr int M = TriShape<P>::M, QV = VolumeRuleSize<P, R>::value, H = M - 1;
  float phi[QV][H > 0 ? H : 1];
  float dxi[QV][H > 0 ? H : 1];
  float deta[QV][H > 0 ? H : 1];
  float w[QV];
};

template <int P, int R> __constant__ MixedVolume<P, R> c_mix;
// FP64 sum of the reference edge weights of each local edge.
template <int P> __constant__ double c_edge_wsum[3];

// Primitive values of a cell average, FP64, with one reciprocal.  Written
// with explicit round-to-nearest operations (no multiply-add contraction), so
// every call site produces the same bits: the two sides of a face evaluate it
// independently in the tile kernel and must agree exactly.
struct MeanState {
  double rho, mx, my, e, u, v, p, h; // h = E + p
};

__device__ __forceinline__ MeanState mean_state(double gamma, const double *s) {
  MeanState m;
  m.rho = s[0];
  m.mx = s[1];
  m.my = s[2];
  m.e = s[3];
  const double inv = 1.0 / s[0];
  m.u = __dmul_rn(s[1], inv);
  m.v = __dmul_rn(s[2], inv);
  const double kinetic = __dmul_rn(0.5, __dadd_rn(__dmul_rn(s[1], m.u), __dmul_rn(s[2], m.v)));
  m.p = __dmul_rn(gamma - 1.0, __dsub_rn(s[3], kinetic));
  m.h = __dadd_rn(s[3], m.p);
  return m;
}

// Physical flux of a cell average along n, FP64 (explicit rounding as above).
__device__ __forceinline__ void mean_normal_flux(const MeanState &m, double nx, double ny,
                                                 double *f) {
  const double un = __dadd_rn(__dmul_rn(m.u, nx), __dmul_rn(m.v, ny));
  f[0] = __dmul_rn(m.rho, un);
  f[1] = __dadd_rn(__dmul_rn(m.mx, un), __dmul_rn(m.p, nx));
  f[2] = __dadd_rn(__dmul_rn(m.my, un), __dmul_rn(m.p, ny));
  f[3] = __dmul_rn(m.h, un);
}

// HLLC in FP64 with shared reciprocals: the flux of hllc() with fewer divisions.
__device__ __forceinline__ void hllc_fast(double gamma, const double *l, const double *r, double nx,
                                          double ny, double *f) {
  const double il = 1.0 / l[0], ir = 1.0 / r[0];
  const double lu = l[1] * il, lv = l[2] * il, ru = r[1] * ir, rv = r[2] * ir;
  const double lp = (gamma - 1.0) * (l[3] - 0.5 * (l[1] * lu + l[2] * lv));
  const double rp = (gamma - 1.0) * (r[3] - 0.5 * (r[1] * ru + r[2] * rv));
  const double lun = lu * nx + lv * ny, run = ru * nx + rv * ny;
  const double lc = sqrt(gamma * lp * il), rc = sqrt(gamma * rp * ir);
  const double sl = fmin(lun - lc, run - rc);
  const double sr = fmax(lun + lc, run + rc);
  if (sl >= 0.0) {
    f[0] = l[0] * lun;
    f[1] = l[1] * lun + lp * nx;
    f[2] = l[2] * lun + lp * ny;
    f[3] = (l[3] + lp) * lun;
    return;
  }
  if (sr <= 0.0) {
    f[0] = r[0] * run;
    f[1] = r[1] * run + rp * nx;
    f[2] = r[2] * run + rp * ny;
    f[3] = (r[3] + rp) * run;
    return;
  }
  const double dl = l[0] * (sl - lun), dr = r[0] * (sr - run);
  const double contact = (rp - lp + lun * dl - run * dr) / (dl - dr);
  const bool left = contact >= 0.0;
  const double *s = left ? l : r;
  const double is = left ? il : ir;
  const double un = left ? lun : run, ps = left ? lp : rp, wave = left ? sl : sr;
  const double vx = left ? lu : ru, vy = left ? lv : rv;
  const double d = s[0] * (wave - un);
  const double rho_star = d / (wave - contact);
  const double shift = contact - un;
  const double e_star = s[3] * is + shift * (contact + ps / d);
  f[0] = s[0] * un + wave * (rho_star - s[0]);
  f[1] = s[1] * un + ps * nx + wave * (rho_star * (vx + shift * nx) - s[1]);
  f[2] = s[2] * un + ps * ny + wave * (rho_star * (vy + shift * ny) - s[2]);
  f[3] = (s[3] + ps) * un + wave * (rho_star * e_star - s[3]);
}

// A reference state (a cell average) in FP32 for the perturbation formulas.
struct Ref32 {
  float rho, u, v, e, h, mx, my, p;
};

__device__ __forceinline__ Ref32 ref32(const MeanState &m) {
  return {static_cast<float>(m.rho), static_cast<float>(m.u), static_cast<float>(m.v),
          static_cast<float>(m.e),   static_cast<float>(m.h), static_cast<float>(m.mx),
          static_cast<float>(m.my),  static_cast<float>(m.p)};
}

// The state U_bar + d along n: primitive values and the normal-flux change
// dFn = F(U_bar + d).n - F(U_bar).n, every term proportional to d.
struct Side32 {
  float rho, inv, u, v, p, un, dun, e, c, dfn[4];
};

// Smallest point density FP32 works with, as a fraction of the mean: the
// positivity limiter keeps point values above its floors in FP64, but near
// vacuum mean + perturbation can round to zero or below in FP32; there the
// density used for velocities and sound speed is clamped to this fraction of
// the mean (and the pressure to zero), which changes nothing elsewhere.
constexpr float kVacuumFraction = 1e-6f;

// The reciprocal of the perturbation formulas: correctly rounded (the tile
// kernels, whose launch shapes agree bit for bit), or the one-instruction
// approximation of the SFU, within one unit in the last place (FAST: the
// patch kernel; FP32 carries only perturbations there).
template <bool FAST> __device__ __forceinline__ float perturbation_rcp(float x) {
  if constexpr (FAST) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else {
    return __frcp_rn(x);
  }
}

template <bool FAST = false>
__device__ __forceinline__ Side32 perturbed_side(const Ref32 &b, const float *d, float g1,
                                                 float gamma, float nx, float ny) {
  Side32 s;
  s.rho = fmaxf(b.rho + d[0], kVacuumFraction * b.rho);
  s.inv = perturbation_rcp<FAST>(s.rho);
  const float du = (d[1] - b.u * d[0]) * s.inv;
  const float dv = (d[2] - b.v * d[0]) * s.inv;
  s.u = b.u + du;
  s.v = b.v + dv;
  const float dmu = b.mx * du + d[1] * s.u + b.my * dv + d[2] * s.v;
  const float dp = g1 * (d[3] - 0.5f * dmu);
  s.p = b.p + dp;
  s.e = b.e + d[3];
  s.dun = du * nx + dv * ny;
  s.un = s.u * nx + s.v * ny;
  s.c = sqrtf(fmaxf(gamma * s.p * s.inv, 0.0f));
  s.dfn[0] = d[1] * nx + d[2] * ny;
  s.dfn[1] = b.mx * s.dun + d[1] * s.un + dp * nx;
  s.dfn[2] = b.my * s.dun + d[2] * s.un + dp * ny;
  s.dfn[3] = b.h * s.dun + (d[3] + dp) * s.un;
  return s;
}

// HLLC(U_bar + dl, U_bar + dr).n - F(U_bar).n in perturbation form: the wave
// speeds and branch are those of the HLLC flux (cpp/include/wasl/flux/hllc.hpp:40-74);
// the star-state jumps are rewritten so that no O(1) terms cancel:
//   S* - u_L = (dp - rho_R (S_R - u_R) du_n) / D,
//   rho* - rho_K = rho_K (S* - u_K) / (S_K - S*).
template <bool FAST = false>
__device__ __forceinline__ void hllc_perturbed(const Ref32 &b, const float *dl, const float *dr,
                                               float g1, float gamma, float nx, float ny,
                                               float *f) {
  const Side32 L = perturbed_side<FAST>(b, dl, g1, gamma, nx, ny);
  const Side32 R = perturbed_side<FAST>(b, dr, g1, gamma, nx, ny);
  const float sl = fminf(L.un - L.c, R.un - R.c);
  const float sr = fmaxf(L.un + L.c, R.un + R.c);
  // The star states are evaluated unconditionally and the supersonic cases
  // selected afterwards, so a warp never diverges on the flow regime.
  const float dpress = (R.p - b.p) - (L.p - b.p);
  const float dn = R.dun - L.dun;
  // den <= 0 always (sl <= u_L - c_L, sr >= u_R + c_R); it is zero only when
  // both sound speeds vanish, which FP32 rounding can produce near vacuum.
  const float den = fminf(L.rho * (sl - L.un) - R.rho * (sr - R.un), -1e-30f);
  const float sigma_l = (dpress - R.rho * (sr - R.un) * dn) / den; // S* - u_L
  const float star = L.un + sigma_l;
  const bool left = star >= 0.0f;
  const float krho = left ? L.rho : R.rho, ku = left ? L.u : R.u, kv = left ? L.v : R.v;
  const float ke = left ? L.e : R.e, kinv = left ? L.inv : R.inv, kp = left ? L.p : R.p;
  const float kun = left ? L.un : R.un;
  const float wave = left ? sl : sr;
  const float sigma = left ? sigma_l : sigma_l - dn; // S* - u_K
  // S_K - S* and S_K - u_K keep their sign (negative on the left, positive
  // on the right) and stay off zero in the FP32 near-vacuum corner case.
  const float wave_gap = left ? fminf(wave - star, -1e-30f) : fmaxf(wave - star, 1e-30f);
  const float kun_gap = left ? fminf(wave - kun, -1e-30f) : fmaxf(wave - kun, 1e-30f);
  const float drho = krho * sigma / wave_gap;
  const float rho_star = krho + drho;
  const float t = rho_star * sigma;
  const float jump[4] = {drho, drho * ku + t * nx, drho * kv + t * ny,
                         drho * ke * kinv + t * (star + kp / (krho * kun_gap))};
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const float starf = (left ? L.dfn[v] : R.dfn[v]) + wave * jump[v];
    f[v] = sl >= 0.0f ? L.dfn[v] : (sr <= 0.0f ? R.dfn[v] : starf);
  }
}

// FP64 mode-0 values of periodic boundary faces, one thread per boundary face:
// value[v][b] = sum_q w_q HLLC(U_own, U_donor).n at the face's edge points,
// from FP64 traces.  The partner face across the period is evaluated the same
// way by its own element, so the two contributions cancel to FP64 round-off
// as in the plain path.
template <int P> __global__ void boundary_mode0(const StageArgs a) {
  using S = TriShape<P>;
  constexpr int M = S::M, QF = S::QF;
  const std::int64_t b = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= a.boundary.count)
    return;
  const std::int64_t ne = a.mesh.ne;
  const std::int64_t e = a.boundary.element[b];
  const int le = a.boundary.local_edge[b];
  const double nx = a.boundary.normal[b], ny = a.boundary.normal[a.boundary.count + b];
  const FaceTable<P, double> *F = static_cast<const FaceTable<P, double> *>(a.face_table64);
  const double *__restrict__ in = a.in;
  double sum[4] = {0.0, 0.0, 0.0, 0.0};
  for (int q = 0; q < QF; ++q) {
    const std::int64_t point = b * QF + q;
    const std::int64_t d = a.mesh.donor[point];
    const double *db = a.mesh.donor_basis + point * M;
    double us[4], ud[4], f[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double s = 0.0, o = 0.0;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        s += in[(static_cast<std::int64_t>(v) * M + m) * ne + d] * db[m];
        o += in[(static_cast<std::int64_t>(v) * M + m) * ne + e] * F->lb[le][q][m];
      }
      ud[v] = s;
      us[v] = o;
    }
    hllc_fast(a.gamma, us, ud, nx, ny, f);
#pragma unroll
    for (int v = 0; v < 4; ++v)
      sum[v] += F->ew[le][q] * f[v];
  }
#pragma unroll
  for (int v = 0; v < 4; ++v)
    a.boundary.value[v * a.boundary.count + b] = sum[v];
}

// Per-face record written by the face kernel and gathered by the element
// kernel: the HLLC perturbation at each edge point (around the left mean),
// the change of reference from the left to the right mean, and the full FP64
// face value that mode 0 takes (both sides read the same numbers).
template <int P> struct FaceRecord {
  float dflux[TriShape<P>::QF][4];
  float shift[4];
  double mode0[4];
};

template <int P>
__global__ void __launch_bounds__(128) euler_tri_faces_mixed(const StageArgs a) {
  using S = TriShape<P>;
  constexpr int M = S::M, QF = S::QF, H = M - 1;
  constexpr double phi0 = 0.70710678118654752440;
  // The edge tables, shared by the block.
  __shared__ FaceTable<P, float> table;
  {
    const float *src = static_cast<const float *>(a.face_table);
    float *dst = reinterpret_cast<float *>(&table);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(table) / sizeof(float)); i += blockDim.x)
      dst[i] = src[i];
  }
  __syncthreads();
  const std::int64_t nf = a.faces.count;
  const std::int64_t f = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= nf)
    return;
  const std::int64_t ne = a.mesh.ne;
  const double *__restrict__ in = a.in;
  const FaceTable<P, float> *F = &table;
  const double gamma = a.gamma;
  const float gamma32 = static_cast<float>(gamma), g1 = static_cast<float>(gamma - 1.0);
  const std::int32_t L = a.faces.left[f], R = a.faces.right[f];
  const unsigned code = a.faces.code[f];
  if (code & 0x80u) // the far copy of a paired periodic face: evaluated with its partner
    return;
  const int le = (code >> 1) & 3u, re = (code >> 3) & 3u, flip = (code >> 5) & 1u;
  const double nx = a.faces.normal[f], ny = a.faces.normal[nf + f];
  const float nxf = static_cast<float>(nx), nyf = static_cast<float>(ny);

  double lmean[4], rmean[4];
  float lh[4][H], rh[4][H];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    lmean[v] = __ldg(in + (static_cast<std::int64_t>(v) * M) * ne + L) * phi0;
#pragma unroll
    for (int m = 0; m < H; ++m)
      lh[v][m] = static_cast<float>(__ldg(in + (static_cast<std::int64_t>(v) * M + m + 1) * ne + L));
  }
  const bool interior = R >= 0;
  const bool paired = !interior && a.boundary.paired;
  if (paired) {
    const std::int64_t d = a.mesh.donor[static_cast<std::int64_t>(-R - 1) * QF];
#pragma unroll
    for (int v = 0; v < 4; ++v)
      rmean[v] = __ldg(in + (static_cast<std::int64_t>(v) * M) * ne + d) * phi0;
  }
  if (interior) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      rmean[v] = __ldg(in + (static_cast<std::int64_t>(v) * M) * ne + R) * phi0;
#pragma unroll
      for (int m = 0; m < H; ++m)
        rh[v][m] = static_cast<float>(__ldg(in + (static_cast<std::int64_t>(v) * M + m + 1) * ne + R));
    }
  }
  const MeanState ml = mean_state(gamma, lmean);
  const Ref32 ref = ref32(ml);
  double fln[4];
  mean_normal_flux(ml, nx, ny, fln);
  FaceRecord<P> rec;
  float jump[4];
  if (interior || paired) {
    const MeanState mr = mean_state(gamma, rmean);
    double frn[4];
    mean_normal_flux(mr, nx, ny, frn);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      jump[v] = interior ? static_cast<float>(rmean[v] - lmean[v]) : 0.0f;
      rec.shift[v] = static_cast<float>(fln[v] - frn[v]);
    }
  } else {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      jump[v] = 0.0f;
      rec.shift[v] = 0.0f;
    }
  }
  const float(*lb)[M] = F->lb[le];
  const float(*rb)[M] = F->rb[(le * 3 + re) * 2 + flip];
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int q = 0; q < QF; ++q) {
    float dl[4], dr[4], fl[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      float sl = 0.0f, sr = 0.0f;
#pragma unroll
      for (int m = 0; m < H; ++m) {
        sl = fmaf(lh[v][m], lb[q][m + 1], sl);
        if (interior)
          sr = fmaf(rh[v][m], rb[q][m + 1], sr);
      }
      dl[v] = sl;
      dr[v] = jump[v] + sr;
    }
    if (!interior) {
      if (a.mesh.boundary == 3) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          dr[v] = dl[v];
      } else {
        const std::int64_t point = static_cast<std::int64_t>(-R - 1) * QF + q;
        const std::int64_t d = a.mesh.donor[point];
        const double *db = a.mesh.donor_basis + point * M;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          double s = 0.0;
#pragma unroll
          for (int m = 0; m < M; ++m)
            s += __ldg(in + (static_cast<std::int64_t>(v) * M + m) * ne + d) * db[m];
          dr[v] = static_cast<float>(s - lmean[v]);
        }
      }
    }
    hllc_perturbed(ref, dl, dr, g1, gamma32, nxf, nyf, fl);
    const float w = F->ew[le][q];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      rec.dflux[q][v] = fl[v];
      acc[v] = fmaf(w, fl[v], acc[v]);
    }
  }
  const bool periodic_boundary = !interior && a.mesh.boundary != 3 && !paired;
#pragma unroll
  for (int v = 0; v < 4; ++v)
    rec.mode0[v] = periodic_boundary ? a.boundary.value[v * a.boundary.count + (-R - 1)]
                                     : fln[v] * c_edge_wsum<P>[le] + static_cast<double>(acc[v]);
  static_cast<FaceRecord<P> *>(a.faces.record)[f] = rec;
}

template <int P, int R>
__global__ void __launch_bounds__(128) euler_tri_elements_mixed(const StageArgs a) {
  using S = TriShape<P>;
  constexpr int M = S::M, QV = MixedVolume<P, R>::QV, QF = S::QF, H = M - 1;
  constexpr double phi0 = 0.70710678118654752440;
  const std::int64_t ne = a.mesh.ne;
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= ne)
    return;
  const double *__restrict__ in = a.in;
  const MixedVolume<P, R> &T = c_mix<P, R>;
  const FaceTable<P, float> *__restrict__ F = static_cast<const FaceTable<P, float> *>(a.face_table);
  const FaceRecord<P> *__restrict__ records = static_cast<const FaceRecord<P> *>(a.faces.record);
  const double gamma = a.gamma;
  const float g1 = static_cast<float>(gamma - 1.0);
  static_assert(sizeof(FaceRecord<P>) % 16 == 0, "face records are copied in 16-byte chunks");

  double mean[4];
  float ch[4][H];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    mean[v] = in[(static_cast<std::int64_t>(v) * M) * ne + e] * phi0;
#pragma unroll
    for (int m = 0; m < H; ++m)
      ch[v][m] = static_cast<float>(in[(static_cast<std::int64_t>(v) * M + m + 1) * ne + e]);
  }
  const double *__restrict__ geo = a.mesh.geo;
  const Ref32 bb = ref32(mean_state(gamma, mean));

  // Stage this element's three face records into shared memory now; the
  // copies complete while the volume term is computed.
  __shared__ __align__(16) FaceRecord<P> staged[3][128];
  std::int32_t staged_face[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    staged_face[k] = a.faces.slot_face[k * ne + e];
    const char *src = reinterpret_cast<const char *>(records + staged_face[k]);
    char *dst = reinterpret_cast<char *>(&staged[k][threadIdx.x]);
    const unsigned sdst = static_cast<unsigned>(__cvta_generic_to_shared(dst));
#pragma unroll
    for (int c = 0; c < static_cast<int>(sizeof(FaceRecord<P>)) / 16; ++c)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sdst + 16 * c),
                   "l"(src + 16 * c)
                   : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");

  // Volume term of the high modes: the element's own mean flux cancels
  // against its faces (divergence theorem, both rules exact), leaving the
  // perturbation flux dF.  The 1/2 of the scaled gradient is folded into w.
  float racc[4][H];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < H; ++m)
      racc[v][m] = 0.0f;
  {
    const float fax = static_cast<float>(geo[e]), fay = static_cast<float>(geo[ne + e]);
    const float fbx = static_cast<float>(geo[2 * ne + e]), fby = static_cast<float>(geo[3 * ne + e]);
#pragma unroll 5
    for (int q = 0; q < QV; ++q) {
      float d[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        float s = 0.0f;
#pragma unroll
        for (int m = 0; m < H; ++m)
          s = fmaf(ch[v][m], T.phi[q][m], s);
        d[v] = s;
      }
      const float inv = __frcp_rn(fmaxf(bb.rho + d[0], kVacuumFraction * bb.rho));
      const float du = (d[1] - bb.u * d[0]) * inv;
      const float dv = (d[2] - bb.v * d[0]) * inv;
      const float uu = bb.u + du, vv = bb.v + dv;
      const float dmu = bb.mx * du + d[1] * uu + bb.my * dv + d[2] * vv;
      const float dp = g1 * (d[3] - 0.5f * dmu);
      const float dep = d[3] + dp;
      const float fx[4] = {d[1], bb.mx * du + d[1] * uu + dp, bb.my * du + d[2] * uu,
                           bb.h * du + dep * uu};
      const float fy[4] = {d[2], bb.mx * dv + d[1] * vv, bb.my * dv + d[2] * vv + dp,
                           bb.h * dv + dep * vv};
      const float w = T.w[q];
      const float wby = w * fby, wbx = w * fbx, wax = w * fax, way = w * fay;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float gxi = wby * fx[v] - wbx * fy[v];
        const float geta = wax * fy[v] - way * fx[v];
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(T.dxi[q][m], gxi, fmaf(T.deta[q][m], geta, racc[v][m]));
      }
    }
  }

  // Gather the three faces, in ascending face index, from the staged records.
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  double r0[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const unsigned code = a.mesh.slot_code[k * ne + e];
    const double scale = a.mesh.slot_geo[(3 * k + 2) * ne + e];
    const bool self_left = code & 1u;
    const int le = (code >> 1) & 3u, re = (code >> 3) & 3u, flip = (code >> 5) & 1u;
    const float(*own)[M] = self_left ? F->lb[le] : F->rb[(le * 3 + re) * 2 + flip];
    if (code & 0x40u) // far side of a paired periodic face: the donor basis is this element's
      own = reinterpret_cast<const float(*)[M]>(
          a.boundary.basis32 + static_cast<std::int64_t>(-a.faces.right[staged_face[k]] - 1) * QF * M);
    const FaceRecord<P> &rec = staged[k][threadIdx.x];
    const float fscale = static_cast<float>(scale);
#pragma unroll
    for (int q = 0; q < QF; ++q) {
      const float w = F->ew[le][q];
      const float wsc = (self_left ? -w : w) * fscale;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float value = wsc * (self_left ? rec.dflux[q][v] : rec.dflux[q][v] + rec.shift[v]);
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(value, own[q][m + 1], racc[v][m]);
      }
    }
    const double sgn = self_left ? -1.0 : 1.0;
#pragma unroll
    for (int v = 0; v < 4; ++v)
      r0[v] += sgn * scale * phi0 * rec.mode0[v];
  }

  const double inv = geo[4 * ne + e];
  const double dt = a.dt ? *a.dt : a.dt_value;
  double rho[M];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const std::int64_t idx = (static_cast<std::int64_t>(v) * M + m) * ne + e;
      const double cur = in[idx];
      const double rr = (m == 0 ? r0[v] : static_cast<double>(racc[v][m > 0 ? m - 1 : 0])) * inv;
      double o;
      if (a.stage == 0)
        o = cur + dt * rr;
      else if (a.stage == 1)
        o = 0.75 * a.u0[idx] + 0.25 * (cur + dt * rr);
      else
        o = (1.0 / 3.0) * a.u0[idx] + (2.0 / 3.0) * (cur + dt * rr);
      a.out[idx] = o;
      if (v == 0)
        rho[m] = o;
    }

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

// FP32 trace of high modes h at one edge point: sum_m h[v][m] basis[m+1],
// with explicit fused multiply-adds so both sides of a face get the same bits.
template <int P>
__device__ __forceinline__ void high_trace(const float (&h)[4][TriShape<P>::M - 1],
                                           const float *basis, float *out) {
  constexpr int H = TriShape<P>::M - 1;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    float s = 0.0f;
#pragma unroll
    for (int m = 0; m < H; ++m)
      s = fmaf(h[v][m], basis[m + 1], s);
    out[v] = s;
  }
}

// Relative jump of density or energy between two cell means above which a
// face is evaluated in FP64: near discontinuities the perturbations are as
// large as the means and FP32 point states lose the positivity margins the
// limiter keeps in FP64.
constexpr double kFp64Jump = 0.05;

__device__ __forceinline__ bool mean_jump(double rho_a, double rho_b, double e_a, double e_b) {
  return fabs(rho_a - rho_b) > kFp64Jump * fmin(rho_a, rho_b) ||
         fabs(e_a - e_b) > kFp64Jump * fmin(e_a, e_b);
}

// One face in FP64 (the mixed form's islands): traces of both elements from
// their FP64 coefficients (rows stride apart) and the FP64 face tables, HLLC
// in FP64 (reference order of operations up to contraction), then the
// high-mode perturbations dflux[q][v] = F_q - F(U_L bar).n (FP32) and the
// full mode-0 value sum_q w_q F_q.  Both elements of a face call it with the
// same inputs in the same roles, so they get the same bits.
template <int P>
__device__ __noinline__ void face_fp64(double gamma, const double *own, std::int64_t own_stride,
                                       const double *other, std::int64_t other_stride,
                                       bool boundary, bool self_left, const double *own_basis,
                                       const double *other_basis, const double *weights,
                                       double nx, double ny, const double *fln,
                                       float (*dflux)[4], double *mode0) {
  constexpr int M = TriShape<P>::M, QF = TriShape<P>::QF;
#pragma unroll
  for (int v = 0; v < 4; ++v)
    mode0[v] = 0.0;
  for (int q = 0; q < QF; ++q) {
    double to[4], tn[4], ul[4], ur[4], f[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double so = 0.0, sn = 0.0;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        so = fma(own[(v * M + m) * own_stride], own_basis[q * M + m], so);
        if (!boundary)
          sn = fma(other[(v * M + m) * other_stride], other_basis[q * M + m], sn);
      }
      to[v] = so;
      tn[v] = sn;
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      ul[v] = boundary || self_left ? to[v] : tn[v];
      ur[v] = boundary ? to[v] : (self_left ? tn[v] : to[v]);
    }
    hllc_fast(gamma, ul, ur, nx, ny, f);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      dflux[q][v] = static_cast<float>(f[v] - fln[v]);
      mode0[v] = fma(weights[q], f[v], mode0[v]);
    }
  }
}


// The end of a tile kernel's stage for element e (thread t of the tile):
// residual scaling by 1/det J, the Shu-Osher combination in FP64
// (cpp/include/wasl/time/ssp_rk3.hpp:44-60), and, when asked for, the next
// step's CFL speed and the modal-decay sensor on the result.
template <int P, int TILE>
__device__ __forceinline__ void tile_finish(const StageArgs &a, std::int64_t e, int t, int case_id,
                                            const double (*sstate)[TILE], const double (&r0)[4],
                                            const float (&racc)[4][TriShape<P>::M - 1]) {
  constexpr int M = TriShape<P>::M;
  const std::int64_t ne = a.mesh.ne;
  const double gamma = a.gamma;
  const double *__restrict__ geo = a.mesh.geo;
  const double inv = geo[4 * ne + e];
  const double dt = a.case_dt ? a.case_dt[case_id] : (a.dt ? *a.dt : a.dt_value);
  double rho[M], avg[4];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const std::int64_t idx = (static_cast<std::int64_t>(v) * M + m) * ne + e;
      const double cur = sstate[v * M + m][t];
      const double rr = (m == 0 ? r0[v] : static_cast<double>(racc[v][m > 0 ? m - 1 : 0])) * inv;
      double o;
      if (a.stage == 0)
        o = cur + dt * rr;
      else if (a.stage == 1)
        o = 0.75 * a.u0[idx] + 0.25 * (cur + dt * rr);
      else
        o = (1.0 / 3.0) * a.u0[idx] + (2.0 / 3.0) * (cur + dt * rr);
      a.out[idx] = o;
      if (v == 0)
        rho[m] = o;
      if (m == 0)
        avg[v] = o;
    }

  if (a.speed_max) {
    // The next step's CFL speed from this stage's cell averages.
    const double scale = 1.0 / sqrt(2.0);
    const double sa[4] = {__dmul_rn(scale, avg[0]), __dmul_rn(scale, avg[1]),
                          __dmul_rn(scale, avg[2]), __dmul_rn(scale, avg[3])};
    bool physical = true;
    const double speed = cfl_speed(gamma, sa, 2, physical);
    unsigned long long best = 0;
    if (physical)
      best = __double_as_longlong(speed);
    else
      raise_error(a.error, kNonPhysicalAverage, e);
    // Warp max over whichever lanes are still active (past the tile's end,
    // or handed to the rough pass, lanes have returned): the 64-bit max of
    // positive FP64 bits as the max of the high words, then of the low words
    // among the lanes holding it; one atomic per warp and case.
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    // (No lane's match set is the whole mask unless all lanes share the case,
    // so the branch is uniform across the warp.)
    if (__match_any_sync(mask, case_id) == mask) {
      const unsigned hi = __reduce_max_sync(mask, static_cast<unsigned>(best >> 32));
      const unsigned lo = __reduce_max_sync(
          mask, static_cast<unsigned>(best >> 32) == hi ? static_cast<unsigned>(best) : 0u);
      if (lane == __ffs(mask) - 1)
        atomicMax(a.speed_max + case_id, (static_cast<unsigned long long>(hi) << 32) | lo);
    } else {
      // Lanes of one warp from different cases (the rough pass of a batch).
      atomicMax(a.speed_max + case_id, best);
    }
  }

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
    const unsigned active_mask = __activemask();
    const unsigned ballot = __ballot_sync(active_mask, troubled);
    if (ballot) {
      const int lane = threadIdx.x & 31;
      const int leader = __ffs(ballot) - 1;
      int base = 0;
      if (lane == leader)
        base = atomicAdd(a.troubled_count, __popc(ballot));
      base = __shfl_sync(active_mask, base, leader);
      if (troubled)
        a.troubled[base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<std::int32_t>(e);
    }
  }
}

// The fused mixed stage on a tile of TILE consecutive elements per CTA.
// The tile's state is staged in shared memory (FP64 means, FP32 high modes)
// with asynchronous copies; each thread then computes its element's volume
// term and all three of its faces, reading a neighbour inside the tile from
// shared memory and one outside it from global memory (L2).  Each face is
// evaluated by both of its elements with the same instructions on the same
// inputs (the HLLC perturbation is always taken around the face's left mean),
// so the two mode-0 contributions cancel exactly, as in the face-centric form.
// MINB: resident CTAs per SM the register budget is sized for (1: no cap).
//
// ROUGH = false: the FP32 pass.  An element with a face across which the two
// cell means jump (kFp64Jump; a test both elements of the face make alike) is
// not computed here but appended to the rough list (when a.rough is set).
// ROUGH = true: the elements of the rough list (one per thread, neighbours
// read from global memory); faces with a jump are evaluated in FP64
// (face_fp64), the others with the same FP32 code as the FP32 pass, so both
// elements of every face still compute the same values.
// One element's share of the tile kernel's stage, once its tile is staged:
// volume term, the three faces, and the finish.  An element of the FP32 pass
// with a face across a jump of the means returns early (handed to the rough
// pass).  Shared by the one-tile-per-CTA and the persistent kernels.
template <int P, int R, int TILE, bool ROUGH>
__device__ __forceinline__ void tile_element(const StageArgs &a, const FaceTable<P, float> &table,
                                             const double (*sstate)[TILE], int t,
                                             std::int64_t e, std::int64_t first,
                                             std::int64_t count, int case_id) {
  using S = TriShape<P>;
  constexpr int M = S::M, QV = MixedVolume<P, R>::QV, QF = S::QF, H = M - 1;
  constexpr double phi0 = 0.70710678118654752440;
  const std::int64_t ne = a.mesh.ne;
  const double *__restrict__ in = a.in;
  double mean[4];
  float ch[4][H];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    mean[v] = sstate[v * M][t] * phi0;
#pragma unroll
    for (int m = 0; m < H; ++m)
      ch[v][m] = static_cast<float>(sstate[v * M + m + 1][t]);
  }

  const MixedVolume<P, R> &T = c_mix<P, R>;
  const double gamma = a.gamma;
  const float gamma32 = static_cast<float>(gamma), g1 = static_cast<float>(gamma - 1.0);
  const double *__restrict__ geo = a.mesh.geo;
  const MeanState own = mean_state(gamma, mean);
  const Ref32 bb = ref32(own);

  // Volume term of the high modes (perturbation flux, as in the element kernel).
  float racc[4][H];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < H; ++m)
      racc[v][m] = 0.0f;
  {
    const float fax = static_cast<float>(geo[e]), fay = static_cast<float>(geo[ne + e]);
    const float fbx = static_cast<float>(geo[2 * ne + e]), fby = static_cast<float>(geo[3 * ne + e]);
#pragma unroll 3
    for (int q = 0; q < QV; ++q) {
      float d[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        float s = 0.0f;
#pragma unroll
        for (int m = 0; m < H; ++m)
          s = fmaf(ch[v][m], T.phi[q][m], s);
        d[v] = s;
      }
      const float inv = __frcp_rn(fmaxf(bb.rho + d[0], kVacuumFraction * bb.rho));
      const float du = (d[1] - bb.u * d[0]) * inv;
      const float dv = (d[2] - bb.v * d[0]) * inv;
      const float uu = bb.u + du, vv = bb.v + dv;
      const float dmu = bb.mx * du + d[1] * uu + bb.my * dv + d[2] * vv;
      const float dp = g1 * (d[3] - 0.5f * dmu);
      const float dep = d[3] + dp;
      const float fx[4] = {d[1], bb.mx * du + d[1] * uu + dp, bb.my * du + d[2] * uu,
                           bb.h * du + dep * uu};
      const float fy[4] = {d[2], bb.mx * dv + d[1] * vv, bb.my * dv + d[2] * vv + dp,
                           bb.h * dv + dep * vv};
      const float w = T.w[q];
      const float wby = w * fby, wbx = w * fbx, wax = w * fax, way = w * fay;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float gxi = wby * fx[v] - wbx * fy[v];
        const float geta = wax * fy[v] - way * fx[v];
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(T.dxi[q][m], gxi, fmaf(T.deta[q][m], geta, racc[v][m]));
      }
    }
  }

  // The three faces, in the element's slot order.
  double r0[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const std::int64_t slot = k * ne + e;
    const unsigned code = a.tile.code[slot];
    const std::int32_t nb = a.tile.nbr[slot];
    const bool self_left = code & 1u;
    const int le = (code >> 1) & 3u, re = (code >> 3) & 3u, flip = (code >> 5) & 1u;
    const double nx = a.mesh.slot_geo[(3 * k) * ne + e];
    const double ny = a.mesh.slot_geo[(3 * k + 1) * ne + e];
    const double scale = a.mesh.slot_geo[(3 * k + 2) * ne + e];
    const float *lb = &table.lb[le][0][0];
    const float *rb = &table.rb[(le * 3 + re) * 2 + flip][0][0];
    const float *own_basis = self_left ? lb : rb;
    const float *other_basis = self_left ? rb : lb;
    if (code & 0xC0u) {
      const float *periodic = a.boundary.basis32 + static_cast<std::int64_t>(a.tile.aux[slot]) * QF * M;
      if (code & 0x40u)
        own_basis = periodic;
      else
        other_basis = periodic;
    }
    // The element across the face: its mean and high modes.
    double nmean[4] = {0.0, 0.0, 0.0, 0.0};
    float nh[4][H];
    const bool boundary = nb < 0;
    if (!boundary) {
      const std::int64_t local = nb - first;
      if (!ROUGH && local >= 0 && local < count) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          nmean[v] = sstate[v * M][local] * phi0;
#pragma unroll
          for (int m = 0; m < H; ++m)
            nh[v][m] = static_cast<float>(sstate[v * M + m + 1][local]);
        }
      } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double *row = in + static_cast<std::int64_t>(v) * M * ne + nb;
          nmean[v] = __ldg(row) * phi0;
#pragma unroll
          for (int m = 0; m < H; ++m)
            nh[v][m] = static_cast<float>(__ldg(row + (m + 1) * ne));
        }
      }
    }
    // FP32 pass: an element with a face across a jump of the means is left
    // to the rough pass (its work so far is dropped, nothing was written).
    if (!ROUGH && a.rough && !boundary && mean_jump(nmean[0], mean[0], nmean[3], mean[3])) {
      a.rough[atomicAdd(a.rough_count, 1)] = static_cast<std::int32_t>(e);
      return;
    }
    // The face's left state is the reference of the perturbation form.
    MeanState ml;
    if (self_left)
      ml = own;
    else
      ml = mean_state(gamma, nmean);
    const Ref32 ref = ref32(ml);
    double fln[4];
    mean_normal_flux(ml, nx, ny, fln);
    float jump[4], shift[4];
    if (boundary) {
#pragma unroll
      for (int v = 0; v < 4; ++v)
        jump[v] = shift[v] = 0.0f;
    } else {
#pragma unroll
      for (int v = 0; v < 4; ++v)
        jump[v] = static_cast<float>(self_left ? nmean[v] - mean[v] : mean[v] - nmean[v]);
      if (!self_left) {
        double frn[4];
        mean_normal_flux(own, nx, ny, frn);
#pragma unroll
        for (int v = 0; v < 4; ++v)
          shift[v] = static_cast<float>(fln[v] - frn[v]);
      }
    }
    const float nxf = static_cast<float>(nx), nyf = static_cast<float>(ny);
    const float fscale = static_cast<float>(scale);
    const double sgn = self_left ? -1.0 : 1.0;
    // Near a discontinuity (symmetric test on the two means): the face in FP64.
    if (ROUGH && !boundary && mean_jump(nmean[0], mean[0], nmean[3], mean[3])) {
      const FaceTable<P, double> *T64 = static_cast<const FaceTable<P, double> *>(a.face_table64);
      const double *lb64 = &T64->lb[le][0][0];
      const double *rb64 = &T64->rb[(le * 3 + re) * 2 + flip][0][0];
      const double *own64 = self_left ? lb64 : rb64;
      const double *other64 = self_left ? rb64 : lb64;
      if (code & 0xC0u) {
        const double *periodic =
            a.mesh.donor_basis + static_cast<std::int64_t>(a.tile.aux[slot]) * QF * M;
        if (code & 0x40u)
          own64 = periodic;
        else
          other64 = periodic;
      }
      float dq[QF][4];
      double m0[4];
      face_fp64<P>(gamma, &sstate[0][t], TILE, in + nb, ne, false, self_left, own64, other64,
                   &T64->ew[le][0], nx, ny, fln, dq, m0);
#pragma unroll
      for (int q = 0; q < QF; ++q) {
        const float w = table.ew[le][q];
        const float wsc = (self_left ? -w : w) * fscale;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const float value = wsc * (self_left ? dq[q][v] : dq[q][v] + shift[v]);
#pragma unroll
          for (int m = 0; m < H; ++m)
            racc[v][m] = fmaf(value, own_basis[q * M + m + 1], racc[v][m]);
        }
      }
#pragma unroll
      for (int v = 0; v < 4; ++v)
        r0[v] += sgn * scale * phi0 * m0[v];
      continue;
    }
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int q = 0; q < QF; ++q) {
      float to[4], tn[4], dl[4], dr[4], fl[4];
      high_trace<P>(ch, own_basis + q * M, to);
      if (boundary) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          dl[v] = dr[v] = to[v];
      } else {
        high_trace<P>(nh, other_basis + q * M, tn);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          dl[v] = self_left ? to[v] : tn[v];
          dr[v] = jump[v] + (self_left ? tn[v] : to[v]);
        }
      }
      hllc_perturbed(ref, dl, dr, g1, gamma32, nxf, nyf, fl);
      const float w = table.ew[le][q];
      const float wsc = (self_left ? -w : w) * fscale;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        acc[v] = fmaf(w, fl[v], acc[v]);
        const float value = wsc * (self_left ? fl[v] : fl[v] + shift[v]);
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(value, own_basis[q * M + m + 1], racc[v][m]);
      }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const double mode0 = fln[v] * c_edge_wsum<P>[le] + static_cast<double>(acc[v]);
      r0[v] += sgn * scale * phi0 * mode0;
    }
  }

  tile_finish<P, TILE>(a, e, t, case_id, sstate, r0, racc);
}

template <int P, int R, int TILE, int MINB, bool ROUGH>
__global__ void __launch_bounds__(TILE, MINB) euler_tri_tile_mixed(const StageArgs a) {
  using S = TriShape<P>;
  constexpr int M = S::M;
  __shared__ FaceTable<P, float> table;
  // The tile's FP64 state, row v M + m (dynamic shared memory, 4 M TILE doubles).
  extern __shared__ __align__(16) double tile_state[];
  double(*sstate)[TILE] = reinterpret_cast<double(*)[TILE]>(tile_state);

  const int t = threadIdx.x;
  const std::int64_t ne = a.mesh.ne;
  std::int64_t first = 0, count = 0, e = 0;
  int case_id = 0;
  bool active;
  if (ROUGH) {
    const std::int64_t list = *a.rough_count;
    if (static_cast<std::int64_t>(blockIdx.x) * TILE >= list)
      return; // the whole CTA is past the list (uniform: no barrier reached)
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * TILE + t;
    active = i < list;
    if (active) {
      e = a.rough[i];
      case_id = a.element_case ? a.element_case[e] : 0;
    }
  } else {
    if (a.work) {
      const TileWork w = a.work[blockIdx.x];
      first = w.first;
      count = w.count;
      case_id = w.case_id;
    } else {
      first = static_cast<std::int64_t>(blockIdx.x) * TILE;
      count = a.mesh.ne - first < TILE ? a.mesh.ne - first : TILE;
    }
    active = t < count;
    e = first + t;
  }
  const double *__restrict__ in = a.in;

  // Stage this tile's state (asynchronous 8-byte copies, coalesced per row)
  // and the face tables.
  if (active) {
    const unsigned base = static_cast<unsigned>(__cvta_generic_to_shared(&sstate[0][t]));
#pragma unroll
    for (int r = 0; r < 4 * M; ++r)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(base + r * TILE * 8),
                   "l"(in + r * ne + e)
                   : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  {
    const float *src = static_cast<const float *>(a.face_table);
    float *dst = reinterpret_cast<float *>(&table);
    for (int i = t; i < static_cast<int>(sizeof(table) / sizeof(float)); i += TILE)
      dst[i] = src[i];
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  if (!active)
    return;
  tile_element<P, R, TILE, ROUGH>(a, table, sstate, t, e, first, count, case_id);
}

// The FP32 pass of the tile kernel as a persistent kernel: each CTA loads the
// face tables once and then takes the work list's tiles (or the mesh's
// TILE-element tiles) gridDim.x apart, staging each one's state in turn; the
// per-element arithmetic is the tile kernel's, so the results are the same
// bit for bit.
template <int P, int R, int TILE, int MINB>
__global__ void __launch_bounds__(TILE, MINB) euler_tri_tile_persistent(const StageArgs a) {
  using S = TriShape<P>;
  constexpr int M = S::M;
  __shared__ FaceTable<P, float> table;
  extern __shared__ __align__(16) double tile_state[];
  double(*sstate)[TILE] = reinterpret_cast<double(*)[TILE]>(tile_state);
  const int t = threadIdx.x;
  const std::int64_t ne = a.mesh.ne;
  const double *__restrict__ in = a.in;
  {
    const float *src = static_cast<const float *>(a.face_table);
    float *dst = reinterpret_cast<float *>(&table);
    for (int i = t; i < static_cast<int>(sizeof(table) / sizeof(float)); i += TILE)
      dst[i] = src[i];
  }
  const std::int64_t tiles = a.work ? a.work_count : (ne + TILE - 1) / TILE;
  for (std::int64_t b = blockIdx.x; b < tiles; b += gridDim.x) {
    std::int64_t first, count;
    int case_id = 0;
    if (a.work) {
      const TileWork w = a.work[b];
      first = w.first;
      count = w.count;
      case_id = w.case_id;
    } else {
      first = b * TILE;
      count = ne - first < TILE ? ne - first : TILE;
    }
    const bool active = t < count;
    const std::int64_t e = first + t;
    if (active) {
      const unsigned base = static_cast<unsigned>(__cvta_generic_to_shared(&sstate[0][t]));
#pragma unroll
      for (int r = 0; r < 4 * M; ++r)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(base + r * TILE * 8),
                     "l"(in + r * ne + e)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads(); // the tile is staged (and, the first time, the tables)
    if (active)
      tile_element<P, R, TILE, false>(a, table, sstate, t, e, first, count, case_id);
    __syncthreads(); // every element is done with the tile before the next one lands
  }
}

// Dynamic shared memory of the shared-face tile kernel, in this order:
//   state  double [4 M][TILE]    the tile's FP64 state rows (as the tile kernel)
//   prim   double [4][TILE]      u, v, p, E + p of each element's cell average
//   flux   float  [4 QF][3 TILE] face records: the FP32 HLLC perturbation at
//                                each edge point (column = record)
//   items  uint16 [3 TILE]       faces to evaluate, element * 4 + slot
//   rec    int16  [3][TILE]      each slot's record; <= -2: -(2 + k' TILE + j),
//                                the record of slot k' of tile element j;
//                                -1: none (a rough element's unneeded face)
template <int P, int TILE> struct SharedFaceSmem {
  static constexpr int M = TriShape<P>::M, QF = TriShape<P>::QF;
  static constexpr std::size_t state = 0;
  static constexpr std::size_t prim = state + sizeof(double) * 4 * M * TILE;
  static constexpr std::size_t flux = prim + sizeof(double) * 4 * TILE;
  static constexpr std::size_t items = flux + sizeof(float) * 4 * QF * 3 * TILE;
  static constexpr std::size_t rec = items + sizeof(std::uint16_t) * 3 * TILE;
  static constexpr std::size_t bytes = rec + sizeof(std::int16_t) * 3 * TILE;
};

// The fused mixed stage with the faces inside a tile evaluated once.
//
// The arithmetic is that of euler_tri_tile_mixed<..., ROUGH = false> and the
// output is the same, bit for bit; what changes is who evaluates a face.  In
// that kernel every element evaluates its three faces, so a face between two
// elements evaluates its HLLC flux twice.  Here a face whose two elements are
// both in the tile (and not joined across the period) is evaluated once, for
// its left element; every other face is evaluated for the tile's element on
// it (a face between two tiles is still evaluated by both, identically).
// The faces to evaluate are collected in a list that all threads of the CTA
// share out evenly, each writing an FP32 record per face (the HLLC
// perturbation at the edge points) in shared memory; then each thread lifts
// its element's three records onto its modes, in slot order, and sums the
// records' weighted values (in the tile kernel's order) for mode 0, adding
// the FP64 mean terms itself.  The left mean state of a face is taken from
// shared memory when its element is in the tile.
// With a rough list (a.rough), the elements with a face across a jump of the
// cell means are appended to it and left to the second pass, as in the tile
// kernel; their faces are evaluated only where an element that stays needs
// them.
// Each element's geometry, slot and (stages 1 and 2) u^n rows are prefetched
// into L2 at the start, so the later loads that depend on one another (slot
// codes, then neighbours' slots; normals; geometry) do not each wait on DRAM
// when the state and mesh are not in L2 (1.5% faster per step in the
// vortex benchmark, which flushes L2 between steps).
template <int P, int R, int TILE, int MINB>
__global__ void __launch_bounds__(TILE, MINB) euler_tri_tile_shared(const StageArgs a) {
  using S = TriShape<P>;
  using L = SharedFaceSmem<P, TILE>;
  constexpr int M = S::M, QV = MixedVolume<P, R>::QV, QF = S::QF, H = M - 1;
  constexpr double phi0 = 0.70710678118654752440;
  static_assert(3 * TILE < 16384, "record indices are 16-bit");
  __shared__ FaceTable<P, float> table;
  __shared__ int item_count;
  extern __shared__ __align__(16) unsigned char smem[];
  double(*sstate)[TILE] = reinterpret_cast<double(*)[TILE]>(smem + L::state);
  double(*prim)[TILE] = reinterpret_cast<double(*)[TILE]>(smem + L::prim);
  float(*rflux)[3 * TILE] = reinterpret_cast<float(*)[3 * TILE]>(smem + L::flux);
  std::uint16_t *items = reinterpret_cast<std::uint16_t *>(smem + L::items);
  std::int16_t(*rec)[TILE] = reinterpret_cast<std::int16_t(*)[TILE]>(smem + L::rec);

  const int t = threadIdx.x;
  const std::int64_t ne = a.mesh.ne;
  std::int64_t first = 0, count = 0;
  int case_id = 0;
  if (a.work) {
    const TileWork w = a.work[blockIdx.x];
    first = w.first;
    count = w.count;
    case_id = w.case_id;
  } else {
    first = static_cast<std::int64_t>(blockIdx.x) * TILE;
    count = a.mesh.ne - first < TILE ? a.mesh.ne - first : TILE;
  }
  const bool active = t < count;
  const std::int64_t e = first + t;
  const double *__restrict__ in = a.in;
  const double gamma = a.gamma;

  if (active) {
#pragma unroll
    for (int r = 0; r < 5; ++r)
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(a.mesh.geo + r * ne + e));
#pragma unroll
    for (int r = 0; r < 9; ++r)
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(a.mesh.slot_geo + r * ne + e));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(a.tile.nbr + k * ne + e));
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(a.tile.code + k * ne + e));
    }
    if (a.stage > 0) {
#pragma unroll
      for (int r = 0; r < 4 * M; ++r)
        asm volatile("prefetch.global.L2 [%0];\n" ::"l"(a.u0 + r * ne + e));
    }
  }
  // Stage the tile's state and the face tables (as the tile kernel).
  if (active) {
    const unsigned base = static_cast<unsigned>(__cvta_generic_to_shared(&sstate[0][t]));
#pragma unroll
    for (int r = 0; r < 4 * M; ++r)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(base + r * TILE * 8),
                   "l"(in + r * ne + e)
                   : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  {
    const float *src = static_cast<const float *>(a.face_table);
    float *dst = reinterpret_cast<float *>(&table);
    for (int i = t; i < static_cast<int>(sizeof(table) / sizeof(float)); i += TILE)
      dst[i] = src[i];
  }
  if (t == 0)
    item_count = 0;
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();

  // Each element: its mean's primitive values, the rough test, and its
  // slots' records (an item to evaluate, or the left element's record).
  bool rough = false;
  if (active) {
    double mean[4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
      mean[v] = sstate[v * M][t] * phi0;
    const MeanState own = mean_state(gamma, mean);
    prim[0][t] = own.u;
    prim[1][t] = own.v;
    prim[2][t] = own.p;
    prim[3][t] = own.h;
    if (a.rough) {
#pragma unroll 1
      for (int k = 0; k < 3; ++k) {
        const std::int32_t nb = a.tile.nbr[k * ne + e];
        if (nb < 0)
          continue;
        const std::int64_t local = nb - first;
        double n0, n3;
        if (local >= 0 && local < count) {
          n0 = sstate[0][local] * phi0;
          n3 = sstate[3 * M][local] * phi0;
        } else {
          n0 = __ldg(in + nb) * phi0;
          n3 = __ldg(in + static_cast<std::int64_t>(3) * M * ne + nb) * phi0;
        }
        rough = rough || mean_jump(n0, mean[0], n3, mean[3]);
      }
    }
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
      const std::int64_t slot = k * ne + e;
      const unsigned code = a.tile.code[slot];
      const std::int32_t nb = a.tile.nbr[slot];
      const std::int64_t local = nb - first;
      const bool shared = nb >= 0 && local >= 0 && local < count && !(code & 0xC0u);
      int r = -1;
      if (shared && !(code & 1u)) {
        // The left element's slot for this face.
        for (int k2 = 0; k2 < 3; ++k2) {
          const std::int64_t s2 = k2 * ne + nb;
          const unsigned c2 = a.tile.code[s2];
          if (a.tile.nbr[s2] == e && (c2 & 1u) && !(c2 & 0xC0u))
            r = -(2 + k2 * TILE + static_cast<int>(local));
        }
      }
      if (r == -1 && (shared || !rough)) {
        // A jump face is evaluated by neither element (both are rough); a
        // rough element's other faces only when the element across stays.
        bool jump_face = false;
        if (rough && nb >= 0) {
          double n0, n3;
          if (local >= 0 && local < count) {
            n0 = sstate[0][local] * phi0;
            n3 = sstate[3 * M][local] * phi0;
          } else {
            n0 = __ldg(in + nb) * phi0;
            n3 = __ldg(in + static_cast<std::int64_t>(3) * M * ne + nb) * phi0;
          }
          jump_face = mean_jump(n0, mean[0], n3, mean[3]);
        }
        if (!jump_face) {
          r = atomicAdd(&item_count, 1);
          items[r] = static_cast<std::uint16_t>(t * 4 + k);
        }
      }
      rec[k][t] = static_cast<std::int16_t>(r);
    }
  }
  __syncthreads();

  // Evaluate the listed faces, shared out over all threads: whole faces in
  // full rounds of TILE, then the remaining faces split into one unit per
  // edge point, so no thread is left with a whole extra face while the
  // others wait at the barrier.
  {
    const float gamma32 = static_cast<float>(gamma), g1 = static_cast<float>(gamma - 1.0);
    const int n = item_count;
    // Points [q0, q0 + NQ) of face item i (NQ = QF or 1).
    auto evaluate = [&](int i, int q0, auto whole) {
      constexpr int NQ = decltype(whole)::value ? QF : 1;
      const int te = items[i] >> 2, k = items[i] & 3;
      const std::int64_t ee = first + te, slot = k * ne + ee;
      const unsigned code = a.tile.code[slot];
      const std::int32_t nb = a.tile.nbr[slot];
      const bool self_left = code & 1u;
      const int le = (code >> 1) & 3u, re = (code >> 3) & 3u, flip = (code >> 5) & 1u;
      const double nx = a.mesh.slot_geo[(3 * k) * ne + ee];
      const double ny = a.mesh.slot_geo[(3 * k + 1) * ne + ee];
      const float *lb = &table.lb[le][0][0];
      const float *rb = &table.rb[(le * 3 + re) * 2 + flip][0][0];
      const float *own_basis = self_left ? lb : rb;
      const float *other_basis = self_left ? rb : lb;
      if (code & 0xC0u) {
        const float *periodic =
            a.boundary.basis32 + static_cast<std::int64_t>(a.tile.aux[slot]) * QF * M;
        if (code & 0x40u)
          own_basis = periodic;
        else
          other_basis = periodic;
      }
      double mean[4];
      float ch[4][H];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        mean[v] = sstate[v * M][te] * phi0;
#pragma unroll
        for (int m = 0; m < H; ++m)
          ch[v][m] = static_cast<float>(sstate[v * M + m + 1][te]);
      }
      double nmean[4] = {0.0, 0.0, 0.0, 0.0};
      float nh[4][H];
      const bool boundary = nb < 0;
      const std::int64_t local = nb - first;
      const bool near = !boundary && local >= 0 && local < count;
      if (near) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          nmean[v] = sstate[v * M][local] * phi0;
#pragma unroll
          for (int m = 0; m < H; ++m)
            nh[v][m] = static_cast<float>(sstate[v * M + m + 1][local]);
        }
      } else if (!boundary) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double *row = in + static_cast<std::int64_t>(v) * M * ne + nb;
          nmean[v] = __ldg(row) * phi0;
#pragma unroll
          for (int m = 0; m < H; ++m)
            nh[v][m] = static_cast<float>(__ldg(row + (m + 1) * ne));
        }
      }
      // The face's left mean state: the reference of the perturbation form.
      MeanState ml;
      const bool own_left = self_left || boundary;
      const int li = own_left ? te : static_cast<int>(local);
      if (own_left || near) {
        ml.rho = own_left ? mean[0] : nmean[0];
        ml.mx = own_left ? mean[1] : nmean[1];
        ml.my = own_left ? mean[2] : nmean[2];
        ml.e = own_left ? mean[3] : nmean[3];
        ml.u = prim[0][li];
        ml.v = prim[1][li];
        ml.p = prim[2][li];
        ml.h = prim[3][li];
      } else {
        ml = mean_state(gamma, nmean);
      }
      const Ref32 ref = ref32(ml);
      float jump[4];
#pragma unroll
      for (int v = 0; v < 4; ++v)
        jump[v] = boundary ? 0.0f
                           : static_cast<float>(self_left ? nmean[v] - mean[v] : mean[v] - nmean[v]);
      const float nxf = static_cast<float>(nx), nyf = static_cast<float>(ny);
#pragma unroll
      for (int j = 0; j < NQ; ++j) {
        const int q = q0 + j;
        float to[4], tn[4], dl[4], dr[4], fl[4];
        high_trace<P>(ch, own_basis + q * M, to);
        if (boundary) {
#pragma unroll
          for (int v = 0; v < 4; ++v)
            dl[v] = dr[v] = to[v];
        } else {
          high_trace<P>(nh, other_basis + q * M, tn);
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            dl[v] = self_left ? to[v] : tn[v];
            dr[v] = jump[v] + (self_left ? tn[v] : to[v]);
          }
        }
        hllc_perturbed(ref, dl, dr, g1, gamma32, nxf, nyf, fl);
#pragma unroll
        for (int v = 0; v < 4; ++v)
          rflux[q * 4 + v][i] = fl[v];
      }
    };
    const int whole = n / TILE * TILE;
#pragma unroll 1
    for (int i = t; i < whole; i += TILE)
      evaluate(i, 0, std::true_type{});
#pragma unroll 1
    for (int u = t; u < (n - whole) * QF; u += TILE)
      evaluate(whole + u / QF, u % QF, std::false_type{});
  }
  __syncthreads();
  if (!active)
    return;
  if (rough) {
    a.rough[atomicAdd(a.rough_count, 1)] = static_cast<std::int32_t>(e);
    return;
  }

  double mean[4];
  float ch[4][H];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    mean[v] = sstate[v * M][t] * phi0;
#pragma unroll
    for (int m = 0; m < H; ++m)
      ch[v][m] = static_cast<float>(sstate[v * M + m + 1][t]);
  }
  MeanState own;
  own.rho = mean[0];
  own.mx = mean[1];
  own.my = mean[2];
  own.e = mean[3];
  own.u = prim[0][t];
  own.v = prim[1][t];
  own.p = prim[2][t];
  own.h = prim[3][t];

  const MixedVolume<P, R> &T = c_mix<P, R>;
  const float g1 = static_cast<float>(gamma - 1.0);
  const double *__restrict__ geo = a.mesh.geo;
  const Ref32 bb = ref32(own);

  // Volume term of the high modes (as the tile kernel, fully unrolled).
  float racc[4][H];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < H; ++m)
      racc[v][m] = 0.0f;
  {
    const float fax = static_cast<float>(geo[e]), fay = static_cast<float>(geo[ne + e]);
    const float fbx = static_cast<float>(geo[2 * ne + e]), fby = static_cast<float>(geo[3 * ne + e]);
#pragma unroll
    for (int q = 0; q < QV; ++q) {
      float d[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        float s = 0.0f;
#pragma unroll
        for (int m = 0; m < H; ++m)
          s = fmaf(ch[v][m], T.phi[q][m], s);
        d[v] = s;
      }
      const float inv = __frcp_rn(fmaxf(bb.rho + d[0], kVacuumFraction * bb.rho));
      const float du = (d[1] - bb.u * d[0]) * inv;
      const float dv = (d[2] - bb.v * d[0]) * inv;
      const float uu = bb.u + du, vv = bb.v + dv;
      const float dmu = bb.mx * du + d[1] * uu + bb.my * dv + d[2] * vv;
      const float dp = g1 * (d[3] - 0.5f * dmu);
      const float dep = d[3] + dp;
      const float fx[4] = {d[1], bb.mx * du + d[1] * uu + dp, bb.my * du + d[2] * uu,
                           bb.h * du + dep * uu};
      const float fy[4] = {d[2], bb.mx * dv + d[1] * vv, bb.my * dv + d[2] * vv + dp,
                           bb.h * dv + dep * vv};
      const float w = T.w[q];
      const float wby = w * fby, wbx = w * fbx, wax = w * fax, way = w * fay;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float gxi = wby * fx[v] - wbx * fy[v];
        const float geta = wax * fy[v] - way * fx[v];
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(T.dxi[q][m], gxi, fmaf(T.deta[q][m], geta, racc[v][m]));
      }
    }
  }

  // Lift the three faces' records, in the element's slot order.
  double r0[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const std::int64_t slot = k * ne + e;
    const unsigned code = a.tile.code[slot];
    const std::int32_t nb = a.tile.nbr[slot];
    const bool self_left = code & 1u;
    const int le = (code >> 1) & 3u, re = (code >> 3) & 3u, flip = (code >> 5) & 1u;
    const double nx = a.mesh.slot_geo[(3 * k) * ne + e];
    const double ny = a.mesh.slot_geo[(3 * k + 1) * ne + e];
    const double scale = a.mesh.slot_geo[(3 * k + 2) * ne + e];
    const float *lb = &table.lb[le][0][0];
    const float *rb = &table.rb[(le * 3 + re) * 2 + flip][0][0];
    const float *own_basis = self_left ? lb : rb;
    if (code & 0x40u)
      own_basis = a.boundary.basis32 + static_cast<std::int64_t>(a.tile.aux[slot]) * QF * M;
    int r = rec[k][t];
    if (r < 0) {
      const int j = -r - 2;
      r = rec[j / TILE][j % TILE];
    }
    const bool boundary = nb < 0;
    MeanState ml;
    if (self_left) {
      ml = own;
    } else {
      const std::int64_t local = nb - first;
      if (local >= 0 && local < count) {
        ml.rho = sstate[0][local] * phi0;
        ml.mx = sstate[M][local] * phi0;
        ml.my = sstate[2 * M][local] * phi0;
        ml.e = sstate[3 * M][local] * phi0;
        ml.u = prim[0][local];
        ml.v = prim[1][local];
        ml.p = prim[2][local];
        ml.h = prim[3][local];
      } else {
        double nmean[4];
#pragma unroll
        for (int v = 0; v < 4; ++v)
          nmean[v] = __ldg(in + static_cast<std::int64_t>(v) * M * ne + nb) * phi0;
        ml = mean_state(gamma, nmean);
      }
    }
    double fln[4];
    mean_normal_flux(ml, nx, ny, fln);
    float shift[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (!boundary && !self_left) {
      double frn[4];
      mean_normal_flux(own, nx, ny, frn);
#pragma unroll
      for (int v = 0; v < 4; ++v)
        shift[v] = static_cast<float>(fln[v] - frn[v]);
    }
    const float fscale = static_cast<float>(scale);
    const double sgn = self_left ? -1.0 : 1.0;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int q = 0; q < QF; ++q) {
      const float w = table.ew[le][q];
      const float wsc = (self_left ? -w : w) * fscale;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float fl = rflux[q * 4 + v][r];
        acc[v] = fmaf(w, fl, acc[v]);
        const float value = wsc * (self_left ? fl : fl + shift[v]);
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(value, own_basis[q * M + m + 1], racc[v][m]);
      }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const double mode0 = fln[v] * c_edge_wsum<P>[le] + static_cast<double>(acc[v]);
      r0[v] += sgn * scale * phi0 * mode0;
    }
  }

  tile_finish<P, TILE>(a, e, t, case_id, sstate, r0, racc);
}

// ---- patch kernel ------------------------------------------------------------
//
// The mixed stage over a patch of TILE consecutive elements per CTA, each
// face evaluated once per patch, with every element's traces computed once.
// On a mesh whose element order keeps neighbours close (the solvers order
// elements along a space-filling curve), most faces lie inside a patch.
//
//   A. Each thread loads its element's state: the FP64 mean and its primitive
//      values, and the high modes in FP32 (shared memory), and evaluates the
//      high-mode traces at the Gauss points of its three local edges
//      (c_patch: that edge's points in its own order).  It lists the faces
//      it evaluates: a face inside the patch by its left element, a face to an
//      element outside the patch (or on a transmissive boundary) by this
//      element, so such a face is evaluated by both patches, identically.
//   B. All threads share out the listed faces (whole faces in full rounds,
//      the rest one edge point per thread): the HLLC flux perturbation around
//      the face's left mean, from the two traces (an outside neighbour's from
//      its coefficients in global memory, with the same instructions its own
//      patch uses), written over the evaluating element's trace in its own
//      point order.
//   C. Each thread computes its element's volume term (as the tile kernel),
//      lifts the flux records of its three edges (from its own record or from
//      its left neighbour's inside the patch) in the face's point order, and
//      forms mode 0 from the left mean's FP64 normal flux and the FP32
//      record sum, in the same order on both sides of the face; then the FP64
//      Shu-Osher combination.
//
// Both elements of a face apply the same mode-0 value bit for bit, so mass,
// momentum and energy are conserved to FP64 round-off, as in the tile kernel.
template <int P> struct PatchEdge {
  static constexpr int M = TriShape<P>::M, QF = TriShape<P>::QF, H = M - 1;
  float phi[3][QF][H]; // modes 1..M-1 at local edge j's points, in its order
  float w[3][QF];      // reference edge weights
};
template <int P> __constant__ PatchEdge<P> c_patch;

// ---- the volume term on the tensor cores (patch kernel, MMA variant) ---------
//
// Per warp, for its 32 elements (two 16-row tiles), the two contractions of
// the volume term run as TF32 tensor-core products with FP32 accumulation:
//   evaluation  d[e][v][q] = sum_m hi[e][v][m] phi[q][m]           (16 x K1 x 8)
//   projection  r[e][v][m] = sum_q dxi[q][m] Gxi[e][v][q] + deta[q][m] Geta[e][v][q]
// each operand split into a TF32 high part and the TF32 remainder
// (a b ~ ahi bhi + alo bhi + ahi blo), which keeps the products at about
// FP32 accuracy.  The pointwise perturbation flux between the two runs on
// the FP32 pipe in the evaluation's accumulator layout, and the projection
// takes its operands straight from those registers: its K index runs over
// the points in the order (2c, 2c+1) of the accumulator's columns, with the
// projection table permuted to match.  The results go through shared memory
// (over the element's high modes, no longer needed) to each element's thread.
template <int P, int R> struct VolumeMmaShape {
  static constexpr int H = TriShape<P>::M - 1, QV = MixedVolume<P, R>::QV;
  static constexpr int KS1 = (H + 7) / 8;  // evaluation k-steps (modes)
  static constexpr int NB = (QV + 7) / 8;  // point blocks
  static constexpr int KS2 = 2 * NB;       // projection k-steps (direction, point block)
  static constexpr int MB = (H + 7) / 8;   // projection mode blocks
  static constexpr int FRAGS = KS1 * NB + KS2 * MB; // float4 per lane
};

__device__ __forceinline__ unsigned tf32_of(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x as a TF32 high part and the TF32 rounding of the remainder.
__device__ __forceinline__ void tf32_split(float x, unsigned &hi, unsigned &lo) {
  hi = tf32_of(x);
  lo = tf32_of(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 "
               "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// d += A B with both split: alo bhi, ahi blo, then ahi bhi.
__device__ __forceinline__ void mma_tf32x3(float (&d)[4], const unsigned (&ahi)[4],
                                           const unsigned (&alo)[4], const float4 &b) {
  mma_tf32(d, alo, __float_as_uint(b.x), __float_as_uint(b.y));
  mma_tf32(d, ahi, __float_as_uint(b.z), __float_as_uint(b.w));
  mma_tf32(d, ahi, __float_as_uint(b.x), __float_as_uint(b.y));
}

// The B fragments of both products for every lane, split into TF32 high
// parts (x, y) and remainders (z, w): [KS1][NB] evaluation blocks, then
// [KS2][MB] projection blocks, 32 lanes each.  For lane (g = lane / 4,
// c = lane % 4) a block holds B[c][g] and B[c + 4][g].
template <int P, int R> __device__ void fill_volume_fragments(float4 *frag, int t, int threads) {
  using V = VolumeMmaShape<P, R>;
  const MixedVolume<P, R> &T = c_mix<P, R>;
  for (int i = t; i < V::FRAGS * 32; i += threads) {
    const int block = i / 32, lane = i % 32, g = lane / 4, c = lane % 4;
    float b[2];
    if (block < V::KS1 * V::NB) {
      const int ks = block / V::NB, nb = block % V::NB;
      const int q = nb * 8 + g;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = ks * 8 + c + 4 * h;
        b[h] = q < V::QV && m < V::H ? T.phi[q][m] : 0.0f;
      }
    } else {
      const int j = block - V::KS1 * V::NB, ks = j / V::MB, mb = j % V::MB;
      const int dir = ks / V::NB, nb = ks % V::NB, m = mb * 8 + g;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = c + 4 * h;
        const int q = nb * 8 + (k < 4 ? 2 * k : 2 * (k - 4) + 1);
        b[h] = q < V::QV && m < V::H ? (dir == 0 ? T.dxi[q][m] : T.deta[q][m]) : 0.0f;
      }
    }
    unsigned h0, l0, h1, l1;
    tf32_split(b[0], h0, l0);
    tf32_split(b[1], h1, l1);
    frag[i] = make_float4(__uint_as_float(h0), __uint_as_float(h1), __uint_as_float(l0),
                          __uint_as_float(l1));
  }
}

// The warp's volume term: hi modes in shi[4 H][TILE] (FP32), each element's
// FP32 mean state in sbb[8][TILE] (rho, u, v, E, E + p, rho u, rho v, p) and
// map columns in sgeo[4][TILE]; the results replace the warp's columns of shi
// (racc[v][m] at row v H + m).  All 32 lanes of the warp must call it.
template <int P, int R, int TILE>
__device__ __forceinline__ void patch_volume_mma(float (*shi)[TILE], const float (*sbb)[TILE],
                                                 const float (*sgeo)[TILE], const float4 *frag,
                                                 float g1, int warp_base, int lane) {
  using V = VolumeMmaShape<P, R>;
  constexpr int H = V::H;
  const MixedVolume<P, R> &T = c_mix<P, R>;
  const int g = lane >> 2, c = lane & 3;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = warp_base + mt * 16 + g, r1 = r0 + 8;
    // Evaluation: d[v][nb] holds (r0, 2c), (r0, 2c + 1), (r1, 2c), (r1, 2c + 1).
    float d[4][V::NB][4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
#pragma unroll
      for (int nb = 0; nb < V::NB; ++nb)
#pragma unroll
        for (int k = 0; k < 4; ++k)
          d[v][nb][k] = 0.0f;
#pragma unroll
      for (int ks = 0; ks < V::KS1; ++ks) {
        const int m0 = ks * 8 + c, m1 = m0 + 4;
        const float x[4] = {m0 < H ? shi[v * H + m0][r0] : 0.0f, m0 < H ? shi[v * H + m0][r1] : 0.0f,
                            m1 < H ? shi[v * H + m1][r0] : 0.0f, m1 < H ? shi[v * H + m1][r1] : 0.0f};
        unsigned ahi[4], alo[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
          tf32_split(x[k], ahi[k], alo[k]);
#pragma unroll
        for (int nb = 0; nb < V::NB; ++nb)
          mma_tf32x3(d[v][nb], ahi, alo, frag[(ks * V::NB + nb) * 32 + lane]);
      }
    }
    // Pointwise perturbation flux in the contravariant form, as the FP32 pass.
    Ref32 bb[2];
    float geo[2][4];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int r = s ? r1 : r0;
      bb[s] = {sbb[0][r], sbb[1][r], sbb[2][r], sbb[3][r],
               sbb[4][r], sbb[5][r], sbb[6][r], sbb[7][r]};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        geo[s][k] = sgeo[k][r];
    }
    __syncwarp(); // every lane has read its rows' hi modes (overwritten below)
    // The projection's A operands: G[v][direction][nb][slot], slots in the A
    // fragment's order (r0, 2c), (r1, 2c), (r0, 2c + 1), (r1, 2c + 1).
    float G[4][2][V::NB][4];
#pragma unroll
    for (int nb = 0; nb < V::NB; ++nb)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int s = k >> 1, q = nb * 8 + 2 * c + (k & 1);
        const Ref32 &b = bb[s];
        const float w = q < V::QV ? T.w[q] : 0.0f;
        const float dd[4] = {d[0][nb][k], d[1][nb][k], d[2][nb][k], d[3][nb][k]};
        const float inv = perturbation_rcp<true>(fmaxf(b.rho + dd[0], kVacuumFraction * b.rho));
        const float du = (dd[1] - b.u * dd[0]) * inv;
        const float dv = (dd[2] - b.v * dd[0]) * inv;
        const float uu = b.u + du, vv = b.v + dv;
        const float dmu = b.mx * du + dd[1] * uu + b.my * dv + dd[2] * vv;
        const float dp = g1 * (dd[3] - 0.5f * dmu);
        const float dep = dd[3] + dp;
        const float fx[4] = {dd[1], b.mx * du + dd[1] * uu + dp, b.my * du + dd[2] * uu,
                             b.h * du + dep * uu};
        const float fy[4] = {dd[2], b.mx * dv + dd[1] * vv, b.my * dv + dd[2] * vv + dp,
                             b.h * dv + dep * vv};
        const float wby = w * geo[s][3], wbx = w * geo[s][2], wax = w * geo[s][0],
                    way = w * geo[s][1];
        // Accumulator slot k = (row s, column 2c + (k & 1)) -> A slot (k & 1) * 2 + s.
        const int slot = (k & 1) * 2 + s;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          G[v][0][nb][slot] = wby * fx[v] - wbx * fy[v];
          G[v][1][nb][slot] = wax * fy[v] - way * fx[v];
        }
      }
    // Projection onto the high modes; results over the hi modes of the rows.
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      unsigned ghi[2][V::NB][4], glo[2][V::NB][4];
#pragma unroll
      for (int dir = 0; dir < 2; ++dir)
#pragma unroll
        for (int nb = 0; nb < V::NB; ++nb)
#pragma unroll
          for (int k = 0; k < 4; ++k)
            tf32_split(G[v][dir][nb][k], ghi[dir][nb][k], glo[dir][nb][k]);
#pragma unroll
      for (int mb = 0; mb < V::MB; ++mb) {
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int dir = 0; dir < 2; ++dir)
#pragma unroll
          for (int nb = 0; nb < V::NB; ++nb)
            mma_tf32x3(acc, ghi[dir][nb], glo[dir][nb],
                       frag[(V::KS1 * V::NB + (dir * V::NB + nb) * V::MB + mb) * 32 + lane]);
        const int m0 = mb * 8 + 2 * c, m1 = m0 + 1;
        if (m0 < H) {
          shi[v * H + m0][r0] = acc[0];
          shi[v * H + m0][r1] = acc[2];
        }
        if (m1 < H) {
          shi[v * H + m1][r0] = acc[1];
          shi[v * H + m1][r1] = acc[3];
        }
      }
    }
  }
  __syncwarp();
}

// Dynamic shared memory of the patch kernel, in this order:
//   mean  double [4][TILE]        cell means
//   prim  double [4][TILE]        u, v, p, E + p of each mean
//   hi    float  [4 H][TILE]      high modes, FP32
//   edge  float  [3 QF 4][TILE]   per (local edge, point, variable): the
//                                 element's trace, then the face's flux
//                                 perturbation (own point order)
//   items uint16 [3 TILE]         faces to evaluate: element * 4 + edge
//   and with the volume term on the tensor cores (MMA):
//   frag  float4 [FRAGS][32]      B fragments of its two products
//   bb    float  [8][TILE]        each mean state in FP32 (Ref32's fields)
//   geo   float  [4][TILE]        each element's map columns a_x, a_y, b_x, b_y
template <int P, int R, int TILE, bool MMA> struct PatchSmem {
  static constexpr int M = TriShape<P>::M, QF = TriShape<P>::QF, H = M - 1;
  static constexpr std::size_t mean = 0;
  static constexpr std::size_t prim = mean + sizeof(double) * 4 * TILE;
  static constexpr std::size_t hi = prim + sizeof(double) * 4 * TILE;
  static constexpr std::size_t edge = hi + sizeof(float) * 4 * H * TILE;
  static constexpr std::size_t frag = edge + sizeof(float) * 3 * QF * 4 * TILE;
  static constexpr std::size_t bb =
      frag + (MMA ? sizeof(float4) * 32 * VolumeMmaShape<P, R>::FRAGS : 0);
  static constexpr std::size_t geo = bb + (MMA ? sizeof(float) * 8 * TILE : 0);
  static constexpr std::size_t items = geo + (MMA ? sizeof(float) * 4 * TILE : 0);
  static constexpr std::size_t bytes = items + sizeof(std::uint16_t) * 3 * TILE;
};

// Asks the TMA engine to bring the 16-byte-aligned interior of [begin,
// begin + bytes) into L2 (one instruction per row; no data returns to the
// SM).  Only addresses inside the range are named.
__device__ __forceinline__ void prefetch_row_l2(const void *begin, std::size_t bytes) {
  const std::uintptr_t a = reinterpret_cast<std::uintptr_t>(begin);
  const std::uintptr_t lo = (a + 15) & ~static_cast<std::uintptr_t>(15);
  const std::uintptr_t hi = (a + bytes) & ~static_cast<std::uintptr_t>(15);
  if (hi > lo)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(lo),
                 "r"(static_cast<unsigned>(hi - lo))
                 : "memory");
}

template <int P, int TILE>
__device__ __forceinline__ MeanState patch_mean(const double (*smean)[TILE],
                                                const double (*sprim)[TILE], int i) {
  MeanState m;
  m.rho = smean[0][i];
  m.mx = smean[1][i];
  m.my = smean[2][i];
  m.e = smean[3][i];
  m.u = sprim[0][i];
  m.v = sprim[1][i];
  m.p = sprim[2][i];
  m.h = sprim[3][i];
  return m;
}

// The trace of element nb's high modes (FP64 in global memory) at point q of
// its local edge j: the instructions of phase A, so both patches agree.
template <int P>
__device__ __forceinline__ void patch_outside_trace(const double *__restrict__ in, std::int64_t ne,
                                                    std::int64_t nb, const float *phi, float *out) {
  constexpr int M = TriShape<P>::M, H = M - 1;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    float s = 0.0f;
#pragma unroll
    for (int m = 0; m < H; ++m)
      s = fmaf(static_cast<float>(__ldg(in + (static_cast<std::int64_t>(v) * M + m + 1) * ne + nb)),
               phi[m], s);
    out[v] = s;
  }
}

// The end of the patch kernel's stage for element e: residual scaling, the
// FP64 Shu-Osher combination (cpp/include/wasl/time/ssp_rk3.hpp:44-60) and the
// optional next-step CFL speed and sensor (as tile_finish, with the stage
// input read from global memory).
template <int P>
__device__ __forceinline__ void patch_finish(const StageArgs &a, std::int64_t e, int case_id,
                                             const double (&r0)[4],
                                             const float (&racc)[4][TriShape<P>::M - 1]) {
  constexpr int M = TriShape<P>::M;
  const std::int64_t ne = a.mesh.ne;
  const double inv = a.mesh.geo[4 * ne + e];
  const double dt = a.case_dt ? a.case_dt[case_id] : (a.dt ? *a.dt : a.dt_value);
  double rho[M], avg[4];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const std::int64_t idx = (static_cast<std::int64_t>(v) * M + m) * ne + e;
      const double cur = a.in[idx];
      const double rr = (m == 0 ? r0[v] : static_cast<double>(racc[v][m > 0 ? m - 1 : 0])) * inv;
      double o;
      if (a.stage == 0)
        o = cur + dt * rr;
      else if (a.stage == 1)
        o = 0.75 * a.u0[idx] + 0.25 * (cur + dt * rr);
      else
        o = (1.0 / 3.0) * a.u0[idx] + (2.0 / 3.0) * (cur + dt * rr);
      a.out[idx] = o;
      if (v == 0)
        rho[m] = o;
      if (m == 0)
        avg[v] = o;
    }
  if (a.speed_max) {
    const double scale = 1.0 / sqrt(2.0);
    const double sa[4] = {__dmul_rn(scale, avg[0]), __dmul_rn(scale, avg[1]),
                          __dmul_rn(scale, avg[2]), __dmul_rn(scale, avg[3])};
    bool physical = true;
    const double speed = cfl_speed(a.gamma, sa, 2, physical);
    unsigned long long best = 0;
    if (physical)
      best = __double_as_longlong(speed);
    else
      raise_error(a.error, kNonPhysicalAverage, e);
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    if (__match_any_sync(mask, case_id) == mask) {
      const unsigned hi = __reduce_max_sync(mask, static_cast<unsigned>(best >> 32));
      const unsigned lo = __reduce_max_sync(
          mask, static_cast<unsigned>(best >> 32) == hi ? static_cast<unsigned>(best) : 0u);
      if (lane == __ffs(mask) - 1)
        atomicMax(a.speed_max + case_id, (static_cast<unsigned long long>(hi) << 32) | lo);
    } else {
      atomicMax(a.speed_max + case_id, best);
    }
  }
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
    const unsigned active_mask = __activemask();
    const unsigned ballot = __ballot_sync(active_mask, troubled);
    if (ballot) {
      const int lane = threadIdx.x & 31;
      const int leader = __ffs(ballot) - 1;
      int base = 0;
      if (lane == leader)
        base = atomicAdd(a.troubled_count, __popc(ballot));
      base = __shfl_sync(active_mask, base, leader);
      if (troubled)
        a.troubled[base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<std::int32_t>(e);
    }
  }
}

template <int P, int R, int TILE, int MINB, bool MMA, bool ISLANDS>
__global__ void __launch_bounds__(TILE, MINB) euler_tri_patch(const StageArgs a) {
  using S = TriShape<P>;
  using L = PatchSmem<P, R, TILE, MMA>;
  constexpr int M = S::M, QV = MixedVolume<P, R>::QV, QF = S::QF, H = M - 1;
  constexpr double phi0 = 0.70710678118654752440;
  static_assert(4 * TILE < 65536, "face items are 16-bit");
  __shared__ PatchEdge<P> table; // for the few runtime-indexed reads
  __shared__ int item_count;
  extern __shared__ __align__(16) unsigned char smem[];
  double(*smean)[TILE] = reinterpret_cast<double(*)[TILE]>(smem + L::mean);
  double(*sprim)[TILE] = reinterpret_cast<double(*)[TILE]>(smem + L::prim);
  float(*shi)[TILE] = reinterpret_cast<float(*)[TILE]>(smem + L::hi);
  float(*sedge)[TILE] = reinterpret_cast<float(*)[TILE]>(smem + L::edge);
  std::uint16_t *items = reinterpret_cast<std::uint16_t *>(smem + L::items);
  float4 *sfrag = reinterpret_cast<float4 *>(smem + L::frag);
  float(*sbb)[TILE] = reinterpret_cast<float(*)[TILE]>(smem + L::bb);
  float(*sgeo)[TILE] = reinterpret_cast<float(*)[TILE]>(smem + L::geo);
  // The next launch on the stream may start its CTAs (into SM slots this
  // grid's tail leaves free) and run up to its own wait, which holds until
  // this grid has completed.
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");

  const int t = threadIdx.x;
  const std::int64_t ne = a.mesh.ne;
  std::int64_t first = 0, count = 0;
  int case_id = 0;
  if (a.work) {
    const TileWork w = a.work[blockIdx.x];
    first = w.first;
    count = w.count;
    case_id = w.case_id;
  } else {
    first = static_cast<std::int64_t>(blockIdx.x) * TILE;
    count = ne - first < TILE ? ne - first : TILE;
  }
  const bool active = t < count;
  const std::int64_t e = first + t;
  const double *__restrict__ in = a.in;
  const double gamma = a.gamma;
  const PatchEdges pe = a.patch;
  // ISLANDS (with the limiter): faces across jumps of the cell means in FP64.
  constexpr bool islands = ISLANDS;

  {
    const float *src = reinterpret_cast<const float *>(&c_patch<P>);
    float *dst = reinterpret_cast<float *>(&table);
    for (int i = t; i < static_cast<int>(sizeof(table) / sizeof(float)); i += TILE)
      dst[i] = src[i];
  }
  if (t == 0)
    item_count = 0;
  if constexpr (MMA)
    fill_volume_fragments<P, R>(sfrag, t, TILE);
  // The patch's rows of mesh data (read in every phase) and, in stages 2-3,
  // of u^n (read at the end) into L2, one bulk prefetch per row.
  {
    constexpr int kMeshRows = 5 + 9 + 3 + 3;
    const int rows = kMeshRows + (a.stage > 0 ? 4 * M : 0);
    if (t < rows) {
      const void *row;
      std::size_t bytes;
      if (t < 5) {
        row = a.mesh.geo + t * ne + first, bytes = 8 * count;
      } else if (t < 14) {
        row = pe.geo + (t - 5) * ne + first, bytes = 8 * count;
      } else if (t < 17) {
        row = pe.nbr + (t - 14) * ne + first, bytes = 4 * count;
      } else if (t < 20) {
        row = pe.info + (t - 17) * ne + first, bytes = count;
      } else {
        row = a.u0 + (t - kMeshRows) * ne + first, bytes = 8 * count;
      }
      prefetch_row_l2(row, bytes);
    }
  }

  // Launched as a programmatic dependent of the launch before it on the
  // stream (the previous RK stage, or the dt kernel): everything above reads
  // only the mesh, the tables and (as a prefetch hint) u^n.  Wait here for
  // that launch to complete and its writes to be visible before the state,
  // dt or any output is touched.  Without the launch attribute the wait
  // returns at once.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");

  // A. State, traces, and the faces this element evaluates.
  bool evaluates[3] = {false, false, false};
  if (active) {
    std::int32_t nbrs[3];
    unsigned infos[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      nbrs[j] = pe.nbr[j * ne + e];
      if (nbrs[j] >= 0)
        nbrs[j] = static_cast<std::int32_t>(checked_index(nbrs[j], ne, a.error));
      infos[j] = pe.info[j * ne + e];
    }
    double mean[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const double *row = in + static_cast<std::int64_t>(v) * M * ne + e;
      mean[v] = row[0] * phi0;
      float h[H];
#pragma unroll
      for (int m = 0; m < H; ++m) {
        h[m] = static_cast<float>(row[(m + 1) * ne]);
        shi[v * H + m][t] = h[m];
      }
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int q = 0; q < QF; ++q) {
          float s = 0.0f;
#pragma unroll
          for (int m = 0; m < H; ++m)
            s = fmaf(h[m], c_patch<P>.phi[j][q][m], s);
          sedge[(j * QF + q) * 4 + v][t] = s;
        }
    }
    const MeanState own = mean_state(gamma, mean);
#pragma unroll
    for (int v = 0; v < 4; ++v)
      smean[v][t] = mean[v];
    sprim[0][t] = own.u;
    sprim[1][t] = own.v;
    sprim[2][t] = own.p;
    sprim[3][t] = own.h;
    if constexpr (MMA) {
      const Ref32 r = ref32(own);
      const float f[8] = {r.rho, r.u, r.v, r.e, r.h, r.mx, r.my, r.p};
#pragma unroll
      for (int k = 0; k < 8; ++k)
        sbb[k][t] = f[k];
#pragma unroll
      for (int k = 0; k < 4; ++k)
        sgeo[k][t] = static_cast<float>(a.mesh.geo[k * ne + e]);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const std::int64_t local = nbrs[j] - first;
      const bool inside = nbrs[j] >= 0 && local >= 0 && local < count;
      evaluates[j] = !inside || (infos[j] & 1u);
    }
  }
  __syncthreads(); // item_count and the tables are set
  {
    const int lane = t & 31;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const unsigned ballot = __ballot_sync(0xffffffffu, evaluates[j]);
      int base = 0;
      if (lane == 0 && ballot)
        base = atomicAdd(&item_count, __popc(ballot));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (evaluates[j])
        items[base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<std::uint16_t>(t * 4 + j);
    }
  }
  __syncthreads();

  // B. The listed faces, shared out over all threads.
  {
    const float gamma32 = static_cast<float>(gamma), g1 = static_cast<float>(gamma - 1.0);
    const int n = item_count;
    auto evaluate = [&](int i, int q0, auto whole) {
      constexpr int NQ = decltype(whole)::value ? QF : 1;
      const int te = items[i] >> 2, j = items[i] & 3;
      const std::int64_t ee = first + te;
      const std::int32_t raw = pe.nbr[j * ne + ee];
      const std::int32_t nb =
          raw >= 0 ? static_cast<std::int32_t>(checked_index(raw, ne, a.error)) : raw;
      const unsigned info = pe.info[j * ne + ee];
      const bool self_left = info & 1u, rev = info & 8u;
      const int jn = (info >> 1) & 3u;
      const double nx = pe.geo[(3 * j) * ne + ee], ny = pe.geo[(3 * j + 1) * ne + ee];
      const bool boundary = nb < 0;
      const std::int64_t local = nb - first;
      const bool near = !boundary && local >= 0 && local < count;
      double mean[4], nmean[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int v = 0; v < 4; ++v)
        mean[v] = smean[v][te];
      if (near) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          nmean[v] = smean[v][local];
      } else if (!boundary) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          nmean[v] = __ldg(in + static_cast<std::int64_t>(v) * M * ne + nb) * phi0;
      }
      // A face across a jump of the means is evaluated in FP64 by each of its
      // elements in phase C (with the limiter): no record here.
      if (islands && !boundary && mean_jump(nmean[0], mean[0], nmean[3], mean[3]))
        return;
      // The face's left mean state: the reference of the perturbation form.
      MeanState ml;
      if (self_left || boundary)
        ml = patch_mean<P, TILE>(smean, sprim, te);
      else if (near)
        ml = patch_mean<P, TILE>(smean, sprim, static_cast<int>(local));
      else
        ml = mean_state(gamma, nmean);
      const Ref32 ref = ref32(ml);
      float jump[4];
#pragma unroll
      for (int v = 0; v < 4; ++v)
        jump[v] = boundary ? 0.0f
                           : static_cast<float>(self_left ? nmean[v] - mean[v] : mean[v] - nmean[v]);
      const float nxf = static_cast<float>(nx), nyf = static_cast<float>(ny);
#pragma unroll
      for (int jq = 0; jq < NQ; ++jq) {
        const int q = q0 + jq;              // the face's point (left element's order)
        const int qr = rev ? QF - 1 - q : q; // the right element's point
        const int qs = self_left ? q : qr;   // this element's point
        float to[4], tn[4], dl[4], dr[4], fl[4];
#pragma unroll
        for (int v = 0; v < 4; ++v)
          to[v] = sedge[(j * QF + qs) * 4 + v][te];
        if (boundary) {
#pragma unroll
          for (int v = 0; v < 4; ++v)
            dl[v] = dr[v] = to[v];
        } else {
          const int qn = self_left ? qr : q;
          if (near) {
#pragma unroll
            for (int v = 0; v < 4; ++v)
              tn[v] = sedge[(jn * QF + qn) * 4 + v][local];
          } else {
            patch_outside_trace<P>(in, ne, nb, table.phi[jn][qn], tn);
          }
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            dl[v] = self_left ? to[v] : tn[v];
            dr[v] = jump[v] + (self_left ? tn[v] : to[v]);
          }
        }
        hllc_perturbed<true>(ref, dl, dr, g1, gamma32, nxf, nyf, fl);
#pragma unroll
        for (int v = 0; v < 4; ++v)
          sedge[(j * QF + qs) * 4 + v][te] = fl[v];
      }
    };
    const int whole = n / TILE * TILE;
#pragma unroll 1
    for (int i = t; i < whole; i += TILE)
      evaluate(i, 0, std::true_type{});
#pragma unroll 1
    for (int u = t; u < (n - whole) * QF; u += TILE)
      evaluate(whole + u / QF, u % QF, std::false_type{});
  }
  __syncthreads();
  const float g1 = static_cast<float>(gamma - 1.0);
  if constexpr (MMA) // every lane of every warp, active or not
    patch_volume_mma<P, R, TILE>(shi, sbb, sgeo, sfrag, g1, t & ~31, t & 31);
  if (!active)
    return;

  // C. Volume term, lifting, mode 0, combination.
  const MeanState own = patch_mean<P, TILE>(smean, sprim, t);
  float racc[4][H];
  if constexpr (MMA) {
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int m = 0; m < H; ++m)
        racc[v][m] = shi[v * H + m][t];
  } else {
    const Ref32 bb = ref32(own);
    const MixedVolume<P, R> &T = c_mix<P, R>;
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int m = 0; m < H; ++m)
        racc[v][m] = 0.0f;
    float ch[4][H];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int m = 0; m < H; ++m)
        ch[v][m] = shi[v * H + m][t];
    const double *__restrict__ geo = a.mesh.geo;
    const float fax = static_cast<float>(geo[e]), fay = static_cast<float>(geo[ne + e]);
    const float fbx = static_cast<float>(geo[2 * ne + e]), fby = static_cast<float>(geo[3 * ne + e]);
#pragma unroll
    for (int q = 0; q < QV; ++q) {
      float d[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        float s = 0.0f;
#pragma unroll
        for (int m = 0; m < H; ++m)
          s = fmaf(ch[v][m], T.phi[q][m], s);
        d[v] = s;
      }
      const float inv = perturbation_rcp<true>(fmaxf(bb.rho + d[0], kVacuumFraction * bb.rho));
      const float du = (d[1] - bb.u * d[0]) * inv;
      const float dv = (d[2] - bb.v * d[0]) * inv;
      const float uu = bb.u + du, vv = bb.v + dv;
      const float dmu = bb.mx * du + d[1] * uu + bb.my * dv + d[2] * vv;
      const float dp = g1 * (d[3] - 0.5f * dmu);
      const float dep = d[3] + dp;
      const float fx[4] = {d[1], bb.mx * du + d[1] * uu + dp, bb.my * du + d[2] * uu,
                           bb.h * du + dep * uu};
      const float fy[4] = {d[2], bb.mx * dv + d[1] * vv, bb.my * dv + d[2] * vv + dp,
                           bb.h * dv + dep * vv};
      const float w = T.w[q];
      const float wby = w * fby, wbx = w * fbx, wax = w * fax, way = w * fay;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float gxi = wby * fx[v] - wbx * fy[v];
        const float geta = wax * fy[v] - way * fx[v];
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(T.dxi[q][m], gxi, fmaf(T.deta[q][m], geta, racc[v][m]));
      }
    }
  }

  double r0[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const std::int32_t raw = pe.nbr[j * ne + e];
    const std::int32_t nb =
        raw >= 0 ? static_cast<std::int32_t>(checked_index(raw, ne, a.error)) : raw;
    const unsigned info = pe.info[j * ne + e];
    const bool self_left = info & 1u, rev = info & 8u;
    const int jn = (info >> 1) & 3u;
    const double nx = pe.geo[(3 * j) * ne + e], ny = pe.geo[(3 * j + 1) * ne + e];
    const double scale = pe.geo[(3 * j + 2) * ne + e];
    const bool boundary = nb < 0;
    const std::int64_t local = nb - first;
    const bool near = !boundary && local >= 0 && local < count;
    const int jl = self_left ? j : jn; // the face's left local edge (its weights)
    // The face's flux perturbations in the face's point order: from this
    // element's record, or from its left neighbour's inside the patch.
    // (An FP64 face overwrites these with its own values below.)
    float fq[QF][4];
    if (near && !self_left) {
#pragma unroll
      for (int q = 0; q < QF; ++q)
#pragma unroll
        for (int v = 0; v < 4; ++v)
          fq[q][v] = sedge[(jn * QF + q) * 4 + v][local];
    } else {
#pragma unroll
      for (int q = 0; q < QF; ++q) {
        const int qs = self_left || !rev ? q : QF - 1 - q;
#pragma unroll
        for (int v = 0; v < 4; ++v)
          fq[q][v] = sedge[(j * QF + qs) * 4 + v][t];
      }
    }
    // The face's left mean state; with islands, the neighbour's mean for the
    // jump test as well.
    MeanState ml;
    double nmean[4] = {0.0, 0.0, 0.0, 0.0};
    if constexpr (ISLANDS) {
      if (near) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          nmean[v] = smean[v][local];
      } else if (!boundary) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          nmean[v] = __ldg(in + static_cast<std::int64_t>(v) * M * ne + nb) * phi0;
      }
    }
    if (self_left || boundary) {
      ml = own;
    } else if (near) {
      ml = patch_mean<P, TILE>(smean, sprim, static_cast<int>(local));
    } else {
      if constexpr (!ISLANDS) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          nmean[v] = __ldg(in + static_cast<std::int64_t>(v) * M * ne + nb) * phi0;
      }
      ml = mean_state(gamma, nmean);
    }
    double fln[4];
    mean_normal_flux(ml, nx, ny, fln);
    const bool fp64 = ISLANDS && !boundary &&
                      mean_jump(nmean[0], smean[0][t], nmean[3], smean[3][t]);
    double m0[4] = {0.0, 0.0, 0.0, 0.0};
    if constexpr (ISLANDS) {
      if (fp64) {
        // The face in FP64 from both elements' coefficients, as the tile
        // kernels' rough pass evaluates it (the same call with the same roles
        // on both sides, so both elements apply the same bits).
        const FaceTable<P, double> *T64 =
            static_cast<const FaceTable<P, double> *>(a.face_table64);
        const int le = self_left ? j : jn, re = self_left ? jn : j;
        // The tables' flip is the edges' relative direction along the
        // counter-clockwise parametrization; rev compares the edges' own
        // point orders, and edge 2's points run against it.
        const int flip = (rev ? 1 : 0) ^ (le == 2 ? 1 : 0) ^ (re == 2 ? 1 : 0);
        const double *lb64 = &T64->lb[le][0][0];
        const double *rb64 = &T64->rb[(le * 3 + re) * 2 + flip][0][0];
        float dq[QF][4];
        face_fp64<P>(gamma, in + e, ne, in + nb, ne, false, self_left, self_left ? lb64 : rb64,
                     self_left ? rb64 : lb64, &T64->ew[le][0], nx, ny, fln, dq, m0);
#pragma unroll
        for (int q = 0; q < QF; ++q)
#pragma unroll
          for (int v = 0; v < 4; ++v)
            fq[q][v] = dq[q][v];
      }
    }
    float shift[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (!boundary && !self_left) {
      double frn[4];
      mean_normal_flux(own, nx, ny, frn);
#pragma unroll
      for (int v = 0; v < 4; ++v)
        shift[v] = static_cast<float>(fln[v] - frn[v]);
    }
    const float fscale = static_cast<float>(scale);
    const double sgn = self_left ? -1.0 : 1.0;
    if (fp64) {
#pragma unroll
      for (int v = 0; v < 4; ++v)
        r0[v] += sgn * scale * phi0 * m0[v];
    } else {
      float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int q = 0; q < QF; ++q) {
        const float w = table.w[jl][q];
#pragma unroll
        for (int v = 0; v < 4; ++v)
          acc[v] = fmaf(w, fq[q][v], acc[v]);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const double mode0 = fln[v] * c_edge_wsum<P>[jl] + static_cast<double>(acc[v]);
        r0[v] += sgn * scale * phi0 * mode0;
      }
    }
    // High modes at this element's own points qo (the face's point q).
#pragma unroll
    for (int qo = 0; qo < QF; ++qo) {
      const bool flipped = !self_left && rev;
      const float w = table.w[jl][flipped ? QF - 1 - qo : qo];
      const float wsc = (self_left ? -w : w) * fscale;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float f = flipped ? fq[QF - 1 - qo][v] : fq[qo][v];
        const float value = wsc * (self_left ? f : f + shift[v]);
#pragma unroll
        for (int m = 0; m < H; ++m)
          racc[v][m] = fmaf(value, c_patch<P>.phi[j][qo][m], racc[v][m]);
      }
    }
  }
  patch_finish<P>(a, e, case_id, r0, racc);
}

// Per-case CFL speed over a tile work list: the largest cell-average wave
// speed |u| + c of each case (the CFL kernels' formula), max-reduced as FP64
// bits into speed[case]; a non-physical average sets the error word.
__global__ void batch_speed(const double *state, std::int64_t ne, int M, double gamma,
                            const TileWork *work, unsigned long long *speed,
                            unsigned long long *error, int *status) {
  const TileWork w = work[blockIdx.x];
  const int lane = threadIdx.x & 31;
  unsigned long long best = 0;
  for (int i = threadIdx.x; i < w.count; i += blockDim.x) {
    const std::int64_t e = w.first + i;
    const double scale = 1.0 / sqrt(2.0);
    const std::int64_t plane = static_cast<std::int64_t>(M) * ne;
    const double s[4] = {__dmul_rn(scale, state[e]), __dmul_rn(scale, state[plane + e]),
                         __dmul_rn(scale, state[2 * plane + e]),
                         __dmul_rn(scale, state[3 * plane + e])};
    bool physical = true;
    const double speed = cfl_speed(gamma, s, 2, physical);
    if (physical) {
      const unsigned long long bits = __double_as_longlong(speed);
      best = bits > best ? bits : best;
    } else if (status) {
      atomicCAS(status + w.case_id, 0, static_cast<int>(kNonPhysicalAverage));
    } else {
      raise_error(error, kNonPhysicalAverage, e);
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_down_sync(0xffffffffu, best, off);
    best = o > best ? o : best;
  }
  if (lane == 0 && best)
    atomicMax(speed + w.case_id, best);
}

namespace {

void check(cudaError_t rc, const char *what) {
  if (rc != cudaSuccess)
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(rc));
}

template <int P, int R> void upload_mixed() {
  static MixedVolume<P, R> t;
  constexpr int M = TriShape<P>::M, QV = MixedVolume<P, R>::QV;
  const Rule2D rule = R == 0 ? symmetric_triangle_rule(2 * P) : triangle_rule(R);
  if (rule.size() != QV)
    throw std::logic_error("mixed volume table: rule size");
  std::vector<double> gx, ge;
  for (int q = 0; q < QV; ++q) {
    const auto b = dubiner(rule.xi[q], rule.eta[q], P);
    dubiner_gradient(rule.xi[q], rule.eta[q], P, gx, ge);
    for (int m = 1; m < M; ++m) {
      t.phi[q][m - 1] = static_cast<float>(b[m]);
      t.dxi[q][m - 1] = static_cast<float>(gx[m]);
      t.deta[q][m - 1] = static_cast<float>(ge[m]);
    }
    t.w[q] = static_cast<float>(0.5 * rule.w[q]);
  }
  check(cudaMemcpyToSymbol(c_mix<P, R>, &t, sizeof(t)), "upload mixed volume table");
  static FaceTable<P, double> f;
  fill_face_table<P, double>(f);
  double wsum[3];
  for (int le = 0; le < 3; ++le) {
    double sum = 0.0;
    for (int q = 0; q < TriShape<P>::QF; ++q)
      sum += f.ew[le][q];
    wsum[le] = sum;
  }
  check(cudaMemcpyToSymbol(c_edge_wsum<P>, wsum, sizeof(wsum)), "upload edge weight sums");
  static PatchEdge<P> pt;
  for (int le = 0; le < 3; ++le)
    for (int q = 0; q < TriShape<P>::QF; ++q) {
      for (int m = 1; m < TriShape<P>::M; ++m)
        pt.phi[le][q][m - 1] = static_cast<float>(f.lb[le][q][m]);
      pt.w[le][q] = static_cast<float>(f.ew[le][q]);
    }
  check(cudaMemcpyToSymbol(c_patch<P>, &pt, sizeof(pt)), "upload patch edge table");
}

template <int P, int R> void stage_mixed(const StageArgs &a, cudaStream_t s) {
  if (a.boundary.count > 0 && a.mesh.boundary != 3 && !a.boundary.paired)
    boundary_mode0<P><<<static_cast<unsigned>((a.boundary.count + 127) / 128), 128, 0, s>>>(a);
  euler_tri_faces_mixed<P><<<static_cast<unsigned>((a.faces.count + 127) / 128), 128, 0, s>>>(a);
  euler_tri_elements_mixed<P, R>
      <<<static_cast<unsigned>((a.mesh.ne + 127) / 128), 128, 0, s>>>(a);
}

template <int P, int TILE> constexpr std::size_t tile_smem() {
  return sizeof(double) * 4 * TriShape<P>::M * TILE;
}

// Static (face table) plus dynamic shared memory above the default 48 KiB
// needs the opt-in attribute, set once per device and kernel (and before any
// capture).
template <typename Kernel>
void smem_opt_in(Kernel kernel, std::size_t dynamic, std::size_t fixed, bool (&opted_in)[64]) {
  if (dynamic + fixed <= 48 * 1024)
    return;
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  if (device < 64 && opted_in[device])
    return;
  check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(dynamic)),
        "tile kernel shared memory");
  if (device < 64)
    opted_in[device] = true;
}

// A stage kernel launched as a programmatic dependent of the launch before
// it on the stream: its CTAs may start while that launch drains, and wait
// (griddepcontrol.wait) before reading what it wrote.
template <typename Kernel>
void launch_dependent(Kernel kernel, unsigned blocks, unsigned threads, std::size_t smem,
                      cudaStream_t s, const StageArgs &a) {
  cudaLaunchConfig_t config = {};
  config.gridDim = dim3(blocks);
  config.blockDim = dim3(threads);
  config.dynamicSmemBytes = smem;
  config.stream = s;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attribute[0].val.programmaticStreamSerializationAllowed = 1;
  config.attrs = attribute;
  config.numAttrs = 1;
  check(cudaLaunchKernelEx(&config, kernel, a), "patch kernel launch");
}

template <int P, int R, int TILE, int MINB> void tile_opt_in() {
  static bool opted_in[64] = {};
  smem_opt_in(euler_tri_tile_mixed<P, R, TILE, MINB, false>, tile_smem<P, TILE>(),
              sizeof(FaceTable<P, float>), opted_in);
}

template <int P, int R, int TILE, int MINB> void shared_opt_in() {
  static bool opted_in[64] = {};
  smem_opt_in(euler_tri_tile_shared<P, R, TILE, MINB>, SharedFaceSmem<P, TILE>::bytes,
              sizeof(FaceTable<P, float>) + sizeof(int), opted_in);
}

// The second pass: one warp per CTA and no register cap, so a short rough
// list spreads over many SMs (its elements read their neighbours from L2).
constexpr int kRoughTile = 32;

// The FP32 pass over all tiles, then (with a rough list) the pass over the
// elements it left, sized for the worst case: its CTAs beyond the list's
// length return at once.  SHARED picks the shared-face tile kernel for the
// FP32 pass.
template <int P, int R, int TILE, int MINB, bool SHARED = false>
void stage_tile(const StageArgs &a, cudaStream_t s) {
  if constexpr (SHARED)
    shared_opt_in<P, R, TILE, MINB>();
  else
    tile_opt_in<P, R, TILE, MINB>();
  const std::int64_t blocks = a.work ? a.work_count : (a.mesh.ne + TILE - 1) / TILE;
  if (blocks <= 0)
    return;
  if (a.rough)
    check(cudaMemsetAsync(a.rough_count, 0, sizeof(std::int32_t), s), "rough count");
  if constexpr (SHARED)
    euler_tri_tile_shared<P, R, TILE, MINB>
        <<<static_cast<unsigned>(blocks), TILE, SharedFaceSmem<P, TILE>::bytes, s>>>(a);
  else
    euler_tri_tile_mixed<P, R, TILE, MINB, false>
        <<<static_cast<unsigned>(blocks), TILE, tile_smem<P, TILE>(), s>>>(a);
  if (a.rough)
    euler_tri_tile_mixed<P, R, kRoughTile, 1, true>
        <<<static_cast<unsigned>((a.mesh.ne + kRoughTile - 1) / kRoughTile), kRoughTile,
           tile_smem<P, kRoughTile>(), s>>>(a);
}

// The persistent tile kernel's attributes and its grid: every CTA resident
// at once (CTAs per SM at this shape's registers and shared memory, times the
// SMs), found once per device.
template <int P, int R, int TILE, int MINB> int persistent_prepare() {
  static bool opted_in[64] = {};
  static int resident[64] = {};
  smem_opt_in(euler_tri_tile_persistent<P, R, TILE, MINB>, tile_smem<P, TILE>(),
              sizeof(FaceTable<P, float>), opted_in);
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  if (device < 64 && resident[device])
    return resident[device];
  int per_sm = 0, sms = 0;
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, euler_tri_tile_persistent<P, R, TILE, MINB>, TILE, tile_smem<P, TILE>()),
        "persistent tile occupancy");
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
  const int blocks = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  if (device < 64)
    resident[device] = blocks;
  return blocks;
}

// The FP32 pass as the persistent tile kernel (one wave of resident CTAs
// looping over the tiles), then the rough pass as stage_tile runs it.
template <int P, int R, int TILE, int MINB>
void stage_tile_persistent(const StageArgs &a, cudaStream_t s) {
  const int resident = persistent_prepare<P, R, TILE, MINB>();
  const std::int64_t tiles = a.work ? a.work_count : (a.mesh.ne + TILE - 1) / TILE;
  if (tiles <= 0)
    return;
  if (a.rough)
    check(cudaMemsetAsync(a.rough_count, 0, sizeof(std::int32_t), s), "rough count");
  const std::int64_t blocks = tiles < resident ? tiles : resident;
  euler_tri_tile_persistent<P, R, TILE, MINB>
      <<<static_cast<unsigned>(blocks), TILE, tile_smem<P, TILE>(), s>>>(a);
  if (a.rough)
    euler_tri_tile_mixed<P, R, kRoughTile, 1, true>
        <<<static_cast<unsigned>((a.mesh.ne + kRoughTile - 1) / kRoughTile), kRoughTile,
           tile_smem<P, kRoughTile>(), s>>>(a);
}

template <int P, int R, int TILE, int MINB, bool MMA> void patch_opt_in() {
  static bool opted_in[64] = {}, opted_in_islands[64] = {};
  smem_opt_in(euler_tri_patch<P, R, TILE, MINB, MMA, false>, PatchSmem<P, R, TILE, MMA>::bytes,
              sizeof(PatchEdge<P>) + sizeof(int), opted_in);
  if constexpr (!MMA)
    smem_opt_in(euler_tri_patch<P, R, TILE, MINB, false, true>, PatchSmem<P, R, TILE, false>::bytes,
                sizeof(PatchEdge<P>) + sizeof(int), opted_in_islands);
}

// The patch kernel over all patches (no rough pass: runs without the limiter).
template <int P, int R, int TILE, int MINB, bool MMA = false>
void stage_patch(const StageArgs &a, cudaStream_t s) {
  if (!a.patch.nbr)
    throw std::invalid_argument("patch kernel: the mesh has no patch edge arrays");
  patch_opt_in<P, R, TILE, MINB, MMA>();
  const std::int64_t blocks = a.work ? a.work_count : (a.mesh.ne + TILE - 1) / TILE;
  if (blocks <= 0)
    return;
  if (!a.rough) {
    launch_dependent(euler_tri_patch<P, R, TILE, MINB, MMA, false>,
                     static_cast<unsigned>(blocks), TILE, PatchSmem<P, R, TILE, MMA>::bytes, s, a);
  } else if constexpr (!MMA) {
    // With the limiter: faces across jumps of the means in FP64, inline.
    launch_dependent(euler_tri_patch<P, R, TILE, MINB, false, true>,
                     static_cast<unsigned>(blocks), TILE, PatchSmem<P, R, TILE, false>::bytes, s, a);
  } else {
    throw std::invalid_argument("patch kernel with the tensor-core volume: runs without the"
                                " limiter");
  }
}

// Launch shapes of the tile kernels (elements per CTA, register budget):
//   0: 128 elements, <= 128 registers (4 CTAs / 16 warps per SM)
//   1: 128 elements, no register cap
//   2: 256 elements, <= 128 registers (2 CTAs per SM)
//   3:  64 elements, <= 128 registers (8 CTAs per SM)
// and of the shared-face tile kernel:
//   4:  64 elements, sized for 7 CTAs per SM (14 warps)
//   5:  96 elements, sized for 5 CTAs per SM (15 warps)
//   6: 128 elements, sized for 4 CTAs per SM (16 warps)
//   7: 128 elements, sized for 3 CTAs per SM
// and of the patch kernel:
//   8: 128 elements, <= 128 registers (4 CTAs per SM)
//   9: 128 elements, sized for 5 CTAs per SM
//  10:  64 elements, sized for 8 CTAs per SM
//  11:  64 elements, sized for 10 CTAs per SM
// and of the patch kernel with its volume term on the tensor cores:
//  12: 128 elements, <= 128 registers
//  13: 128 elements, sized for 5 CTAs per SM
// and of the persistent tile kernel (one wave of resident CTAs looping over
// the tiles of the mesh or of the batch's work list):
//  14: 128 elements, <= 128 registers
//  15: 256 elements, <= 128 registers
constexpr int kTileShapes = kTileShapeCount;
constexpr int kTileElements[kTileShapes] = {128, 128, 256, 64, 64, 96, 128, 128,
                                            128, 128, 64, 64, 128, 128, 128, 256};
constexpr int kFirstPatchShape = 8, kPatchShapeEnd = 14;

template <int P, int R> struct StageTile {
  static void run(int shape, const StageArgs &a, cudaStream_t s) {
    switch (shape) {
    case 0: stage_tile<P, R, 128, 4>(a, s); break;
    case 1: stage_tile<P, R, 128, 1>(a, s); break;
    case 2: stage_tile<P, R, 256, 2>(a, s); break;
    case 3: stage_tile<P, R, 64, 8>(a, s); break;
    case 4: stage_tile<P, R, 64, 7, true>(a, s); break;
    case 5: stage_tile<P, R, 96, 5, true>(a, s); break;
    case 6: stage_tile<P, R, 128, 4, true>(a, s); break;
    case 7: stage_tile<P, R, 128, 3, true>(a, s); break;
    case 8: stage_patch<P, R, 128, 4>(a, s); break;
    case 9: stage_patch<P, R, 128, 5>(a, s); break;
    case 10: stage_patch<P, R, 64, 8>(a, s); break;
    case 11: stage_patch<P, R, 64, 10>(a, s); break;
    case 12: stage_patch<P, R, 128, 4, true>(a, s); break;
    case 13: stage_patch<P, R, 128, 5, true>(a, s); break;
    case 14: stage_tile_persistent<P, R, 128, 4>(a, s); break;
    case 15: stage_tile_persistent<P, R, 256, 2>(a, s); break;
    default: throw std::invalid_argument("tile kernel: unknown launch shape");
    }
  }
};

template <int P, int R> struct PrepareTile {
  static void run() {
    tile_opt_in<P, R, 128, 4>();
    tile_opt_in<P, R, 128, 1>();
    tile_opt_in<P, R, 256, 2>();
    tile_opt_in<P, R, 64, 8>();
    shared_opt_in<P, R, 64, 7>();
    shared_opt_in<P, R, 96, 5>();
    shared_opt_in<P, R, 128, 4>();
    shared_opt_in<P, R, 128, 3>();
    patch_opt_in<P, R, 128, 4, false>();
    patch_opt_in<P, R, 128, 5, false>();
    patch_opt_in<P, R, 64, 8, false>();
    patch_opt_in<P, R, 64, 10, false>();
    patch_opt_in<P, R, 128, 4, true>();
    patch_opt_in<P, R, 128, 5, true>();
    persistent_prepare<P, R, 128, 4>();
    persistent_prepare<P, R, 256, 2>();
  }
};

// Op<P, R>::run(args...) for a supported (p, rule order) pair.
template <int P, int R> struct UploadMixed {
  static void run() { upload_mixed<P, R>(); }
};
template <int P, int R> struct StageMixed {
  static void run(const StageArgs &a, cudaStream_t s) { stage_mixed<P, R>(a, s); }
};

template <template <int, int> class Op, typename... A> void dispatch_mixed(int p, int rule, A &&...args) {
  if (rule == 0)
    rule = p + 2;
  else if (rule == kSymmetricVolumeRule)
    rule = 0; // the template's code for the symmetric rule
  switch (p * 10 + rule) {
  case 11: Op<1, 1>::run(args...); break;
  case 12: Op<1, 2>::run(args...); break;
  case 13: Op<1, 3>::run(args...); break;
  case 22: Op<2, 2>::run(args...); break;
  case 23: Op<2, 3>::run(args...); break;
  case 24: Op<2, 4>::run(args...); break;
  case 33: Op<3, 3>::run(args...); break;
  case 34: Op<3, 4>::run(args...); break;
  case 35: Op<3, 5>::run(args...); break;
  case 10: Op<1, 0>::run(args...); break;
  case 20: Op<2, 0>::run(args...); break;
  case 30: Op<3, 0>::run(args...); break;
  default:
    throw std::invalid_argument("mixed form: polynomial order must be 1..3 and the volume rule"
                                " order p..p+2");
  }
}

} // namespace

bool euler_tri_mixed_supported(int p, int rule) {
  if (rule == 0)
    rule = p + 2;
  return p >= 1 && p <= 3 && (rule == kSymmetricVolumeRule || (rule >= p && rule <= p + 2));
}

std::size_t euler_tri_mixed_face_record_bytes(int p) {
  switch (p) {
  case 1: return sizeof(FaceRecord<1>);
  case 2: return sizeof(FaceRecord<2>);
  case 3: return sizeof(FaceRecord<3>);
  default: throw std::invalid_argument("mixed form: polynomial order must be 1..3");
  }
}

void upload_euler_tri_tables_mixed(int p, int rule) {
  dispatch_mixed<UploadMixed>(p, rule);
}

int euler_tri_tile_shapes() { return kTileShapes; }

int euler_tri_tile_elements(int shape) {
  return shape >= 0 && shape < kTileShapes ? kTileElements[shape] : 0;
}

bool euler_tri_tile_is_patch(int shape) { return shape >= kFirstPatchShape && shape < kPatchShapeEnd; }

bool euler_tri_tile_limits(int shape) { return shape != 12 && shape != 13; }



void prepare_euler_tri_stage_tile(int p, int rule) { dispatch_mixed<PrepareTile>(p, rule); }

void launch_euler_tri_stage_tile(int p, int rule, int shape, const StageArgs &a, cudaStream_t s) {
  dispatch_mixed<StageTile>(p, rule, shape, a, s);
}

void launch_batch_speed(const double *state, std::int64_t ne, int M, double gamma,
                        const TileWork *work, std::int64_t work_count, unsigned long long *speed,
                        unsigned long long *error, int *status, cudaStream_t s) {
  if (work_count > 0)
    batch_speed<<<static_cast<unsigned>(work_count), 128, 0, s>>>(state, ne, M, gamma, work, speed,
                                                                  error, status);
}

void launch_euler_tri_stage_mixed(int p, int rule, const StageArgs &a, cudaStream_t s) {
  dispatch_mixed<StageMixed>(p, rule, a, s);
}

} // namespace wasl_b200
