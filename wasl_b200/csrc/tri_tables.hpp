// Reference-element tables of the triangle Euler kernels for one polynomial order.
//
// Volume: the collapsed rule of order p+2, (p+3)^2 points, as the reference
// residual uses (cpp/include/wasl/dg/euler/triangle_residual.hpp:32): basis
// values, reference gradients and weights.  Faces: the left element's basis at
// the p+1 Gauss points of each local edge, the edge weights, and the right
// element's basis at the matching points for every (left edge, right edge,
// orientation flip) combination (triangle_face_trace.hpp:16-33).  The tables
// are built on the host from the reference formulas, so they hold the doubles
// the reference evaluates in its loops.
#pragma once

#include <cstddef>

#include "basis.hpp"

namespace wasl_b200 {

template <int P> struct TriShape {
  static constexpr int M = (P + 1) * (P + 2) / 2;
  static constexpr int QV = (P + 3) * (P + 3);
  static constexpr int QF = P + 1;
};

template <int P, typename T> struct VolumeTable {
  static constexpr int M = TriShape<P>::M, QV = TriShape<P>::QV;
  T phi[QV][M];
  T dxi[QV][M];
  T deta[QV][M];
  T w[QV];
};

template <int P, typename T> struct FaceTable {
  static constexpr int M = TriShape<P>::M, QF = TriShape<P>::QF;
  T lb[3][QF][M];        // left basis on local edge le
  T ew[3][QF];           // reference edge weights
  T rb[18][QF][M];       // right basis, index (le * 3 + re) * 2 + flip
};

template <int P, typename T> void fill_volume_table(VolumeTable<P, T> &t) {
  constexpr int M = TriShape<P>::M, QV = TriShape<P>::QV;
  const Rule2D rule = triangle_rule(P + 2);
  std::vector<double> gx, ge;
  for (int q = 0; q < QV; ++q) {
    const auto b = dubiner(rule.xi[q], rule.eta[q], P);
    dubiner_gradient(rule.xi[q], rule.eta[q], P, gx, ge);
    for (int m = 0; m < M; ++m) {
      t.phi[q][m] = static_cast<T>(b[m]);
      t.dxi[q][m] = static_cast<T>(gx[m]);
      t.deta[q][m] = static_cast<T>(ge[m]);
    }
    t.w[q] = static_cast<T>(rule.w[q]);
  }
}

template <int P, typename T> void fill_face_table(FaceTable<P, T> &t) {
  constexpr int M = TriShape<P>::M, QF = TriShape<P>::QF;
  const Rule2D edges = triangle_edges(P);
  for (int le = 0; le < 3; ++le)
    for (int q = 0; q < QF; ++q) {
      const double lxi = edges.xi[le * QF + q], leta = edges.eta[le * QF + q];
      const auto b = dubiner(lxi, leta, P);
      for (int m = 0; m < M; ++m)
        t.lb[le][q][m] = static_cast<T>(b[m]);
      t.ew[le][q] = static_cast<T>(edges.w[le * QF + q]);
      for (int re = 0; re < 3; ++re)
        for (int flip = 0; flip < 2; ++flip) {
          double rxi = 0.0, reta = 0.0;
          neighbour_point(le, re, flip != 0, lxi, leta, rxi, reta);
          const auto rbv = dubiner(rxi, reta, P);
          for (int m = 0; m < M; ++m)
            t.rb[(le * 3 + re) * 2 + flip][q][m] = static_cast<T>(rbv[m]);
        }
    }
}

} // namespace wasl_b200
