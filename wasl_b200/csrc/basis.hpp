// Host-side modal bases and quadrature rules of the Wasl discretization.
//
// These build the reference-element tables the kernels read (basis values and
// gradients at quadrature points, edge traces, neighbour traces).  They follow
// the reference's definitions so that every table entry is the same double
// the reference evaluates:
//   Jacobi recurrence            cpp/include/wasl/basis/jacobi.hpp:12-35
//   orthonormal Legendre         cpp/include/wasl/basis/legendre.hpp:23-60
//   orthonormal Dubiner          cpp/include/wasl/basis/dubiner_triangle.hpp:36-103
//   Gauss-Legendre, n = 1..7     cpp/include/wasl/quadrature/gauss_legendre.hpp:24-65
//   collapsed triangle rule      cpp/include/wasl/quadrature/triangle_volume_rule.hpp:34-51
//   triangle edge rules          cpp/include/wasl/quadrature/triangle_edge_rules.hpp:28-58
// Host code in this library is compiled with -ffp-contract=off so no fused
// multiply-add changes a rounding.
#pragma once

#include <array>
#include <cmath>
#include <stdexcept>
#include <vector>

namespace wasl_b200 {

constexpr int line_modes(int p) { return p + 1; }
constexpr int tri_modes(int p) { return (p + 1) * (p + 2) / 2; }

inline double jacobi(double x, int n, double alpha, double beta) {
  if (n <= 0)
    return 1.0;
  double prev = 1.0;
  double curr = 0.5 * (alpha - beta + (alpha + beta + 2.0) * x);
  for (int k = 1; k < n; ++k) {
    const double ab = 2.0 * k + alpha + beta;
    const double a = 2.0 * (k + 1) * (k + alpha + beta + 1.0) * ab;
    const double b = (ab + 1.0) * (ab * (ab + 2.0) * x + (alpha * alpha - beta * beta));
    const double c = 2.0 * (k + alpha) * (k + beta) * (ab + 2.0);
    const double next = (b * curr - c * prev) / a;
    prev = curr;
    curr = next;
  }
  return curr;
}

inline double jacobi_derivative(double x, int n, double alpha, double beta) {
  if (n <= 0)
    return 0.0;
  return 0.5 * (n + alpha + beta + 1.0) * jacobi(x, n - 1, alpha + 1.0, beta + 1.0);
}

inline double legendre_norm(int j) { return std::sqrt((2.0 * j + 1.0) / 2.0); }

// Orthonormal Legendre modes 0..p at xi.
inline std::vector<double> legendre(double xi, int p) {
  std::vector<double> v(p + 1);
  v[0] = legendre_norm(0);
  if (p <= 0)
    return v;
  double prev = 1.0, curr = xi;
  v[1] = legendre_norm(1) * curr;
  for (int j = 1; j < p; ++j) {
    const double next = ((2.0 * j + 1.0) * xi * curr - j * prev) / (j + 1);
    prev = curr;
    curr = next;
    v[j + 1] = legendre_norm(j + 1) * curr;
  }
  return v;
}

inline std::vector<double> legendre_gradient(double xi, int p) {
  std::vector<double> g(p + 1);
  g[0] = 0.0;
  if (p <= 0)
    return g;
  double prev = 1.0, curr = xi, dprev = 0.0, dcurr = 1.0;
  g[1] = legendre_norm(1) * dcurr;
  for (int j = 1; j < p; ++j) {
    const double next = ((2.0 * j + 1.0) * xi * curr - j * prev) / (j + 1);
    const double dnext = ((2.0 * j + 1.0) * (curr + xi * dcurr) - j * dprev) / (j + 1);
    prev = curr;
    curr = next;
    dprev = dcurr;
    dcurr = dnext;
    g[j + 1] = legendre_norm(j + 1) * dcurr;
  }
  return g;
}

// Collapsed coordinate a(xi, eta) of the Dubiner construction; a = -1 at the apex.
inline double collapsed(double xi, double eta) {
  return (eta < 1.0) ? (2.0 + 2.0 * xi) / (1.0 - eta) - 1.0 : -1.0;
}

inline double dubiner_norm(int i, int n) { return std::sqrt((2.0 * i + 1.0) * (n + 1.0) / 2.0); }

// Orthonormal Dubiner modes, ordered by total degree n then by i, at (xi, eta).
inline std::vector<double> dubiner(double xi, double eta, int p) {
  std::vector<double> v;
  v.reserve(tri_modes(p));
  const double a = collapsed(xi, eta);
  const double half = 0.5 * (1.0 - eta);
  for (int n = 0; n <= p; ++n)
    for (int i = 0; i <= n; ++i) {
      const int j = n - i;
      const double pi = jacobi(a, i, 0.0, 0.0);
      const double warp = std::pow(half, static_cast<double>(i));
      const double qj = jacobi(eta, j, 2.0 * i + 1.0, 0.0);
      v.push_back(dubiner_norm(i, n) * pi * warp * qj);
    }
  return v;
}

// d/dxi and d/deta of every Dubiner mode at an interior point.
inline void dubiner_gradient(double xi, double eta, int p, std::vector<double> &dxi,
                             std::vector<double> &deta) {
  dxi.assign(tri_modes(p), 0.0);
  deta.assign(tri_modes(p), 0.0);
  const double a = collapsed(xi, eta);
  const double half = 0.5 * (1.0 - eta);
  const double inv = 1.0 / (1.0 - eta);
  const double da_dxi = 2.0 * inv;
  const double da_deta = (a + 1.0) * inv;
  int k = 0;
  for (int n = 0; n <= p; ++n)
    for (int i = 0; i <= n; ++i, ++k) {
      const int j = n - i;
      const double norm = dubiner_norm(i, n);
      const double pi = jacobi(a, i, 0.0, 0.0);
      const double warp = std::pow(half, static_cast<double>(i));
      const double qj = jacobi(eta, j, 2.0 * i + 1.0, 0.0);
      const double dpi = jacobi_derivative(a, i, 0.0, 0.0);
      const double dqj = jacobi_derivative(eta, j, 2.0 * i + 1.0, 0.0);
      double dwarp = 0.0;
      if (i > 0)
        dwarp = -0.5 * static_cast<double>(i) * std::pow(half, static_cast<double>(i - 1));
      const double dphi_da = norm * dpi * warp * qj;
      const double dphi_db = norm * (pi * dwarp * qj + pi * warp * dqj);
      dxi[k] = dphi_da * da_dxi;
      deta[k] = dphi_da * da_deta + dphi_db;
    }
}

struct Rule1D {
  std::vector<double> x, w;
};

// n-point Gauss-Legendre rule, points ascending.  The node and weight literals
// are the reference's tabulation; the rules must be the same doubles.
inline Rule1D gauss_legendre(int n) {
  struct Half {
    double node, weight;
  };
  static const std::vector<std::vector<Half>> halves = {
      {},
      {{0.0, 2.0}},
      {{0.5773502691896257, 1.0}},
      {{0.0, 0.8888888888888888}, {0.7745966692414834, 0.5555555555555556}},
      {{0.33998104358485626, 0.6521451548625461}, {0.8611363115940526, 0.34785484513745385}},
      {{0.0, 0.5688888888888889},
       {0.5384693101056831, 0.47862867049936647},
       {0.9061798459386640, 0.2369268850561891}},
      {{0.2386191860831969, 0.4679139345726910},
       {0.6612093864662645, 0.3607615730481386},
       {0.9324695142031521, 0.17132449237917036}},
      {{0.0, 0.4179591836734694},
       {0.4058451513773972, 0.3818300505051188},
       {0.7415311855993945, 0.2797053914892766},
       {0.9491079123427585, 0.1294849661688697}},
  };
  if (n < 1 || n > 7)
    throw std::invalid_argument("Gauss-Legendre rules exist for 1..7 points");
  Rule1D r;
  const auto &h = halves[n];
  for (auto it = h.rbegin(); it != h.rend(); ++it)
    if (it->node != 0.0) {
      r.x.push_back(-it->node);
      r.w.push_back(it->weight);
    }
  for (const auto &half : h) {
    r.x.push_back(half.node);
    r.w.push_back(half.weight);
  }
  return r;
}

struct Rule2D {
  std::vector<double> xi, eta, w;
  int size() const { return static_cast<int>(w.size()); }
};

// Collapsed-coordinate tensor rule with (p+1)^2 points on the reference triangle.
inline Rule2D triangle_rule(int p) {
  const Rule1D g = gauss_legendre(p + 1);
  Rule2D r;
  for (std::size_t b = 0; b < g.x.size(); ++b) {
    const double eta = g.x[b];
    const double jac = 0.5 * (1.0 - eta);
    for (std::size_t a = 0; a < g.x.size(); ++a) {
      r.xi.push_back(0.5 * (g.x[a] + 1.0) * (1.0 - eta) - 1.0);
      r.eta.push_back(eta);
      r.w.push_back(g.w[b] * g.w[a] * jac);
    }
  }
  return r;
}

// Fully symmetric rules on the reference triangle, exact for total degree
// `degree` (2: 3 points, 4: 6, 6: 12): orbits of barycentric points
// (a, a, 1-2a) and (a, b, 1-a-b) with their weights, found by Gauss-Newton
// on the moment equations int lambda1^i lambda2^j = i! j! / (i+j+2)! (over a
// triangle of unit area) from approximate published values (Dunavant's rules
// of those degrees; Int. J. Numer. Meth. Eng. 21 (1985) 1129-1148), then
// checked on every monomial up to the degree.  Weights sum to 2, the
// reference triangle's area.
inline Rule2D symmetric_triangle_rule(int degree) {
  // Unknowns: per S21 orbit (a, w), per S111 orbit (a, b, w).
  struct Start {
    std::vector<double> s21, s111;
  };
  Start start;
  if (degree == 2)
    start = {{1.0 / 6.0, 1.0 / 3.0}, {}};
  else if (degree == 4)
    start = {{0.44595, 0.22338, 0.09158, 0.10995}, {}};
  else if (degree == 6)
    start = {{0.24929, 0.11679, 0.06309, 0.05084}, {0.31035, 0.05314, 0.08285}};
  else
    throw std::invalid_argument("symmetric triangle rule: degree 2, 4 or 6");
  std::vector<double> x = start.s21;
  x.insert(x.end(), start.s111.begin(), start.s111.end());
  const std::size_t n21 = start.s21.size() / 2, n111 = start.s111.size() / 3;
  // Barycentric points and weights (unit-area normalization) of the unknowns.
  auto expand = [&](const std::vector<double> &u, std::vector<std::array<double, 3>> &pts,
                    std::vector<double> &ws) {
    pts.clear();
    ws.clear();
    for (std::size_t k = 0; k < n21; ++k) {
      const double a = u[2 * k], w = u[2 * k + 1], b = 1.0 - 2.0 * a;
      for (const auto &pt : {std::array<double, 3>{a, a, b}, {a, b, a}, {b, a, a}}) {
        pts.push_back(pt);
        ws.push_back(w);
      }
    }
    for (std::size_t k = 0; k < n111; ++k) {
      const double a = u[2 * n21 + 3 * k], b = u[2 * n21 + 3 * k + 1];
      const double w = u[2 * n21 + 3 * k + 2], c = 1.0 - a - b;
      for (const auto &pt : {std::array<double, 3>{a, b, c}, {a, c, b}, {b, a, c}, {b, c, a},
                             {c, a, b}, {c, b, a}}) {
        pts.push_back(pt);
        ws.push_back(w);
      }
    }
  };
  auto factorial = [](int k) {
    double f = 1.0;
    for (int i = 2; i <= k; ++i)
      f *= i;
    return f;
  };
  // Residuals of the moment equations (unit-area triangle: integral x 2).
  auto residual = [&](const std::vector<double> &u) {
    std::vector<std::array<double, 3>> pts;
    std::vector<double> ws;
    expand(u, pts, ws);
    std::vector<double> r;
    for (int i = 0; i <= degree; ++i)
      for (int j = 0; i + j <= degree; ++j) {
        double sum = 0.0;
        for (std::size_t q = 0; q < pts.size(); ++q)
          sum += ws[q] * std::pow(pts[q][0], i) * std::pow(pts[q][1], j);
        r.push_back(sum - 2.0 * factorial(i) * factorial(j) / factorial(i + j + 2));
      }
    return r;
  };
  const std::size_t nu = x.size();
  for (int iteration = 0; iteration < 50; ++iteration) {
    const std::vector<double> r = residual(x);
    // Normal equations J^T J dx = -J^T r with a central-difference Jacobian.
    std::vector<std::vector<double>> J(r.size(), std::vector<double>(nu));
    for (std::size_t k = 0; k < nu; ++k) {
      std::vector<double> hi = x, lo = x;
      const double h = 1e-7;
      hi[k] += h;
      lo[k] -= h;
      const auto rh = residual(hi), rl = residual(lo);
      for (std::size_t e = 0; e < r.size(); ++e)
        J[e][k] = (rh[e] - rl[e]) / (2.0 * h);
    }
    std::vector<std::vector<double>> A(nu, std::vector<double>(nu + 1, 0.0));
    for (std::size_t a = 0; a < nu; ++a) {
      for (std::size_t b = 0; b < nu; ++b)
        for (std::size_t e = 0; e < r.size(); ++e)
          A[a][b] += J[e][a] * J[e][b];
      for (std::size_t e = 0; e < r.size(); ++e)
        A[a][nu] -= J[e][a] * r[e];
    }
    for (std::size_t c = 0; c < nu; ++c) { // Gaussian elimination, partial pivoting
      std::size_t best = c;
      for (std::size_t k = c + 1; k < nu; ++k)
        if (std::fabs(A[k][c]) > std::fabs(A[best][c]))
          best = k;
      std::swap(A[c], A[best]);
      for (std::size_t k = 0; k < nu; ++k)
        if (k != c) {
          const double f = A[k][c] / A[c][c];
          for (std::size_t m = c; m <= nu; ++m)
            A[k][m] -= f * A[c][m];
        }
    }
    double step = 0.0;
    for (std::size_t k = 0; k < nu; ++k) {
      x[k] += A[k][nu] / A[k][k];
      step = std::max(step, std::fabs(A[k][nu] / A[k][k]));
    }
    if (step < 1e-15)
      break;
  }
  for (const double e : residual(x))
    if (std::fabs(e) > 1e-13)
      throw std::runtime_error("symmetric triangle rule: moment equations not solved");
  std::vector<std::array<double, 3>> pts;
  std::vector<double> ws;
  expand(x, pts, ws);
  Rule2D r;
  for (std::size_t q = 0; q < pts.size(); ++q) {
    // Reference triangle (-1,-1), (1,-1), (-1,1): x = -l0 + l1 - l2, etc.
    r.xi.push_back(-1.0 + 2.0 * pts[q][1]);
    r.eta.push_back(-1.0 + 2.0 * pts[q][2]);
    r.w.push_back(2.0 * ws[q]);
  }
  return r;
}

// p+1 Gauss points on each reference edge (0: v0->v1, 1: v1->v2, 2: v2->v0),
// packed [edge][point]; weights scaled by the reference edge length.
inline Rule2D triangle_edges(int p) {
  const Rule1D g = gauss_legendre(p + 1);
  const double inv_sqrt2 = 1.0 / std::sqrt(2.0);
  Rule2D r;
  r.xi.resize(3 * g.x.size());
  r.eta.resize(3 * g.x.size());
  r.w.resize(3 * g.x.size());
  const std::size_t n = g.x.size();
  for (std::size_t q = 0; q < n; ++q) {
    const double s = g.x[q], w = g.w[q];
    r.xi[q] = s;
    r.eta[q] = -1.0;
    r.w[q] = w;
    r.xi[n + q] = 1.0 + 0.5 * (s + 1.0) * (-2.0);
    r.eta[n + q] = -1.0 + 0.5 * (s + 1.0) * (2.0);
    r.w[n + q] = w * 2.0 * inv_sqrt2;
    r.xi[2 * n + q] = -1.0;
    r.eta[2 * n + q] = s;
    r.w[2 * n + q] = w;
  }
  return r;
}

// Reference point of the right element matching a left-element edge point:
// reduce to the edge parameter along the left traversal, reverse it when the
// two sides traverse the edge in opposite directions, place it on the right
// local edge (cpp/include/wasl/dg/triangle_face_trace.hpp:16-33).
inline void neighbour_point(int left_edge, int right_edge, bool flip, double lxi, double leta,
                            double &rxi, double &reta) {
  double t = left_edge == 0 ? lxi : left_edge == 1 ? leta : -leta;
  if (flip)
    t = -t;
  rxi = -1.0;
  reta = -1.0;
  if (right_edge == 0) {
    rxi = t;
  } else if (right_edge == 1) {
    rxi = -t;
    reta = t;
  } else {
    reta = -t;
  }
}

} // namespace wasl_b200
