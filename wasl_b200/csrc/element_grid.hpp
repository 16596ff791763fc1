// The uniform bucket grid of the periodic donor search, shared by the host
// search (mesh.cpp) and the device search (setup_device.cu) so that both bin
// every element and every point into the same cells with the same arithmetic.
//
// The grid has floor(sqrt(elements / 2)) cells per side over the mesh's
// bounding box; an element covers the cells its bounding box, padded by 1e-6
// of its extent, overlaps, so an element that passes the 1e-10
// reference-coordinate containment test of its point is always one of the
// candidates of the point's cell.
#pragma once

#include <cmath>

#ifndef WASL_HD
#if defined(__CUDACC__)
#define WASL_HD __host__ __device__ __forceinline__
#else
#define WASL_HD inline
#endif
#endif

namespace wasl_b200 {

struct GridShape {
  double x0, y0, dx, dy;
  int nx, ny;
};

WASL_HD int grid_clamp(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

WASL_HD int grid_cell(const GridShape &g, double x, double y) {
  const int i = grid_clamp(static_cast<int>(std::floor((x - g.x0) / g.dx)), g.nx);
  const int j = grid_clamp(static_cast<int>(std::floor((y - g.y0) / g.dy)), g.ny);
  return j * g.nx + i;
}

// The cells [i0, i1] x [j0, j1] a triangle's padded bounding box covers.
WASL_HD void grid_cell_range(const GridShape &g, const double *v, int &i0, int &i1, int &j0,
                             int &j1) {
  const double lx = fmin(v[0], fmin(v[2], v[4])), hx = fmax(v[0], fmax(v[2], v[4]));
  const double ly = fmin(v[1], fmin(v[3], v[5])), hy = fmax(v[1], fmax(v[3], v[5]));
  const double pad = 1e-6 * ((hx - lx) + (hy - ly));
  i0 = grid_clamp(static_cast<int>(std::floor((lx - pad - g.x0) / g.dx)), g.nx);
  i1 = grid_clamp(static_cast<int>(std::floor((hx + pad - g.x0) / g.dx)), g.nx);
  j0 = grid_clamp(static_cast<int>(std::floor((ly - pad - g.y0) / g.dy)), g.ny);
  j1 = grid_clamp(static_cast<int>(std::floor((hy + pad - g.y0) / g.dy)), g.ny);
}

// Reference coordinates of (x, y) in the triangle v = (x0, y0, x1, y1, x2,
// y2): TriMap::to_reference's arithmetic (mesh.cpp), in the same order.
WASL_HD void grid_to_reference(const double *v, double x, double y, double &xi, double &eta) {
  const double ax = v[2] - v[0], ay = v[3] - v[1], bx = v[4] - v[0], by = v[5] - v[1];
  const double dx = x - v[0];
  const double dy = y - v[1];
  const double inverse_det = 1.0 / (ax * by - bx * ay);
  const double s = (by * dx - bx * dy) * inverse_det;
  const double t = (-ay * dx + ax * dy) * inverse_det;
  xi = 2.0 * s - 1.0;
  eta = 2.0 * t - 1.0;
}

// The donor search's containment test (tolerance 1e-10 in reference
// coordinates).
WASL_HD bool grid_contains(double xi, double eta) {
  constexpr double tolerance = 1e-10;
  return xi >= -1.0 - tolerance && eta >= -1.0 - tolerance && xi + eta <= tolerance;
}

} // namespace wasl_b200
