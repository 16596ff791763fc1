#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <thread>
#include <unordered_map>

#include "basis.hpp"

namespace wasl_b200 {

// ---- affine triangle map (cpp/include/wasl/mesh/triangle/triangle_geometry.hpp) ----

void TriMap::to_physical(double xi, double eta, double &x, double &y) const {
  x = x0 + 0.5 * (ax() * (xi + 1.0) + bx() * (eta + 1.0));
  y = y0 + 0.5 * (ay() * (xi + 1.0) + by() * (eta + 1.0));
}

void TriMap::to_reference(double x, double y, double &xi, double &eta) const {
  const double dx = x - x0;
  const double dy = y - y0;
  const double inverse_det = 1.0 / det_a();
  const double s = (by() * dx - bx() * dy) * inverse_det;
  const double t = (-ay() * dx + ax() * dy) * inverse_det;
  xi = 2.0 * s - 1.0;
  eta = 2.0 * t - 1.0;
}

void TriMap::edge_vector(int edge, double &ex, double &ey) const {
  if (edge == 0) {
    ex = x1 - x0;
    ey = y1 - y0;
  } else if (edge == 1) {
    ex = x2 - x1;
    ey = y2 - y1;
  } else {
    ex = x0 - x2;
    ey = y0 - y2;
  }
}

double TriMap::edge_length(int edge) const {
  double ex = 0.0, ey = 0.0;
  edge_vector(edge, ex, ey);
  return std::hypot(ex, ey);
}

void TriMap::edge_normal(int edge, double &nx, double &ny) const {
  double ex = 0.0, ey = 0.0;
  edge_vector(edge, ex, ey);
  const double length = std::hypot(ex, ey);
  const double tx = ex / length;
  const double ty = ey / length;
  const int sign = orientation();
  nx = sign * ty;
  ny = sign * (-tx);
}

void TriMap::shift(double ox, double oy) {
  x0 += ox;
  x1 += ox;
  x2 += ox;
  y0 += oy;
  y1 += oy;
  y2 += oy;
}

namespace {

constexpr int edge_vertices[3][2] = {{0, 1}, {1, 2}, {2, 0}};

std::unordered_map<std::int64_t, std::int64_t> node_index(std::int64_t count,
                                                          const std::int64_t *tags,
                                                          const char *context) {
  std::unordered_map<std::int64_t, std::int64_t> index;
  index.reserve(static_cast<std::size_t>(count) * 2);
  for (std::int64_t i = 0; i < count; ++i)
    if (!index.emplace(tags[i], i).second)
      throw std::runtime_error(std::string(context) + ": duplicate node tag " +
                               std::to_string(tags[i]));
  return index;
}

double reference_edge_length(int edge) { return edge == 1 ? 2.0 * std::sqrt(2.0) : 2.0; }

} // namespace

TriTopology build_triangle_topology(std::int64_t node_count, const std::int64_t *node_tags,
                                    const double *node_xy, std::int64_t element_count,
                                    const std::int64_t *element_nodes) {
  if (element_count <= 0)
    throw std::runtime_error("triangle mesh: document contains no triangle elements");
  if (element_count > std::numeric_limits<std::int32_t>::max())
    throw std::runtime_error("triangle mesh: more elements than 32-bit indices address");
  const auto index = node_index(node_count, node_tags, "triangle mesh");
  TriTopology mesh;
  mesh.element_count = element_count;
  mesh.maps.resize(element_count);
  mesh.nodes.resize(3 * element_count);
  for (std::int64_t e = 0; e < element_count; ++e) {
    std::int64_t tag[3];
    double x[3], y[3];
    for (int k = 0; k < 3; ++k) {
      tag[k] = element_nodes[3 * e + k];
      const auto found = index.find(tag[k]);
      if (found == index.end())
        throw std::runtime_error("triangle mesh: element references missing node " +
                                 std::to_string(tag[k]));
      x[k] = node_xy[2 * found->second];
      y[k] = node_xy[2 * found->second + 1];
    }
    const double area2 = x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]);
    if (area2 == 0.0)
      throw std::runtime_error("triangle mesh: zero-area element " + std::to_string(e + 1));
    if (area2 < 0.0) {
      std::swap(x[1], x[2]);
      std::swap(y[1], y[2]);
      std::swap(tag[1], tag[2]);
    }
    mesh.maps[e] = TriMap{x[0], y[0], x[1], y[1], x[2], y[2]};
    for (int k = 0; k < 3; ++k)
      mesh.nodes[3 * e + k] = tag[k];
  }

  // Each element edge keyed by its sorted vertex pair; a stable sort keeps the
  // element order inside a key, so the first entry is the first element to
  // reach the edge.
  struct Side {
    std::int64_t lo, hi, v0;
    std::int32_t element;
    std::int32_t edge;
  };
  std::vector<Side> sides(3 * element_count);
  for (std::int64_t e = 0; e < element_count; ++e)
    for (int k = 0; k < 3; ++k) {
      const std::int64_t a = mesh.nodes[3 * e + edge_vertices[k][0]];
      const std::int64_t b = mesh.nodes[3 * e + edge_vertices[k][1]];
      sides[3 * e + k] = {std::min(a, b), std::max(a, b), a, static_cast<std::int32_t>(e), k};
    }
  std::stable_sort(sides.begin(), sides.end(), [](const Side &a, const Side &b) {
    return a.lo != b.lo ? a.lo < b.lo : a.hi < b.hi;
  });

  struct Face {
    std::int32_t left, right, le, re;
    std::uint8_t flip;
  };
  std::vector<Face> faces;
  faces.reserve(sides.size() / 2 + 64);
  for (std::size_t i = 0; i < sides.size();) {
    std::size_t j = i + 1;
    while (j < sides.size() && sides[j].lo == sides[i].lo && sides[j].hi == sides[i].hi)
      ++j;
    if (j - i > 2)
      throw std::runtime_error("triangle mesh: edge " + std::to_string(sides[i].lo) + "-" +
                               std::to_string(sides[i].hi) +
                               " has more than two adjacent elements (non-conforming mesh)");
    if (j - i == 2)
      faces.push_back({sides[i].element, sides[i + 1].element, sides[i].edge, sides[i + 1].edge,
                       static_cast<std::uint8_t>(sides[i].v0 != sides[i + 1].v0)});
    else
      faces.push_back({sides[i].element, -1, sides[i].edge, 0, 0});
    i = j;
  }
  std::sort(faces.begin(), faces.end(), [](const Face &a, const Face &b) {
    return a.left != b.left ? a.left < b.left : a.le < b.le;
  });

  const std::size_t nf = faces.size();
  mesh.face_left.resize(nf);
  mesh.face_right.resize(nf);
  mesh.face_left_edge.resize(nf);
  mesh.face_right_edge.resize(nf);
  mesh.face_flip.resize(nf);
  mesh.face_nx.resize(nf);
  mesh.face_ny.resize(nf);
  mesh.face_scale.resize(nf);
  for (std::size_t f = 0; f < nf; ++f) {
    const Face &face = faces[f];
    mesh.face_left[f] = face.left;
    mesh.face_right[f] = face.right;
    mesh.face_left_edge[f] = face.le;
    mesh.face_right_edge[f] = face.re;
    mesh.face_flip[f] = face.flip;
    const TriMap &m = mesh.maps[face.left];
    m.edge_normal(face.le, mesh.face_nx[f], mesh.face_ny[f]);
    mesh.face_scale[f] = m.edge_length(face.le) / reference_edge_length(face.le);
  }
  return mesh;
}

LineTopology build_line_topology(std::int64_t node_count, const std::int64_t *node_tags,
                                 const double *node_x, std::int64_t element_count,
                                 const std::int64_t *element_nodes) {
  if (element_count <= 0)
    throw std::runtime_error("line mesh: document contains no line elements");
  const auto index = node_index(node_count, node_tags, "line mesh");
  struct Segment {
    std::int64_t left_node, right_node;
    double xl, xr;
  };
  std::vector<Segment> segs(element_count);
  for (std::int64_t e = 0; e < element_count; ++e) {
    const auto a = index.find(element_nodes[2 * e]);
    const auto b = index.find(element_nodes[2 * e + 1]);
    if (a == index.end() || b == index.end())
      throw std::runtime_error("line mesh: element references missing node");
    const double xa = node_x[a->second], xb = node_x[b->second];
    if (xa == xb)
      throw std::runtime_error("line mesh: zero-length element " + std::to_string(e + 1));
    segs[e] = xa < xb ? Segment{a->first, b->first, xa, xb} : Segment{b->first, a->first, xb, xa};
  }
  std::stable_sort(segs.begin(), segs.end(),
                   [](const Segment &a, const Segment &b) { return a.xl < b.xl; });
  LineTopology mesh;
  mesh.element_count = element_count;
  for (std::int64_t e = 0; e < element_count; ++e) {
    if (e + 1 < element_count && segs[e].right_node != segs[e + 1].left_node)
      throw std::runtime_error("line mesh: gap or discontinuity between elements " +
                               std::to_string(e) + " and " + std::to_string(e + 1));
    mesh.x_left.push_back(segs[e].xl);
    mesh.x_right.push_back(segs[e].xr);
  }
  mesh.face_left.push_back(0);
  mesh.face_right.push_back(-1);
  mesh.face_normal.push_back(-1.0);
  for (std::int64_t e = 0; e + 1 < element_count; ++e) {
    mesh.face_left.push_back(static_cast<std::int32_t>(e));
    mesh.face_right.push_back(static_cast<std::int32_t>(e + 1));
    mesh.face_normal.push_back(1.0);
  }
  mesh.face_left.push_back(static_cast<std::int32_t>(element_count - 1));
  mesh.face_right.push_back(-1);
  mesh.face_normal.push_back(1.0);
  return mesh;
}

namespace {

struct Box {
  double min_x = std::numeric_limits<double>::max();
  double max_x = std::numeric_limits<double>::lowest();
  double min_y = std::numeric_limits<double>::max();
  double max_y = std::numeric_limits<double>::lowest();
};

Box bounding_box(const TriTopology &mesh) {
  Box b;
  for (const auto &m : mesh.maps) {
    b.min_x = std::min({b.min_x, m.x0, m.x1, m.x2});
    b.max_x = std::max({b.max_x, m.x0, m.x1, m.x2});
    b.min_y = std::min({b.min_y, m.y0, m.y1, m.y2});
    b.max_y = std::max({b.max_y, m.y0, m.y1, m.y2});
  }
  return b;
}

// Uniform bucket grid over element bounding boxes, padded so that any element
// passing the 1e-10 reference-coordinate containment test is a candidate.
class ElementGrid {
public:
  explicit ElementGrid(const TriTopology &mesh) : mesh_(mesh) {
    const Box box = bounding_box(mesh);
    x0_ = box.min_x;
    y0_ = box.min_y;
    const double n = std::max(1.0, std::sqrt(static_cast<double>(mesh.element_count) / 2.0));
    nx_ = ny_ = static_cast<int>(n);
    dx_ = std::max((box.max_x - box.min_x) / nx_, 1e-300);
    dy_ = std::max((box.max_y - box.min_y) / ny_, 1e-300);
    start_.assign(static_cast<std::size_t>(nx_) * ny_ + 1, 0);
    std::vector<std::pair<int, std::int32_t>> entries;
    for (std::int64_t e = 0; e < mesh.element_count; ++e) {
      int i0, i1, j0, j1;
      cells(e, i0, i1, j0, j1);
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i)
          entries.emplace_back(j * nx_ + i, static_cast<std::int32_t>(e));
    }
    std::stable_sort(entries.begin(), entries.end(),
                     [](const auto &a, const auto &b) { return a.first < b.first; });
    items_.resize(entries.size());
    for (std::size_t k = 0; k < entries.size(); ++k) {
      items_[k] = entries[k].second;
      ++start_[entries[k].first + 1];
    }
    for (std::size_t c = 1; c < start_.size(); ++c)
      start_[c] += start_[c - 1];
  }

  // The first element, by index, containing (x, y) within the tolerance.
  std::int32_t find(double x, double y, double &xi, double &eta) const {
    constexpr double tolerance = 1e-10;
    const int i = clamp_cell(static_cast<int>(std::floor((x - x0_) / dx_)), nx_);
    const int j = clamp_cell(static_cast<int>(std::floor((y - y0_) / dy_)), ny_);
    const std::size_t c = static_cast<std::size_t>(j) * nx_ + i;
    for (std::size_t k = start_[c]; k < start_[c + 1]; ++k) { // ascending element index
      const std::int32_t e = items_[k];
      mesh_.maps[e].to_reference(x, y, xi, eta);
      if (xi >= -1.0 - tolerance && eta >= -1.0 - tolerance && xi + eta <= tolerance)
        return e;
    }
    return -1;
  }

private:
  static int clamp_cell(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

  void cells(std::int64_t e, int &i0, int &i1, int &j0, int &j1) const {
    const TriMap &m = mesh_.maps[e];
    const double lx = std::min({m.x0, m.x1, m.x2}), hx = std::max({m.x0, m.x1, m.x2});
    const double ly = std::min({m.y0, m.y1, m.y2}), hy = std::max({m.y0, m.y1, m.y2});
    const double pad = 1e-6 * ((hx - lx) + (hy - ly));
    i0 = clamp_cell(static_cast<int>(std::floor((lx - pad - x0_) / dx_)), nx_);
    i1 = clamp_cell(static_cast<int>(std::floor((hx + pad - x0_) / dx_)), nx_);
    j0 = clamp_cell(static_cast<int>(std::floor((ly - pad - y0_) / dy_)), ny_);
    j1 = clamp_cell(static_cast<int>(std::floor((hy + pad - y0_) / dy_)), ny_);
  }

  const TriTopology &mesh_;
  double x0_, y0_, dx_, dy_;
  int nx_, ny_;
  std::vector<std::size_t> start_;
  std::vector<std::int32_t> items_;
};

template <typename F> void parallel_for(std::int64_t n, F &&body) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const std::int64_t workers = std::min<std::int64_t>(hw, std::max<std::int64_t>(1, n / 256));
  if (workers <= 1) {
    body(0, n);
    return;
  }
  std::vector<std::thread> pool;
  for (std::int64_t w = 0; w < workers; ++w)
    pool.emplace_back([&, w] { body(n * w / workers, n * (w + 1) / workers); });
  for (auto &t : pool)
    t.join();
}

} // namespace

PeriodicTrace periodic_trace(const TriTopology &mesh, int p) {
  const int Q = p + 1, M = tri_modes(p);
  const Rule2D edges = triangle_edges(p);
  const Box box = bounding_box(mesh);
  const std::int64_t nf = mesh.face_count();
  PeriodicTrace trace;
  trace.donors.assign(nf * Q, -1);
  trace.basis.assign(nf * Q * M, 0.0);
  const ElementGrid grid(mesh);
  for (std::int64_t f = 0; f < nf; ++f) {
    if (mesh.face_right[f] >= 0)
      continue;
    const TriMap &m = mesh.maps[mesh.face_left[f]];
    const int le = mesh.face_left_edge[f];
    const double nx = mesh.face_nx[f], ny = mesh.face_ny[f];
    for (int q = 0; q < Q; ++q) {
      double x = 0.0, y = 0.0;
      m.to_physical(edges.xi[le * Q + q], edges.eta[le * Q + q], x, y);
      if (std::fabs(nx) > 0.5 && std::fabs(ny) < 1e-10)
        x += nx < 0.0 ? box.max_x - box.min_x : box.min_x - box.max_x;
      else if (std::fabs(ny) > 0.5 && std::fabs(nx) < 1e-10)
        y += ny < 0.0 ? box.max_y - box.min_y : box.min_y - box.max_y;
      else
        throw std::runtime_error("simulation: 2D periodic boundaries require an axis-aligned box");
      double xi = 0.0, eta = 0.0;
      const std::int32_t donor = grid.find(x, y, xi, eta);
      if (donor < 0)
        throw std::runtime_error("simulation: periodic 2D trace has no donor element");
      trace.donors[f * Q + q] = donor;
      const auto b = dubiner(xi, eta, p);
      std::copy(b.begin(), b.end(), trace.basis.begin() + (f * Q + q) * M);
    }
  }
  return trace;
}

namespace {

// Record a neighbour once, in the first free slot (limiter_stencil_assembly.hpp:27-40).
void add_neighbor(LimiterStencil &s, std::int64_t element, std::int32_t neighbor) {
  std::int32_t *slot = s.neighbors.data() + element * s.maximum_neighbors;
  for (int k = 0; k < s.maximum_neighbors; ++k) {
    if (slot[k] == neighbor)
      return;
    if (slot[k] == -1) {
      slot[k] = neighbor;
      return;
    }
  }
}

double period_shift(double gap, double period) {
  return gap > 0.5 * period ? period : gap < -0.5 * period ? -period : 0.0;
}

} // namespace

LimiterStencil triangle_stencil(const TriTopology &mesh, int p,
                                const std::vector<std::int32_t> &periodic_donors) {
  const std::int64_t ne = mesh.element_count;
  const int M = tri_modes(p), Q = p + 1;
  LimiterStencil s;
  s.mode_count = M;
  s.maximum_neighbors = 3;
  s.highest_degree_begin = p > 0 ? tri_modes(p - 1) : M;
  s.neighbors.assign(ne * 3, -1);
  s.normal_x.assign(ne, 1.0);
  s.normal_y.assign(ne, 0.0);
  std::vector<std::uint8_t> has_normal(ne, 0);
  // Each element's characteristic direction is the first face giving it a
  // neighbour, outward from it (euler_limiter_stencil_triangle.cpp:16-44).
  for (std::int64_t f = 0; f < mesh.face_count(); ++f) {
    const std::int32_t left = mesh.face_left[f];
    std::int32_t right = mesh.face_right[f];
    const bool boundary = right < 0;
    if (boundary && !periodic_donors.empty())
      right = periodic_donors[f * Q];
    if (right < 0)
      continue;
    add_neighbor(s, left, right);
    if (!has_normal[left]) {
      s.normal_x[left] = mesh.face_nx[f];
      s.normal_y[left] = mesh.face_ny[f];
      has_normal[left] = 1;
    }
    if (!boundary) {
      add_neighbor(s, right, left);
      if (!has_normal[right]) {
        s.normal_x[right] = -mesh.face_nx[f];
        s.normal_y[right] = -mesh.face_ny[f];
        has_normal[right] = 1;
      }
    }
  }

  // transform[t][s]: L2 projection of neighbour mode s onto target mode t over
  // the target element, the neighbour shifted by a period when its centroid
  // lies more than half a period away (candidate_transform.hpp:18-39,
  // euler_limiter_stencil_triangle.cpp:51-79).
  const Box box = bounding_box(mesh);
  const double width = box.max_x - box.min_x, height = box.max_y - box.min_y;
  const Rule2D rule = triangle_rule(p);
  std::vector<std::vector<double>> target_basis(rule.size());
  for (int q = 0; q < rule.size(); ++q)
    target_basis[q] = dubiner(rule.xi[q], rule.eta[q], p);
  s.transforms.assign(static_cast<std::size_t>(ne) * 3 * M * M, 0.0);
  parallel_for(ne, [&](std::int64_t begin, std::int64_t end) {
    std::vector<std::vector<double>> source_basis(rule.size());
    for (std::int64_t e = begin; e < end; ++e) {
      const TriMap &target = mesh.maps[e];
      for (int k = 0; k < 3; ++k) {
        const std::int32_t nb = s.neighbors[e * 3 + k];
        if (nb < 0)
          continue;
        TriMap source = mesh.maps[nb];
        source.shift(
            period_shift((target.x0 + target.x1 + target.x2 - source.x0 - source.x1 - source.x2) /
                             3.0,
                         width),
            period_shift((target.y0 + target.y1 + target.y2 - source.y0 - source.y1 - source.y2) /
                             3.0,
                         height));
        for (int q = 0; q < rule.size(); ++q) {
          double x = 0.0, y = 0.0, sxi = 0.0, seta = 0.0;
          target.to_physical(rule.xi[q], rule.eta[q], x, y);
          source.to_reference(x, y, sxi, seta);
          source_basis[q] = dubiner(sxi, seta, p);
        }
        double *matrix = s.transforms.data() + (e * 3 + k) * M * M;
        for (int sm = 0; sm < M; ++sm) {
          // modal_sum of the unit coefficient vector e_sm, kept literal so the
          // rounding (and signed zeros) match the reference.
          std::vector<double> column(M, 0.0);
          for (int q = 0; q < rule.size(); ++q) {
            double value = 0.0;
            for (int m = 0; m < M; ++m)
              value += (m == sm ? 1.0 : 0.0) * source_basis[q][m];
            for (int t = 0; t < M; ++t)
              column[t] += rule.w[q] * value * target_basis[q][t];
          }
          for (int t = 0; t < M; ++t)
            matrix[t * M + sm] = column[t];
        }
      }
    }
  });

  // Check points: volume rule of order p, then the three edge rules
  // (euler_limiter_stencil_triangle.cpp:81-93).
  const Rule2D edges = triangle_edges(p);
  for (int q = 0; q < rule.size(); ++q) {
    const auto b = dubiner(rule.xi[q], rule.eta[q], p);
    s.check_basis.insert(s.check_basis.end(), b.begin(), b.end());
  }
  for (int q = 0; q < edges.size(); ++q) {
    const auto b = dubiner(edges.xi[q], edges.eta[q], p);
    s.check_basis.insert(s.check_basis.end(), b.begin(), b.end());
  }
  return s;
}

LimiterStencil line_stencil(const LineTopology &mesh, int p, bool periodic) {
  const std::int64_t ne = mesh.element_count;
  const int M = line_modes(p);
  LimiterStencil s;
  s.mode_count = M;
  s.maximum_neighbors = 2;
  s.highest_degree_begin = p > 0 ? M - 1 : M;
  s.neighbors.assign(ne * 2, -1);
  s.normal_x.assign(ne, 1.0);
  s.normal_y.assign(ne, 0.0);
  std::int32_t left_end = -1, right_end = -1;
  for (std::int64_t f = 0; f < mesh.face_count(); ++f) {
    if (mesh.face_right[f] >= 0) {
      add_neighbor(s, mesh.face_left[f], mesh.face_right[f]);
      add_neighbor(s, mesh.face_right[f], mesh.face_left[f]);
    } else if (mesh.face_normal[f] < 0.0) {
      left_end = mesh.face_left[f];
    } else {
      right_end = mesh.face_left[f];
    }
  }
  if (periodic && left_end >= 0 && right_end >= 0) {
    add_neighbor(s, left_end, right_end);
    add_neighbor(s, right_end, left_end);
  }
  const Rule1D rule = gauss_legendre(std::max(1, p + 1));
  const double period = mesh.x_right[ne - 1] - mesh.x_left[0];
  s.transforms.assign(static_cast<std::size_t>(ne) * 2 * M * M, 0.0);
  for (std::int64_t e = 0; e < ne; ++e) {
    const double txl = mesh.x_left[e], txr = mesh.x_right[e];
    for (int k = 0; k < 2; ++k) {
      const std::int32_t nb = s.neighbors[e * 2 + k];
      if (nb < 0)
        continue;
      double sxl = mesh.x_left[nb], sxr = mesh.x_right[nb];
      const double offset = period_shift((txl + txr) / 2.0 - (sxl + sxr) / 2.0, period);
      sxl += offset;
      sxr += offset;
      double *matrix = s.transforms.data() + (e * 2 + k) * M * M;
      for (std::size_t q = 0; q < rule.x.size(); ++q) {
        const double x = (txl + txr) / 2.0 + (txr - txl) / 2.0 * rule.x[q];
        const double sxi = (x - (sxl + sxr) / 2.0) / ((sxr - sxl) / 2.0);
        const auto sb = legendre(sxi, p);
        const auto tb = legendre(rule.x[q], p);
        for (int t = 0; t < M; ++t)
          for (int sm = 0; sm < M; ++sm)
            matrix[t * M + sm] += rule.w[q] * tb[t] * sb[sm];
      }
    }
  }
  for (double x : rule.x) {
    const auto b = legendre(x, p);
    s.check_basis.insert(s.check_basis.end(), b.begin(), b.end());
  }
  for (double x : {-1.0, 1.0}) {
    const auto b = legendre(x, p);
    s.check_basis.insert(s.check_basis.end(), b.begin(), b.end());
  }
  return s;
}

TriSlots build_tri_slots(const TriTopology &mesh, const PeriodicTrace *trace, int QF, int M) {
  const std::int64_t ne = mesh.element_count, nf = mesh.face_count();
  TriSlots t;
  t.geo.resize(5 * ne);
  for (std::int64_t e = 0; e < ne; ++e) {
    const TriMap &m = mesh.maps[e];
    t.geo[e] = m.ax();
    t.geo[ne + e] = m.ay();
    t.geo[2 * ne + e] = m.bx();
    t.geo[3 * ne + e] = m.by();
    t.geo[4 * ne + e] = 1.0 / m.jacobian_determinant();
  }
  t.slot_nbr.resize(3 * ne);
  t.slot_code.resize(3 * ne);
  t.slot_geo.resize(9 * ne);
  t.slot_face.resize(3 * ne);
  t.face_right.resize(nf);
  t.left_slot.assign(nf, 0);
  t.face_code.resize(nf);
  t.face_normal.resize(2 * nf);
  std::vector<int> fill(ne, 0);
  std::vector<double> bny;
  for (std::int64_t f = 0; f < nf; ++f) {
    const std::int32_t L = mesh.face_left[f], R = mesh.face_right[f];
    const unsigned le = mesh.face_left_edge[f], re = mesh.face_right_edge[f];
    const unsigned shared = (le << 1) | (re << 3) | (static_cast<unsigned>(mesh.face_flip[f]) << 5);
    std::int32_t right = R;
    if (R < 0) {
      right = -static_cast<std::int32_t>(t.boundary_count + 1);
      t.bnd_element.push_back(L);
      t.bnd_edge.push_back(static_cast<std::uint8_t>(le));
      t.bnd_normal.push_back(mesh.face_nx[f]);
      bny.push_back(mesh.face_ny[f]);
      if (trace)
        for (int q = 0; q < QF; ++q) {
          t.donors.push_back(trace->donors[f * QF + q]);
          t.donor_basis.insert(t.donor_basis.end(), trace->basis.begin() + (f * QF + q) * M,
                               trace->basis.begin() + (f * QF + q + 1) * M);
        }
      ++t.boundary_count;
    }
    t.face_right[f] = right;
    t.face_code[f] = static_cast<std::uint8_t>(shared | 1u);
    t.face_normal[f] = mesh.face_nx[f];
    t.face_normal[nf + f] = mesh.face_ny[f];
    t.left_slot[f] = fill[L];
    auto put = [&](std::int32_t e, std::int32_t other, unsigned code) {
      const int k = fill[e]++;
      if (k >= 3)
        throw std::runtime_error("triangle mesh: element with more than three faces");
      t.slot_face[k * ne + e] = static_cast<std::int32_t>(f);
      t.slot_nbr[k * ne + e] = other;
      t.slot_code[k * ne + e] = static_cast<std::uint8_t>(code);
      t.slot_geo[(3 * k) * ne + e] = mesh.face_nx[f];
      t.slot_geo[(3 * k + 1) * ne + e] = mesh.face_ny[f];
      t.slot_geo[(3 * k + 2) * ne + e] = mesh.face_scale[f];
    };
    put(L, right, shared | 1u);
    if (R >= 0)
      put(R, L, shared);
  }
  for (std::int64_t e = 0; e < ne; ++e)
    if (fill[e] != 3)
      throw std::runtime_error("triangle mesh: element without three faces");
  t.bnd_normal.insert(t.bnd_normal.end(), bny.begin(), bny.end());
  return t;
}

double minimum_altitude(const TriTopology &mesh) {
  double result = std::numeric_limits<double>::max();
  for (const auto &m : mesh.maps) {
    const double longest = std::max({m.edge_length(0), m.edge_length(1), m.edge_length(2)});
    result = std::min(result, 4.0 * m.jacobian_determinant() / longest);
  }
  return result;
}

double minimum_length(const LineTopology &mesh) {
  double result = std::numeric_limits<double>::max();
  for (std::int64_t e = 0; e < mesh.element_count; ++e)
    result = std::min(result, mesh.x_right[e] - mesh.x_left[e]);
  return result;
}

} // namespace wasl_b200
