#include "mesh.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <unordered_map>

#include "basis.hpp"
#include "parallel.hpp"

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

// Position of every node tag: a direct table when the tags are dense (the
// usual 1..N numbering), a hash map otherwise.  Throws on the first
// duplicate tag in input order.
class NodeIndex {
public:
  NodeIndex(std::int64_t count, const std::int64_t *tags, const char *context) {
    std::int64_t lo = std::numeric_limits<std::int64_t>::max(), hi = std::numeric_limits<std::int64_t>::min();
    for (std::int64_t i = 0; i < count; ++i)
      lo = std::min(lo, tags[i]), hi = std::max(hi, tags[i]);
    dense_ = count > 0 && hi - lo < 4 * count + 1024;
    if (dense_) {
      base_ = lo;
      table_.assign(static_cast<std::size_t>(hi - lo + 1), -1);
    } else {
      map_.reserve(static_cast<std::size_t>(count) * 2);
    }
    for (std::int64_t i = 0; i < count; ++i) {
      const bool fresh = dense_ ? table_[tags[i] - base_] < 0 : map_.emplace(tags[i], i).second;
      if (!fresh)
        throw std::runtime_error(std::string(context) + ": duplicate node tag " +
                                 std::to_string(tags[i]));
      if (dense_)
        table_[tags[i] - base_] = i;
    }
  }
  // -1 when the tag is not a node.
  std::int64_t find(std::int64_t tag) const {
    if (dense_) {
      if (tag < base_ || tag - base_ >= static_cast<std::int64_t>(table_.size()))
        return -1;
      return table_[tag - base_];
    }
    const auto it = map_.find(tag);
    return it == map_.end() ? -1 : it->second;
  }

private:
  bool dense_ = false;
  std::int64_t base_ = 0;
  std::vector<std::int64_t> table_;
  std::unordered_map<std::int64_t, std::int64_t> map_;
};

double reference_edge_length(int edge) { return edge == 1 ? 2.0 * std::sqrt(2.0) : 2.0; }

} // namespace

TriTopology build_triangle_topology(std::int64_t node_count, const std::int64_t *node_tags,
                                    const double *node_xy, std::int64_t element_count,
                                    const std::int64_t *element_nodes) {
  if (element_count <= 0)
    throw std::runtime_error("triangle mesh: document contains no triangle elements");
  if (element_count > std::numeric_limits<std::int32_t>::max())
    throw std::runtime_error("triangle mesh: more elements than 32-bit indices address");
  const NodeIndex index(node_count, node_tags, "triangle mesh");
  TriTopology mesh;
  mesh.element_count = element_count;
  mesh.maps.resize(element_count);
  mesh.nodes.resize(3 * element_count);
  // Node positions of every element's vertices (after reorientation), and the
  // first failing element in element order, reported as a serial loop would.
  std::vector<std::int64_t> position(3 * element_count);
  std::atomic<std::int64_t> first_error{element_count};
  std::vector<std::string> messages(element_count > 0 ? 1 : 0);
  std::mutex message_lock;
  parallel_for(element_count, [&](std::int64_t begin, std::int64_t end) {
    for (std::int64_t e = begin; e < end; ++e) {
      std::int64_t tag[3], at[3];
      double x[3], y[3];
      std::string error;
      for (int k = 0; k < 3 && error.empty(); ++k) {
        tag[k] = element_nodes[3 * e + k];
        at[k] = index.find(tag[k]);
        if (at[k] < 0)
          error = "triangle mesh: element references missing node " + std::to_string(tag[k]);
        else
          x[k] = node_xy[2 * at[k]], y[k] = node_xy[2 * at[k] + 1];
      }
      if (error.empty()) {
        const double area2 = x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]);
        if (area2 == 0.0)
          error = "triangle mesh: zero-area element " + std::to_string(e + 1);
        else if (area2 < 0.0) {
          std::swap(x[1], x[2]);
          std::swap(y[1], y[2]);
          std::swap(tag[1], tag[2]);
          std::swap(at[1], at[2]);
        }
      }
      if (!error.empty()) {
        std::lock_guard<std::mutex> guard(message_lock);
        if (e < first_error.load()) {
          first_error.store(e);
          messages[0] = error;
        }
        return; // later elements of this range cannot come first
      }
      mesh.maps[e] = TriMap{x[0], y[0], x[1], y[1], x[2], y[2]};
      for (int k = 0; k < 3; ++k) {
        mesh.nodes[3 * e + k] = tag[k];
        position[3 * e + k] = at[k];
      }
    }
  });
  if (first_error.load() < element_count)
    throw std::runtime_error(messages[0]);

  // Edges matched through their smaller-tag endpoint: the element edges are
  // bucketed by that node (a counting sort, which keeps element order inside
  // a bucket), and a bucket's edges are grouped by the other endpoint.  An
  // edge's first element (by index, then local edge) is its left side, as
  // the reference's stable sort by (smaller tag, larger tag) makes it.
  const std::int64_t sides = 3 * element_count;
  std::vector<std::int64_t> low(sides), high(sides);
  for (std::int64_t e = 0; e < element_count; ++e)
    for (int k = 0; k < 3; ++k) {
      const int a = edge_vertices[k][0], b = edge_vertices[k][1];
      const bool a_first = mesh.nodes[3 * e + a] < mesh.nodes[3 * e + b];
      low[3 * e + k] = position[3 * e + (a_first ? a : b)];
      high[3 * e + k] = position[3 * e + (a_first ? b : a)];
    }
  std::vector<std::int64_t> start(node_count + 1, 0), bucket(sides);
  for (std::int64_t i = 0; i < sides; ++i)
    ++start[low[i] + 1];
  for (std::int64_t n = 0; n < node_count; ++n)
    start[n + 1] += start[n];
  {
    std::vector<std::int64_t> fill(start.begin(), start.end() - 1);
    for (std::int64_t i = 0; i < sides; ++i)
      bucket[fill[low[i]]++] = i;
  }
  // Per side: the other side of its face (-1: boundary, -2: not yet grouped)
  // and whether it is the face's left side.
  std::vector<std::int64_t> other(sides, -2);
  std::vector<std::uint8_t> is_left(sides, 0);
  std::int64_t worst_low = -1, worst_high = -1; // first edge, by tags, with > 2 sides
  for (std::int64_t n = 0; n < node_count; ++n)
    for (std::int64_t u = start[n]; u < start[n + 1]; ++u) {
      const std::int64_t i = bucket[u];
      if (other[i] != -2)
        continue;
      std::int64_t j = -1, extra = 0;
      for (std::int64_t w = u + 1; w < start[n + 1]; ++w) {
        const std::int64_t c = bucket[w];
        if (other[c] == -2 && high[c] == high[i]) {
          if (j < 0)
            j = c;
          else
            ++extra, other[c] = -1;
        }
      }
      if (extra > 0) {
        const std::int64_t lt = node_tags[low[i]], ht = node_tags[high[i]];
        if (worst_low < 0 || lt < worst_low || (lt == worst_low && ht < worst_high))
          worst_low = lt, worst_high = ht;
      }
      is_left[i] = 1;
      other[i] = j;
      if (j >= 0)
        other[j] = i;
    }
  if (worst_low >= 0)
    throw std::runtime_error("triangle mesh: edge " + std::to_string(worst_low) + "-" +
                             std::to_string(worst_high) +
                             " has more than two adjacent elements (non-conforming mesh)");

  // Faces in (left element, left local edge) order: the left sides in side order.
  std::int64_t nf = 0;
  for (std::int64_t i = 0; i < sides; ++i)
    nf += is_left[i];
  mesh.face_left.resize(nf);
  mesh.face_right.resize(nf);
  mesh.face_left_edge.resize(nf);
  mesh.face_right_edge.resize(nf);
  mesh.face_flip.resize(nf);
  mesh.face_nx.resize(nf);
  mesh.face_ny.resize(nf);
  mesh.face_scale.resize(nf);
  std::vector<std::int64_t> face_side(nf);
  for (std::int64_t i = 0, f = 0; i < sides; ++i)
    if (is_left[i])
      face_side[f++] = i;
  parallel_for(nf, [&](std::int64_t begin, std::int64_t end) {
    for (std::int64_t f = begin; f < end; ++f) {
      const std::int64_t i = face_side[f], j = other[i];
      const std::int32_t left = static_cast<std::int32_t>(i / 3), le = static_cast<std::int32_t>(i % 3);
      mesh.face_left[f] = left;
      mesh.face_left_edge[f] = le;
      if (j >= 0) {
        mesh.face_right[f] = static_cast<std::int32_t>(j / 3);
        mesh.face_right_edge[f] = static_cast<std::int32_t>(j % 3);
        // The two sides traverse the edge from different first vertices.
        mesh.face_flip[f] = static_cast<std::uint8_t>(
            mesh.nodes[3 * (i / 3) + edge_vertices[i % 3][0]] !=
            mesh.nodes[3 * (j / 3) + edge_vertices[j % 3][0]]);
      } else {
        mesh.face_right[f] = -1;
        mesh.face_right_edge[f] = 0;
        mesh.face_flip[f] = 0;
      }
      const TriMap &m = mesh.maps[left];
      m.edge_normal(le, mesh.face_nx[f], mesh.face_ny[f]);
      mesh.face_scale[f] = m.edge_length(le) / reference_edge_length(le);
    }
  });
  return mesh;
}

LineTopology build_line_topology(std::int64_t node_count, const std::int64_t *node_tags,
                                 const double *node_x, std::int64_t element_count,
                                 const std::int64_t *element_nodes) {
  if (element_count <= 0)
    throw std::runtime_error("line mesh: document contains no line elements");
  const NodeIndex index(node_count, node_tags, "line mesh");
  struct Segment {
    std::int64_t left_node, right_node;
    double xl, xr;
  };
  std::vector<Segment> segs(element_count);
  for (std::int64_t e = 0; e < element_count; ++e) {
    const std::int64_t ta = element_nodes[2 * e], tb = element_nodes[2 * e + 1];
    const std::int64_t a = index.find(ta), b = index.find(tb);
    if (a < 0 || b < 0)
      throw std::runtime_error("line mesh: element references missing node");
    const double xa = node_x[a], xb = node_x[b];
    if (xa == xb)
      throw std::runtime_error("line mesh: zero-length element " + std::to_string(e + 1));
    segs[e] = xa < xb ? Segment{ta, tb, xa, xb} : Segment{tb, ta, xb, xa};
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

Box bounding_box(const TriTopology &mesh) {
  Box b{std::numeric_limits<double>::max(), std::numeric_limits<double>::lowest(),
        std::numeric_limits<double>::max(), std::numeric_limits<double>::lowest()};
  for (const auto &m : mesh.maps) {
    b.min_x = std::min({b.min_x, m.x0, m.x1, m.x2});
    b.max_x = std::max({b.max_x, m.x0, m.x1, m.x2});
    b.min_y = std::min({b.min_y, m.y0, m.y1, m.y2});
    b.max_y = std::max({b.max_y, m.y0, m.y1, m.y2});
  }
  return b;
}


GridShape element_grid_shape(const TriTopology &mesh) {
  const Box box = bounding_box(mesh);
  GridShape g;
  g.x0 = box.min_x;
  g.y0 = box.min_y;
  const double n = std::max(1.0, std::sqrt(static_cast<double>(mesh.element_count) / 2.0));
  g.nx = g.ny = static_cast<int>(n);
  g.dx = std::max((box.max_x - box.min_x) / g.nx, 1e-300);
  g.dy = std::max((box.max_y - box.min_y) / g.ny, 1e-300);
  return g;
}

PeriodicImages periodic_images(const TriTopology &mesh, int p) {
  const int Q = p + 1;
  const Rule2D edges = triangle_edges(p);
  const Box box = bounding_box(mesh);
  PeriodicImages im;
  im.points = Q;
  for (std::int64_t f = 0; f < mesh.face_count(); ++f) {
    if (mesh.face_right[f] >= 0)
      continue;
    const double nx = mesh.face_nx[f], ny = mesh.face_ny[f];
    const bool along_x = std::fabs(nx) > 0.5 && std::fabs(ny) < 1e-10;
    const bool along_y = std::fabs(ny) > 0.5 && std::fabs(nx) < 1e-10;
    if (!along_x && !along_y) {
      // Reported after the donors of the faces before it, in face order.
      im.misaligned = true;
      break;
    }
    const TriMap &m = mesh.maps[mesh.face_left[f]];
    const int le = mesh.face_left_edge[f];
    for (int q = 0; q < Q; ++q) {
      double x = 0.0, y = 0.0;
      m.to_physical(edges.xi[le * Q + q], edges.eta[le * Q + q], x, y);
      if (along_x)
        x += nx < 0.0 ? box.max_x - box.min_x : box.min_x - box.max_x;
      else
        y += ny < 0.0 ? box.max_y - box.min_y : box.min_y - box.max_y;
      im.x.push_back(x);
      im.y.push_back(y);
    }
    ++im.faces;
  }
  return im;
}

ImageCells image_cells(const GridShape &g, const PeriodicImages &images) {
  const std::int64_t n = static_cast<std::int64_t>(images.x.size());
  std::vector<std::pair<int, std::int64_t>> by_cell(n);
  for (std::int64_t k = 0; k < n; ++k)
    by_cell[k] = {grid_cell(g, images.x[k], images.y[k]), k};
  std::sort(by_cell.begin(), by_cell.end());
  ImageCells ic;
  for (std::int64_t k = 0; k < n; ++k) {
    if (ic.cells.empty() || ic.cells.back() != by_cell[k].first) {
      ic.cells.push_back(by_cell[k].first);
      ic.start.push_back(k);
    }
    ic.point.push_back(by_cell[k].second);
  }
  ic.start.push_back(n);
  return ic;
}

PeriodicTrace periodic_trace_from_donors(const TriTopology &mesh, int p,
                                         const PeriodicImages &images,
                                         std::vector<std::int32_t> &&donors) {
  const int Q = images.points, M = tri_modes(p);
  PeriodicTrace trace;
  trace.basis.resize(static_cast<std::size_t>(images.faces) * Q * M);
  for (std::int64_t k = 0; k < images.faces * Q; ++k) {
    if (donors[k] < 0)
      throw std::runtime_error("simulation: periodic 2D trace has no donor element");
    double xi = 0.0, eta = 0.0;
    mesh.maps[donors[k]].to_reference(images.x[k], images.y[k], xi, eta);
    const auto b = dubiner(xi, eta, p);
    std::copy(b.begin(), b.end(), trace.basis.begin() + k * M);
  }
  if (images.misaligned)
    throw std::runtime_error("simulation: 2D periodic boundaries require an axis-aligned box");
  trace.donors = std::move(donors);
  return trace;
}

PeriodicTrace part_trace(const TriTopology &mesh, int p, const PartBoundary &part,
                         std::vector<std::int32_t> &stencil_donors) {
  const int Q = p + 1, M = tri_modes(p);
  const Rule2D edges = triangle_edges(p);
  std::int64_t faces = 0;
  for (std::int64_t f = 0; f < mesh.face_count(); ++f)
    faces += mesh.face_right[f] < 0;
  if (part.faces != faces)
    throw std::invalid_argument("partition boundary: " + std::to_string(part.faces) +
                                " faces given, the part's mesh has " + std::to_string(faces));
  if (faces > 0 && (!part.donors || !part.basis))
    throw std::invalid_argument("partition boundary: null donors or basis");
  PeriodicTrace trace;
  trace.donors.resize(static_cast<std::size_t>(faces) * Q);
  trace.basis.resize(static_cast<std::size_t>(faces) * Q * M);
  stencil_donors.assign(part.donors, part.donors + faces * Q);
  for (std::int64_t f = 0, b = 0; f < mesh.face_count(); ++f) {
    if (mesh.face_right[f] >= 0)
      continue;
    const bool own = part.donors[b * Q] == -1;
    for (int q = 0; q < Q; ++q) {
      const std::int32_t d = part.donors[b * Q + q];
      if (own ? d != -1 : (d < 0 || d >= mesh.element_count))
        throw std::invalid_argument("partition boundary: face " + std::to_string(b) +
                                    " has a donor outside the part or mixes owner points");
      std::vector<double> basis;
      if (own) {
        const int le = mesh.face_left_edge[f];
        basis = dubiner(edges.xi[le * Q + q], edges.eta[le * Q + q], p);
      } else {
        basis.assign(part.basis + (b * Q + q) * M, part.basis + (b * Q + q + 1) * M);
      }
      trace.donors[b * Q + q] = own ? mesh.face_left[f] : d;
      std::copy(basis.begin(), basis.end(), trace.basis.begin() + (b * Q + q) * M);
    }
    ++b;
  }
  return trace;
}

PeriodicTrace periodic_trace(const TriTopology &mesh, int p) {
  const PeriodicImages images = periodic_images(mesh, p);
  const std::int64_t n = static_cast<std::int64_t>(images.x.size());
  std::vector<std::int32_t> donors(n, -1);
  if (n > 0) {
    // Every element checks the image points in the cells its padded box
    // covers; a point's donor is the smallest element index that contains it,
    // which is the first candidate of its cell in ascending order.
    const GridShape g = element_grid_shape(mesh);
    const ImageCells ic = image_cells(g, images);
    std::vector<std::atomic<std::int32_t>> best(n);
    for (auto &b : best)
      b.store(std::numeric_limits<std::int32_t>::max());
    parallel_for(mesh.element_count, [&](std::int64_t begin, std::int64_t end) {
      for (std::int64_t e = begin; e < end; ++e) {
        const TriMap &m = mesh.maps[e];
        const double v[6] = {m.x0, m.y0, m.x1, m.y1, m.x2, m.y2};
        int i0, i1, j0, j1;
        grid_cell_range(g, v, i0, i1, j0, j1);
        for (int j = j0; j <= j1; ++j)
          for (int i = i0; i <= i1; ++i) {
            const auto it = std::lower_bound(ic.cells.begin(), ic.cells.end(), j * g.nx + i);
            if (it == ic.cells.end() || *it != j * g.nx + i)
              continue;
            const std::size_t r = static_cast<std::size_t>(it - ic.cells.begin());
            for (std::int64_t k = ic.start[r]; k < ic.start[r + 1]; ++k) {
              const std::int64_t pt = ic.point[k];
              double xi = 0.0, eta = 0.0;
              grid_to_reference(v, images.x[pt], images.y[pt], xi, eta);
              if (!grid_contains(xi, eta))
                continue;
              std::int32_t cur = best[pt].load();
              while (static_cast<std::int32_t>(e) < cur &&
                     !best[pt].compare_exchange_weak(cur, static_cast<std::int32_t>(e))) {
              }
            }
          }
      }
    });
    for (std::int64_t k = 0; k < n; ++k) {
      const std::int32_t b = best[k].load();
      donors[k] = b == std::numeric_limits<std::int32_t>::max() ? -1 : b;
    }
  }
  return periodic_trace_from_donors(mesh, p, images, std::move(donors));
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

// Check points: volume rule of order p, then the three edge rules
// (euler_limiter_stencil_triangle.cpp:81-93).
void fill_check_basis(LimiterStencil &s, int p) {
  const Rule2D rule = triangle_rule(p), edges = triangle_edges(p);
  for (int q = 0; q < rule.size(); ++q) {
    const auto b = dubiner(rule.xi[q], rule.eta[q], p);
    s.check_basis.insert(s.check_basis.end(), b.begin(), b.end());
  }
  for (int q = 0; q < edges.size(); ++q) {
    const auto b = dubiner(edges.xi[q], edges.eta[q], p);
    s.check_basis.insert(s.check_basis.end(), b.begin(), b.end());
  }
}

} // namespace

LimiterStencil triangle_stencil(const TriTopology &mesh, int p,
                                const std::vector<std::int32_t> &periodic_donors,
                                bool transforms) {
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
  std::int64_t b = 0; // boundary face ordinal
  for (std::int64_t f = 0; f < mesh.face_count(); ++f) {
    const std::int32_t left = mesh.face_left[f];
    std::int32_t right = mesh.face_right[f];
    const bool boundary = right < 0;
    if (boundary && !periodic_donors.empty())
      right = periodic_donors[b * Q];
    b += boundary;
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
  if (!transforms) {
    fill_check_basis(s, p);
    return s;
  }
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

  fill_check_basis(s, p);
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
      if (trace) {
        const std::int64_t b = t.boundary_count;
        t.donors.insert(t.donors.end(), trace->donors.begin() + b * QF,
                        trace->donors.begin() + (b + 1) * QF);
        t.donor_basis.insert(t.donor_basis.end(), trace->basis.begin() + b * QF * M,
                             trace->basis.begin() + (b + 1) * QF * M);
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
