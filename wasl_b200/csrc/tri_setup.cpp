// Host-side setup shared by the triangle solvers (see tri_setup.hpp).
#include "tri_setup.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <map>
#include <utility>

#include "../../include/wasl_b200.h"
#include "basis.hpp"
#include "parallel.hpp"

namespace wasl_b200 {

bool pair_periodic_faces(const TriTopology &mesh, int QF, TriSlots &t, std::vector<float> &basis32) {
  const std::int64_t ne = mesh.element_count;
  std::vector<std::int64_t> bface;
  for (std::int64_t f = 0; f < mesh.face_count(); ++f)
    if (mesh.face_right[f] < 0)
      bface.push_back(f);
  const std::size_t nb = bface.size();
  if (t.donors.size() != nb * QF)
    return false;
  // A face whose donor is its own element (the cut face of a partition
  // part, which takes its own trace) has no partner and stays unpaired.
  std::vector<std::int32_t> bdonor(nb);
  std::vector<char> own(nb, 0);
  std::map<std::pair<std::int32_t, std::int32_t>, std::vector<std::size_t>> by_pair;
  for (std::size_t b = 0; b < nb; ++b) {
    bdonor[b] = t.donors[b * QF];
    for (int q = 1; q < QF; ++q)
      if (t.donors[b * QF + q] != bdonor[b])
        return false;
    own[b] = bdonor[b] == mesh.face_left[bface[b]];
    if (!own[b])
      by_pair[{mesh.face_left[bface[b]], bdonor[b]}].push_back(b);
  }
  std::vector<std::size_t> partner(nb);
  for (std::size_t b = 0; b < nb; ++b) {
    if (own[b])
      continue;
    const auto it = by_pair.find({bdonor[b], mesh.face_left[bface[b]]});
    if (it == by_pair.end() || it->second.size() != 1)
      return false;
    partner[b] = it->second[0];
    if (partner[b] == b)
      return false;
  }
  for (std::size_t b = 0; b < nb; ++b)
    if (!own[b] && partner[partner[b]] != b)
      return false;
  for (std::size_t b = 0; b < nb; ++b) {
    if (own[b])
      continue;
    const std::int64_t f = bface[b], c = bface[partner[b]];
    if (f < c)
      continue; // f is the kept face of its pair
    t.face_code[f] |= 0x80u;
    const std::int32_t e = mesh.face_left[f];
    const std::int64_t k = t.left_slot[f];
    t.slot_face[k * ne + e] = static_cast<std::int32_t>(c);
    t.slot_code[k * ne + e] = static_cast<std::uint8_t>((mesh.face_left_edge[c] << 1) | 0x40u);
    t.slot_geo[(3 * k) * ne + e] = mesh.face_nx[c];
    t.slot_geo[(3 * k + 1) * ne + e] = mesh.face_ny[c];
    t.slot_geo[(3 * k + 2) * ne + e] = mesh.face_scale[c];
  }
  basis32.assign(t.donor_basis.begin(), t.donor_basis.end());
  return true;
}

TileSlotArrays build_tile_slots(const TriTopology &mesh, const TriSlots &t, int boundary, int QF) {
  const std::int64_t ne = mesh.element_count;
  TileSlotArrays s;
  s.nbr.resize(3 * ne);
  s.aux.assign(3 * ne, 0);
  s.code.resize(3 * ne);
  for (int k = 0; k < 3; ++k)
    for (std::int64_t e = 0; e < ne; ++e) {
      const std::int64_t slot = k * ne + e;
      const std::int64_t f = t.slot_face[slot];
      const std::int32_t L = mesh.face_left[f], R = t.face_right[f];
      const unsigned bits = (static_cast<unsigned>(mesh.face_left_edge[f]) << 1) |
                            (static_cast<unsigned>(mesh.face_right_edge[f]) << 3) |
                            (static_cast<unsigned>(mesh.face_flip[f]) << 5);
      const bool left = L == e;
      if (R >= 0) {
        s.nbr[slot] = left ? R : L;
        s.code[slot] = static_cast<std::uint8_t>(bits | (left ? 1u : 0u));
      } else if (boundary == WASL_TRANSMISSIVE) {
        s.nbr[slot] = -1;
        s.code[slot] = static_cast<std::uint8_t>(bits | 1u);
      } else if (left && t.donors[static_cast<std::size_t>(-R - 1) * QF] == L) {
        // A face that takes its own element's trace (a partition part's cut
        // face): the kernels' transmissive face.
        s.nbr[slot] = -1;
        s.code[slot] = static_cast<std::uint8_t>(bits | 1u);
      } else {
        const std::int32_t b = -R - 1;
        s.aux[slot] = b;
        if (left) {
          s.nbr[slot] = t.donors[static_cast<std::size_t>(b) * QF];
          s.code[slot] = static_cast<std::uint8_t>(bits | 1u | 0x80u);
        } else {
          s.nbr[slot] = L;
          s.code[slot] = static_cast<std::uint8_t>(bits | 0x40u);
        }
      }
    }
  return s;
}

namespace {

// Whether element b's points on local edge jb run opposite to element a's on
// edge ja (point QF-1-q of b is point q of a); points compared relative to
// each edge's midpoint, so periodic images match too.  -1: no match.
constexpr int kMaxEdgePoints = 8; // Gauss points per edge, order <= 7

int point_order(const TriTopology &mesh, const Rule2D &edges, int QF, std::int64_t a, int ja,
                std::int64_t b, int jb) {
  double ax[kMaxEdgePoints], ay[kMaxEdgePoints], bx[kMaxEdgePoints], by[kMaxEdgePoints];
  double amx = 0.0, amy = 0.0, bmx = 0.0, bmy = 0.0;
  for (int q = 0; q < QF; ++q) {
    mesh.maps[a].to_physical(edges.xi[ja * QF + q], edges.eta[ja * QF + q], ax[q], ay[q]);
    mesh.maps[b].to_physical(edges.xi[jb * QF + q], edges.eta[jb * QF + q], bx[q], by[q]);
    amx += ax[q] / QF, amy += ay[q] / QF, bmx += bx[q] / QF, bmy += by[q] / QF;
  }
  const double tolerance = 1e-9 * mesh.maps[a].edge_length(ja);
  double error[2] = {0.0, 0.0};
  for (int q = 0; q < QF; ++q)
    for (int rev = 0; rev < 2; ++rev) {
      const int qb = rev ? QF - 1 - q : q;
      error[rev] = std::max(error[rev], std::hypot((ax[q] - amx) - (bx[qb] - bmx),
                                                   (ay[q] - amy) - (by[qb] - bmy)));
    }
  const int rev = error[1] < error[0] ? 1 : 0;
  return error[rev] <= tolerance ? rev : -1;
}

} // namespace

bool build_patch_edges(const TriTopology &mesh, const TriSlots &t, int boundary, int QF,
                       PatchEdgeArrays &out) {
  const std::int64_t ne = mesh.element_count, nf = mesh.face_count();
  const Rule2D edges = triangle_edges(QF - 1);
  out.nbr.assign(3 * ne, -2);
  out.info.assign(3 * ne, 0);
  out.geo.assign(9 * ne, 0.0);
  auto set = [&](std::int64_t e, int j, std::int32_t nbr, unsigned info, std::int64_t f) {
    out.nbr[j * ne + e] = nbr;
    out.info[j * ne + e] = static_cast<std::uint8_t>(info);
    out.geo[(3 * j) * ne + e] = mesh.face_nx[f];
    out.geo[(3 * j + 1) * ne + e] = mesh.face_ny[f];
    out.geo[(3 * j + 2) * ne + e] = mesh.face_scale[f];
  };
  // Boundary faces in boundary order, and each one's partner across the period.
  std::vector<std::int64_t> bface;
  for (std::int64_t f = 0; f < nf; ++f)
    if (mesh.face_right[f] < 0)
      bface.push_back(f);
  std::map<std::pair<std::int32_t, std::int32_t>, std::vector<std::size_t>> by_pair;
  const bool periodic = boundary != WASL_TRANSMISSIVE && !bface.empty();
  if (periodic) {
    if (t.donors.size() != bface.size() * QF)
      return false;
    for (std::size_t b = 0; b < bface.size(); ++b)
      if (t.donors[b * QF] != mesh.face_left[bface[b]])
        by_pair[{mesh.face_left[bface[b]], t.donors[b * QF]}].push_back(b);
  }
  if (QF > kMaxEdgePoints)
    return false;
  // Interior faces (each writes only its two sides' slots), on all threads.
  std::atomic<bool> matched{true};
  parallel_for(nf, [&](std::int64_t begin, std::int64_t end) {
    for (std::int64_t f = begin; f < end; ++f) {
      const std::int32_t L = mesh.face_left[f], R = mesh.face_right[f];
      if (R < 0)
        continue;
      const int jl = mesh.face_left_edge[f], jr = mesh.face_right_edge[f];
      const int rev = point_order(mesh, edges, QF, L, jl, R, jr);
      if (rev < 0) {
        matched = false;
        return;
      }
      set(L, jl, R, 1u | (jr << 1) | (rev << 3), f);
      set(R, jr, L, (jl << 1) | (rev << 3), f);
    }
  });
  if (!matched)
    return false;
  for (std::int64_t f = 0, b = 0; f < nf; ++f) {
    const std::int32_t L = mesh.face_left[f], R = mesh.face_right[f];
    const int jl = mesh.face_left_edge[f];
    if (R >= 0)
      continue;
    const std::size_t bi = static_cast<std::size_t>(b++);
    if (!periodic) {
      set(L, jl, -1, 1u, f);
      continue;
    }
    const std::int32_t D = t.donors[bi * QF];
    for (int q = 1; q < QF; ++q)
      if (t.donors[bi * QF + q] != D)
        return false;
    if (D == L) { // takes its own trace (a partition part's cut face)
      set(L, jl, -1, 1u, f);
      continue;
    }
    const auto it = by_pair.find({D, L});
    if (it == by_pair.end() || it->second.size() != 1 || it->second[0] == bi)
      return false;
    const std::int64_t c = bface[it->second[0]];
    if (c < f)
      continue; // the partner is the kept face of the pair
    const int jd = mesh.face_left_edge[c];
    const int rev = point_order(mesh, edges, QF, L, jl, D, jd);
    if (rev < 0)
      return false;
    set(L, jl, D, 1u | (jd << 1) | (rev << 3), f);
    set(D, jd, L, (jl << 1) | (rev << 3), f);
  }
  for (const std::int32_t n : out.nbr)
    if (n == -2)
      return false;
  return true;
}

std::vector<std::int32_t> morton_order(const TriTopology &mesh) {
  const std::int64_t ne = mesh.element_count;
  std::vector<double> cx(ne), cy(ne);
  double x0 = 0.0, y0 = 0.0, x1 = 0.0, y1 = 0.0;
  for (std::int64_t e = 0; e < ne; ++e) {
    const TriMap &m = mesh.maps[e];
    cx[e] = (m.x0 + m.x1 + m.x2) / 3.0;
    cy[e] = (m.y0 + m.y1 + m.y2) / 3.0;
    x0 = e ? std::min(x0, cx[e]) : cx[e], x1 = e ? std::max(x1, cx[e]) : cx[e];
    y0 = e ? std::min(y0, cy[e]) : cy[e], y1 = e ? std::max(y1, cy[e]) : cy[e];
  }
  const double extent = std::max(x1 - x0, y1 - y0);
  const double scale = extent > 0.0 ? 65535.0 / extent : 0.0;
  // 16 bits per axis, interleaved (x in the even bits).
  auto spread = [](std::uint32_t v) {
    std::uint64_t x = v & 0xffffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
  };
  std::vector<std::uint64_t> key(ne);
  for (std::int64_t e = 0; e < ne; ++e) {
    const auto qx = static_cast<std::uint32_t>((cx[e] - x0) * scale);
    const auto qy = static_cast<std::uint32_t>((cy[e] - y0) * scale);
    key[e] = spread(qx) | (spread(qy) << 1);
  }
  std::vector<std::int32_t> order(ne);
  for (std::int64_t e = 0; e < ne; ++e)
    order[e] = static_cast<std::int32_t>(e);
  std::stable_sort(order.begin(), order.end(),
                   [&](std::int32_t a, std::int32_t b) { return key[a] < key[b]; });
  return order;
}

void tri_quadrature(const TriTopology &mesh, int rule_order, double *x, double *y, double *w) {
  const Rule2D rule = triangle_rule(rule_order);
  const int Q = rule.size();
  for (std::int64_t e = 0; e < mesh.element_count; ++e) {
    const TriMap &m = mesh.maps[e];
    const double jac = std::fabs(m.jacobian_determinant());
    for (int q = 0; q < Q; ++q) {
      m.to_physical(rule.xi[q], rule.eta[q], x[e * Q + q], y[e * Q + q]);
      if (w)
        w[e * Q + q] = rule.w[q] * jac;
    }
  }
}

std::vector<double> tri_project(const TriTopology &mesh, int p, int variables, int rule_order,
                                const double *values) {
  const Rule2D rule = triangle_rule(rule_order);
  const int Q = rule.size();
  const int M = (p + 1) * (p + 2) / 2;
  const std::int64_t ne = mesh.element_count;
  std::vector<std::vector<double>> basis(Q);
  for (int q = 0; q < Q; ++q)
    basis[q] = dubiner(rule.xi[q], rule.eta[q], p);
  std::vector<double> c(static_cast<std::size_t>(variables) * M * ne, 0.0);
  for (std::int64_t e = 0; e < ne; ++e)
    for (int q = 0; q < Q; ++q) {
      const double *val = values + (e * Q + q) * variables;
      for (int v = 0; v < variables; ++v)
        for (int m = 0; m < M; ++m)
          c[(static_cast<std::int64_t>(v) * M + m) * ne + e] += rule.w[q] * val[v] * basis[q][m];
    }
  return c;
}

void tri_evaluate(const TriTopology &mesh, int p, int variables, int rule_order,
                  const double *c, double *values) {
  const Rule2D rule = triangle_rule(rule_order);
  const int Q = rule.size();
  const int M = (p + 1) * (p + 2) / 2;
  const std::int64_t ne = mesh.element_count;
  std::vector<std::vector<double>> basis(Q);
  for (int q = 0; q < Q; ++q)
    basis[q] = dubiner(rule.xi[q], rule.eta[q], p);
  for (std::int64_t e = 0; e < ne; ++e)
    for (int q = 0; q < Q; ++q)
      for (int v = 0; v < variables; ++v) {
        double s = 0.0;
        for (int m = 0; m < M; ++m)
          s += c[(static_cast<std::int64_t>(v) * M + m) * ne + e] * basis[q][m];
        values[(e * Q + q) * variables + v] = s;
      }
}

} // namespace wasl_b200
