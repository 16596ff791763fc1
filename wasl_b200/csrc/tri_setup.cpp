// Host-side setup shared by the triangle solvers (see tri_setup.hpp).
#include "tri_setup.hpp"

#include <cmath>
#include <map>
#include <utility>

#include "../../include/wasl_b200.h"
#include "basis.hpp"

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
  std::vector<std::int32_t> bdonor(nb);
  std::map<std::pair<std::int32_t, std::int32_t>, std::vector<std::size_t>> by_pair;
  for (std::size_t b = 0; b < nb; ++b) {
    bdonor[b] = t.donors[b * QF];
    for (int q = 1; q < QF; ++q)
      if (t.donors[b * QF + q] != bdonor[b])
        return false;
    by_pair[{mesh.face_left[bface[b]], bdonor[b]}].push_back(b);
  }
  std::vector<std::size_t> partner(nb);
  for (std::size_t b = 0; b < nb; ++b) {
    const auto it = by_pair.find({bdonor[b], mesh.face_left[bface[b]]});
    if (it == by_pair.end() || it->second.size() != 1)
      return false;
    partner[b] = it->second[0];
    if (partner[b] == b)
      return false;
  }
  for (std::size_t b = 0; b < nb; ++b)
    if (partner[partner[b]] != b)
      return false;
  for (std::size_t b = 0; b < nb; ++b) {
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
