// Host-side setup of the triangle solvers under AddressSanitizer and
// UndefinedBehaviorSanitizer (tests/test_host_sanitized.py compiles this file
// with the library's host sources and -fsanitize=address,undefined).
//
//   host_check <mesh file> <polynomial order> <periodic 0|1>
//
// The mesh file holds node count, element count (int64), node tags (int64),
// coordinates (2 doubles per node) and element nodes (3 int64 per element).
// Every setup step a solver runs on the host is exercised, and the arrays it
// produces are checked for consistency; the exit status is the number of
// failed checks (the sanitizers abort on their own findings).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <vector>

#include "mesh.hpp"
#include "tri_setup.hpp"
#include "wasl_b200.h"

using namespace wasl_b200;

namespace {

int failures = 0;

void check(bool ok, const char *what) {
  if (!ok) {
    std::fprintf(stderr, "check failed: %s\n", what);
    ++failures;
  }
}

template <typename T> std::vector<T> read(std::ifstream &in, std::size_t n) {
  std::vector<T> v(n);
  in.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(n * sizeof(T)));
  return v;
}

} // namespace

int main(int argc, char **argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: host_check <mesh file> <p> <periodic>\n");
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary);
  const auto counts = read<std::int64_t>(in, 2);
  const auto tags = read<std::int64_t>(in, counts[0]);
  const auto xy = read<double>(in, 2 * counts[0]);
  const auto cells = read<std::int64_t>(in, 3 * counts[1]);
  const int p = std::atoi(argv[2]), QF = p + 1, M = (p + 1) * (p + 2) / 2;
  const bool periodic = std::atoi(argv[3]) != 0;

  const TriTopology mesh = build_triangle_topology(counts[0], tags.data(), xy.data(), counts[1],
                                                   cells.data());
  const std::int64_t ne = mesh.element_count, nf = mesh.face_count();
  check(ne == counts[1], "element count");
  PeriodicTrace trace;
  if (periodic)
    trace = periodic_trace(mesh, p);
  TriSlots t = build_tri_slots(mesh, periodic ? &trace : nullptr, QF, M);
  for (std::int64_t e = 0; e < ne; ++e)
    for (int k = 0; k < 3; ++k) {
      const std::int32_t f = t.slot_face[k * ne + e];
      check(f >= 0 && f < nf, "slot face in range");
      check(mesh.face_left[f] == e || mesh.face_right[f] == e, "slot face touches its element");
    }
  if (periodic) {
    std::vector<float> basis32;
    check(pair_periodic_faces(mesh, QF, t, basis32), "periodic faces pair");
  }
  const TileSlotArrays ts = build_tile_slots(mesh, t, periodic ? WASL_PERIODIC : WASL_TRANSMISSIVE,
                                             QF);
  check(ts.nbr.size() == static_cast<std::size_t>(3 * ne), "tile slot size");
  PatchEdgeArrays pe;
  check(build_patch_edges(mesh, t, periodic ? WASL_PERIODIC : WASL_TRANSMISSIVE, QF, pe),
        "patch edges built");
  for (std::int64_t e = 0; e < ne; ++e)
    for (int j = 0; j < 3; ++j) {
      const std::int32_t nb = pe.nbr[j * ne + e];
      if (nb < 0) {
        check(!periodic && (pe.info[j * ne + e] & 1u), "boundary edge is its own left side");
        continue;
      }
      const int jn = (pe.info[j * ne + e] >> 1) & 3;
      check(pe.nbr[jn * ne + nb] == e, "the neighbour's edge points back");
      check(((pe.info[j * ne + e] ^ pe.info[jn * ne + nb]) & 1u) == 1u,
            "exactly one side of a face is its left side");
      check(((pe.info[j * ne + e] ^ pe.info[jn * ne + nb]) & 8u) == 0u,
            "both sides agree on the point order");
      for (int r = 0; r < 3; ++r)
        check(pe.geo[(3 * j + r) * ne + e] == pe.geo[(3 * jn + r) * ne + nb],
              "both sides hold the face's normal and scale");
    }
  const std::vector<std::int32_t> order = morton_order(mesh);
  std::vector<char> seen(ne, 0);
  for (const std::int32_t e : order) {
    check(e >= 0 && e < ne && !seen[e], "the Morton order is a permutation");
    if (e >= 0 && e < ne)
      seen[e] = 1;
  }
  const LimiterStencil st = triangle_stencil(mesh, p, trace.donors);
  for (const std::int32_t n : st.neighbors)
    check(n >= -1 && n < ne, "stencil neighbour in range");
  check(st.transforms.size() == static_cast<std::size_t>(ne) * 3 * M * M, "transform size");
  check(std::isfinite(minimum_altitude(mesh)) && minimum_altitude(mesh) > 0.0, "altitude");
  // The L2 projection of a constant is that constant's mode 0 only.
  const int rule = std::max(p, 5), Q = (rule + 1) * (rule + 1);
  std::vector<double> values(static_cast<std::size_t>(ne) * Q, 2.5);
  const std::vector<double> c = tri_project(mesh, p, 1, rule, values.data());
  for (std::int64_t e = 0; e < ne; ++e) {
    check(std::fabs(c[e] - 2.5 * std::sqrt(2.0)) < 1e-12, "projected mean");
    for (int m = 1; m < M; ++m)
      check(std::fabs(c[m * ne + e]) < 1e-12, "projected high modes vanish");
  }
  std::printf("host setup checked: %lld elements, P%d, %s, %d failures\n",
              static_cast<long long>(ne), p, periodic ? "periodic" : "transmissive", failures);
  return failures;
}
