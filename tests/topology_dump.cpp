// Writes the library's triangle topology (mesh.cpp build_triangle_topology)
// for tests/test_host_topology.py:
//
//   topology_dump <mesh file> <output file>
//
// The mesh file is host_check.cpp's format.  The output holds the element
// count, face count, then vertices [element][6], nodes [element][3], and per
// face: left, right, left edge, right edge (int32), flip (uint8), normal x,
// normal y, scale (double); or "ERR <message>" when the build throws.
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <vector>

#include "mesh.hpp"

using namespace wasl_b200;

namespace {
template <typename T> std::vector<T> read(std::ifstream &in, std::size_t n) {
  std::vector<T> v(n);
  in.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(n * sizeof(T)));
  return v;
}
template <typename T> void write(FILE *f, const std::vector<T> &v) {
  std::fwrite(v.data(), sizeof(T), v.size(), f);
}
} // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: topology_dump <mesh file> <output file>\n");
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary);
  const auto counts = read<std::int64_t>(in, 2);
  const auto tags = read<std::int64_t>(in, counts[0]);
  const auto xy = read<double>(in, 2 * counts[0]);
  const auto cells = read<std::int64_t>(in, 3 * counts[1]);
  FILE *out = std::fopen(argv[2], "wb");
  if (!out)
    return 2;
  try {
    const TriTopology m =
        build_triangle_topology(counts[0], tags.data(), xy.data(), counts[1], cells.data());
    const std::int64_t sizes[2] = {m.element_count, m.face_count()};
    std::fwrite(sizes, sizeof sizes[0], 2, out);
    write(out, m.maps);
    write(out, m.nodes);
    write(out, m.face_left);
    write(out, m.face_right);
    write(out, m.face_left_edge);
    write(out, m.face_right_edge);
    write(out, m.face_flip);
    write(out, m.face_nx);
    write(out, m.face_ny);
    write(out, m.face_scale);
  } catch (const std::exception &e) {
    std::fprintf(out, "ERR %s", e.what());
  }
  std::fclose(out);
  return 0;
}
