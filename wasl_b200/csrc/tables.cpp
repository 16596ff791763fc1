// Host construction of the per-order face tables the triangle kernels read.
#include <cstring>
#include <stdexcept>

#include "kernels.hpp"
#include "tri_tables.hpp"

namespace wasl_b200 {

namespace {
template <int P, typename T> void fill_as(void *out) {
  static FaceTable<P, T> table;
  fill_face_table<P, T>(table);
  std::memcpy(out, &table, sizeof(table));
}
template <int P> std::size_t bytes(bool fp32) {
  return fp32 ? sizeof(FaceTable<P, float>) : sizeof(FaceTable<P, double>);
}
} // namespace

std::size_t euler_tri_face_table_bytes(int p, bool fp32) {
  switch (p) {
  case 0: return bytes<0>(fp32);
  case 1: return bytes<1>(fp32);
  case 2: return bytes<2>(fp32);
  case 3: return bytes<3>(fp32);
  default: throw std::invalid_argument("triangle polynomial order must be 0..3");
  }
}

void fill_euler_tri_face_table(int p, bool fp32, void *out) {
  switch (p) {
  case 0: fp32 ? fill_as<0, float>(out) : fill_as<0, double>(out); break;
  case 1: fp32 ? fill_as<1, float>(out) : fill_as<1, double>(out); break;
  case 2: fp32 ? fill_as<2, float>(out) : fill_as<2, double>(out); break;
  case 3: fp32 ? fill_as<3, float>(out) : fill_as<3, double>(out); break;
  default: throw std::invalid_argument("triangle polynomial order must be 0..3");
  }
}

} // namespace wasl_b200
